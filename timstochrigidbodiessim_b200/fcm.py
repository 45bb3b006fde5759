"""Python mirror of the reference's C++ interface over the C-ABI.

``Suspension`` owns one ``fcm_ctx`` (one suspension on one GPU).  Its methods
carry the names of the reference's methods (fcm_fluid_solver,
collection_of_rigid_bodies, linked_list, gmres_solver); the thin classes at the
end expose the same methods under the reference's class names.  Inputs may be
numpy arrays (host) or CUDA torch tensors (device); outputs are numpy arrays
unless an ``out=`` tensor is given.
"""
import ctypes

import numpy as np

from . import capi
from .params import FcmMcmcState, FcmParams, FcmStepInfo


def _in(a, n, dtype=np.float64):
    """(keep-alive object, pointer) for an input array of n elements."""
    if a is None:
        return None, None
    if hasattr(a, "data_ptr"):  # torch tensor
        assert a.is_contiguous() and a.numel() == n, (a.shape, n)
        return a, ctypes.c_void_p(a.data_ptr())
    arr = np.ascontiguousarray(a, dtype=dtype)
    assert arr.size == n, (arr.size, n)
    return arr, ctypes.c_void_p(arr.ctypes.data)


def _out(out, n, dtype=np.float64):
    if out is not None:
        if hasattr(out, "data_ptr"):
            assert out.is_contiguous() and out.numel() == n
            return out, ctypes.c_void_p(out.data_ptr())
        assert out.size == n and out.dtype == dtype and out.flags.c_contiguous
        return out, ctypes.c_void_p(out.ctypes.data)
    arr = np.zeros(n, dtype=dtype)
    return arr, ctypes.c_void_p(arr.ctypes.data)


class Suspension:
    """One suspension of rigid multi-blob bodies on the GPU."""

    def __init__(self, params: FcmParams, blob_ref_pos, stream=None, _handle=None):
        self.L = capi.load()
        self.p = params.copy()
        self.M = params.num_bodies
        self.nb = params.blobs_per_body
        self.Nb = params.num_blobs
        self.n = params.system_size
        self.P = params.nx * params.ny * params.pad
        self._owned = _handle is None
        if _handle is None:
            keep, ref = _in(blob_ref_pos, 3 * self.nb)
            h = ctypes.c_void_p()
            capi.check(self.L.fcm_create(ctypes.byref(self.p), ref, ctypes.byref(h)), "fcm_create")
            self.h = h
        else:  # a member of a Batch, owned by it
            self.h = ctypes.c_void_p(_handle)
        if stream is not None:
            self.set_stream(stream)

    def close(self):
        if getattr(self, "h", None):
            if self._owned:
                self.L.fcm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, st, where, ok=(0,)):
        return capi.check(st, where, ok)

    def set_stream(self, stream):
        """stream: a torch.cuda.Stream or a raw cudaStream_t integer."""
        s = getattr(stream, "cuda_stream", stream)
        self._c(self.L.fcm_set_stream(self.h, ctypes.c_void_p(int(s))), "fcm_set_stream")

    # -------------------------------------------------- collection_of_rigid_bodies
    def set_bodies(self, x, q):
        kx, px = _in(x, 3 * self.M)
        kq, pq = _in(q, 4 * self.M)
        self._c(self.L.fcm_set_bodies(self.h, px, pq), "fcm_set_bodies")

    def get_bodies(self):
        x, px = _out(None, 3 * self.M)
        q, pq = _out(None, 4 * self.M)
        self._c(self.L.fcm_get_bodies(self.h, px, pq), "fcm_get_bodies")
        return x, q

    def get_midstep_bodies(self):
        x, px = _out(None, 3 * self.M)
        q, pq = _out(None, 4 * self.M)
        self._c(self.L.fcm_get_midstep_bodies(self.h, px, pq), "fcm_get_midstep_bodies")
        return x, q

    def set_external_forces(self, fe):
        k, p = _in(fe, 6 * self.M)
        self._c(self.L.fcm_set_external_forces(self.h, p), "fcm_set_external_forces")

    def fill_all_blob_pos(self, at_midstep=False):
        self._c(self.L.fcm_fill_all_blob_pos(self.h, int(at_midstep)), "fcm_fill_all_blob_pos")

    def set_all_blob_pos(self, Y):
        k, p = _in(Y, 3 * self.Nb)
        self._c(self.L.fcm_set_all_blob_pos(self.h, p), "fcm_set_all_blob_pos")

    def get_all_blob_pos(self, out=None):
        Y, p = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_get_all_blob_pos(self.h, p), "fcm_get_all_blob_pos")
        return Y

    def multiply_by_K_at_midstep(self, U, out=None):
        k, pi = _in(U, 6 * self.M)
        o, po = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_multiply_by_K_at_midstep(self.h, pi, po), "fcm_multiply_by_K_at_midstep")
        return o

    def multiply_by_KT_at_midstep(self, lam, out=None):
        k, pi = _in(lam, 3 * self.Nb)
        o, po = _out(out, 6 * self.M)
        self._c(self.L.fcm_multiply_by_KT_at_midstep(self.h, pi, po), "fcm_multiply_by_KT_at_midstep")
        return o

    def calculate_forces(self):
        self._c(self.L.fcm_calculate_forces(self.h), "fcm_calculate_forces")

    def get_blob_forces(self, out=None):
        F, p = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_get_blob_forces(self.h, p), "fcm_get_blob_forces")
        return F

    def set_blob_forces(self, F):
        k, p = _in(F, 3 * self.Nb)
        self._c(self.L.fcm_set_blob_forces(self.h, p), "fcm_set_blob_forces")

    def advance_to_midstep(self, V=None):
        k, p = _in(V, 3 * self.Nb)
        ov = ctypes.c_int32(0)
        self._c(self.L.fcm_advance_to_midstep(self.h, p, ctypes.byref(ov)), "fcm_advance_to_midstep")
        return bool(ov.value)

    def calculate_divU(self):
        d = ctypes.c_double(0.0)
        self._c(self.L.fcm_calculate_divU(self.h, ctypes.byref(d)), "fcm_calculate_divU")
        return d.value

    def end_of_step_update(self, U, nu=1.0):
        k, p = _in(U, 6 * self.M)
        ov = ctypes.c_int32(0)
        self._c(self.L.fcm_end_of_step_update(self.h, p, float(nu), ctypes.byref(ov)), "fcm_end_of_step_update")
        return bool(ov.value)

    def reset_to_start_of_step(self):
        self._c(self.L.fcm_reset_to_start_of_step(self.h), "fcm_reset_to_start_of_step")

    def check_for_overlap(self):
        ov = ctypes.c_int32(0)
        self._c(self.L.fcm_check_for_overlap(self.h, ctypes.byref(ov)), "fcm_check_for_overlap")
        return bool(ov.value)

    def check_for_channel_wall_overlap(self):
        """collection_of_rigid_bodies.cpp:207-239 (False without a slip channel)."""
        ov = ctypes.c_int32(0)
        self._c(self.L.fcm_check_for_channel_wall_overlap(self.h, ctypes.byref(ov)),
                "fcm_check_for_channel_wall_overlap")
        return bool(ov.value)

    # -------------------------------------------------- linked_list
    def list_populate(self):
        self._c(self.L.fcm_list_populate(self.h), "fcm_list_populate")

    def list_get_cells(self):
        c, p = _out(None, self.Nb, np.int32)
        self._c(self.L.fcm_list_get_cells(self.h, p), "fcm_list_get_cells")
        return c

    def list_get_pairs(self):
        n = ctypes.c_int64(0)
        self._c(self.L.fcm_list_get_pairs(self.h, None, 0, ctypes.byref(n)), "fcm_list_get_pairs")
        out = np.zeros(2 * max(n.value, 1), dtype=np.int32)
        n2 = ctypes.c_int64(0)
        self._c(self.L.fcm_list_get_pairs(self.h, ctypes.c_void_p(out.ctypes.data), n.value, ctypes.byref(n2)),
                "fcm_list_get_pairs")
        return out[: 2 * n2.value].reshape(-1, 2)

    def apply_barrier_forces(self, F=None):
        F = np.zeros(3 * self.Nb) if F is None else np.array(F, dtype=np.float64)
        self._c(self.L.fcm_apply_barrier_forces(self.h, ctypes.c_void_p(F.ctypes.data)), "fcm_apply_barrier_forces")
        return F

    # -------------------------------------------------- fcm_fluid_solver
    def set_up_gaussians(self, Y=None):
        k, p = _in(Y, 3 * self.Nb)
        self._c(self.L.fcm_set_up_gaussians(self.h, p), "fcm_set_up_gaussians")

    def get_gaussians(self, precision=0, width=None):
        """(indices, weights) of the last set_up_gaussians on the grid of one
        precision, each (Nb, 3, W): the reference's indx/indy/indz and
        gaussx/y/z.  W is ngauss for FP64; pass `width` for the FP32 grid."""
        W = self.p.ngauss if width is None else width
        ind = np.zeros(self.Nb * 3 * W, dtype=np.int32)
        w = np.zeros(self.Nb * 3 * W)
        self._c(self.L.fcm_get_gaussians(self.h, precision, ind.ctypes.data, w.ctypes.data), "fcm_get_gaussians")
        return ind.reshape(self.Nb, 3, W), w.reshape(self.Nb, 3, W)

    def produce_random_velocity_field(self, seed, counter):
        self._c(self.L.fcm_produce_random_velocity_field(self.h, seed, counter), "fcm_produce_random_velocity_field")

    def inject_random_stress(self, s6):
        ks = [_in(s, self.P) for s in s6]
        self._c(self.L.fcm_inject_random_stress(self.h, *[p for _, p in ks]), "fcm_inject_random_stress")

    def calculate_random_blob_velocities(self, out=None):
        V, p = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_calculate_random_blob_velocities(self.h, p), "fcm_calculate_random_blob_velocities")
        return V

    def set_up_force_distribution(self, F):
        k, p = _in(F, 3 * self.Nb)
        self._c(self.L.fcm_set_up_force_distribution(self.h, p), "fcm_set_up_force_distribution")

    def produce_deterministic_velocity_field(self):
        self._c(self.L.fcm_produce_deterministic_velocity_field(self.h), "fcm_produce_deterministic_velocity_field")

    def calculate_deterministic_blob_velocities(self, out=None):
        V, p = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_calculate_deterministic_blob_velocities(self.h, p),
                "fcm_calculate_deterministic_blob_velocities")
        return V

    def get_V(self, out=None):
        V, p = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_get_V(self.h, p), "fcm_get_V")
        return V

    def get_velocity_field(self, which=0):
        outs = [np.zeros(self.P) for _ in range(3)]
        self._c(self.L.fcm_get_velocity_field(self.h, which, *[ctypes.c_void_p(o.ctypes.data) for o in outs]),
                "fcm_get_velocity_field")
        return outs

    def apply_mobility(self, F, out=None):
        k, p = _in(F, 3 * self.Nb)
        V, po = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_apply_mobility(self.h, p, po), "fcm_apply_mobility")
        return V

    # -------------------------------------------------- shear forcing (SHEARING_FORCES)
    def produce_shear_velocity_field(self, scale=1.0, wavenumber=1.0):
        """fcm_fluid_solver.cpp:703-842 with SHEAR_FORCE_SCALE = scale and
        SHEAR_WAVENUMBER = wavenumber; later RHS assemblies subtract Vshear and
        GDC steps interpolate it at the midstep."""
        self._c(self.L.fcm_produce_shear_velocity_field(self.h, float(scale), float(wavenumber)),
                "fcm_produce_shear_velocity_field")

    def calculate_shear_blob_velocities(self, out=None):
        """fcm_fluid_solver.cpp:489-550: Vshear (3Nb) on the current Gaussians."""
        V, p = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_calculate_shear_blob_velocities(self.h, p), "fcm_calculate_shear_blob_velocities")
        return V

    def fluid_x_velocity_in_y(self, F):
        """main.cpp:371-433: mean over x and z of ux + ux_shear for every y index,
        ux the flow of blob forces F on the current Gaussians."""
        k, p = _in(F, 3 * self.Nb)
        prof = np.zeros(self.p.ny)
        self._c(self.L.fcm_fluid_x_velocity_in_y(self.h, p, ctypes.c_void_p(prof.ctypes.data)),
                "fcm_fluid_x_velocity_in_y")
        return prof

    # -------------------------------------------------- Metropolis Monte Carlo (main.cpp:113-210)
    def calculate_potential(self):
        U = ctypes.c_double(0.0)
        self._c(self.L.fcm_calculate_potential(self.h, ctypes.byref(U)), "fcm_calculate_potential")
        return U.value

    def mcmc_state(self):
        """The reference's starting state: scale 0.1a, acceptance ratio 0.5."""
        st = FcmMcmcState()
        self._c(self.L.fcm_mcmc_state_init(self.h, ctypes.byref(st)), "fcm_mcmc_state_init")
        return st

    def mcmc_run(self, seed, n_steps, state=None):
        """n_steps Metropolis steps on the device; returns the updated state."""
        st = self.mcmc_state() if state is None else state
        self._c(self.L.fcm_mcmc_run(self.h, seed, n_steps, ctypes.byref(st)), "fcm_mcmc_run")
        return st

    # Force dipoles (no reference counterpart): F, T (3 per blob), S (9 per blob).
    def set_up_dipole_distribution(self, F=None, T=None, S=None):
        kf, pf = _in(F, 3 * self.Nb)
        kt, pt = _in(T, 3 * self.Nb)
        ks, ps = _in(S, 9 * self.Nb)
        self._c(self.L.fcm_set_up_dipole_distribution(self.h, pf, pt, ps), "fcm_set_up_dipole_distribution")

    def calculate_deterministic_blob_rotations(self):
        """(Omega (3Nb), E (9Nb)) of the deterministic velocity grid."""
        Om, po = _out(None, 3 * self.Nb)
        E, pe = _out(None, 9 * self.Nb)
        self._c(self.L.fcm_calculate_deterministic_blob_rotations(self.h, po, pe),
                "fcm_calculate_deterministic_blob_rotations")
        return Om, E

    # The stages of apply_mobility one at a time, on the FP64 (0) or FP32 (1) grid.
    def spread(self, F, precision=0):
        k, p = _in(F, 3 * self.Nb)
        self._c(self.L.fcm_spread(self.h, precision, p), "fcm_spread")

    def stokes_solve(self, precision=0):
        self._c(self.L.fcm_stokes_solve(self.h, precision), "fcm_stokes_solve")

    def interp(self, precision=0, out=None):
        V, po = _out(out, 3 * self.Nb)
        self._c(self.L.fcm_interp(self.h, precision, po), "fcm_interp")
        return V

    # kernel variants: [FP64 spread, FP64 solve, FP32 spread, FP32 solve, FP64
    # interp, FP32 interp]; spread 0 = persistent pipelined, 1 / 2 / 3 = one CTA
    # per tile staging 16 / 8 / 32 blobs per round, 4 = one warp per tile (two
    # y-rows per lane), 5 = one warp per tile on the tensor cores (FP32 only);
    # solve 0 = cuFFT 3D, 1 = cuFFT (y, z) + fused x-transform, 2 = the library's
    # (y, z) + fused x; interp 0 = shuffle reduction, 64 threads per tile, 1 =
    # one warp per tile (two y-rows per lane) with the shuffle reduction, 2 = one
    # warp per tile with a shared-memory reduction, 3 = one warp per tile on the
    # tensor cores (FP32 only)
    NUM_VARIANTS = 6
    NUM_TUNE_TIMES = 32

    def get_variants(self):
        v, pv = _out(None, self.NUM_VARIANTS, np.int32)
        self._c(self.L.fcm_get_variants(self.h, pv), "fcm_get_variants")
        return [int(x) for x in v]

    def set_variants(self, variants):
        v, pv = _in(variants, self.NUM_VARIANTS, np.int32)
        self._c(self.L.fcm_set_variants(self.h, pv), "fcm_set_variants")

    def autotune(self, reps=5):
        """Time every variant the grids allow and keep the fastest.  Returns
        (variants, us): us[16 P + v] microseconds per call for precision P, v = 0-5
        spread variants, 6, 7, 8 solve variants, 9-12 interpolation variants
        (-1 where not available; v = 13-15 unused)."""
        us, pu = _out(None, self.NUM_TUNE_TIMES)
        v, pv = _out(None, self.NUM_VARIANTS, np.int32)
        self._c(self.L.fcm_autotune(self.h, reps, pu, pv), "fcm_autotune")
        return [int(x) for x in v], us

    def produce_reference_matrices(self):
        self._c(self.L.fcm_produce_reference_matrices(self.h), "fcm_produce_reference_matrices")

    def get_reference_matrices(self):
        n3 = 3 * self.nb
        Minv = np.zeros(n3 * n3); N = np.zeros(36); KTKinv = np.zeros(36)
        self._c(self.L.fcm_get_reference_matrices(self.h, *[ctypes.c_void_p(a.ctypes.data) for a in (Minv, N, KTKinv)]),
                "fcm_get_reference_matrices")
        return (Minv.reshape(n3, n3, order="F"), N.reshape(6, 6, order="F"), KTKinv.reshape(6, 6, order="F"))

    def set_reference_matrices(self, Minv, N):
        a = np.ascontiguousarray(np.asarray(Minv).ravel(order="F"), dtype=np.float64)
        b = np.ascontiguousarray(np.asarray(N).ravel(order="F"), dtype=np.float64)
        self._c(self.L.fcm_set_reference_matrices(self.h, ctypes.c_void_p(a.ctypes.data), ctypes.c_void_p(b.ctypes.data)),
                "fcm_set_reference_matrices")

    # -------------------------------------------------- gmres_solver
    def set_body_shapes(self, shapes):
        """Per-body reference blob positions (M, nb, 3) or 3*nb*M; each body gets
        its own ref_KTKinv and the analytic FCM preconditioner blocks."""
        k, p = _in(shapes, 3 * self.nb * self.M)
        self._c(self.L.fcm_set_body_shapes(self.h, p), "fcm_set_body_shapes")

    def set_body_preconditioners(self, Minv=None, N=None):
        n3 = 3 * self.nb
        km, pm = _in(Minv, n3 * n3 * self.M)
        kn, pn = _in(N, 36 * self.M)
        self._c(self.L.fcm_set_body_preconditioners(self.h, pm, pn), "fcm_set_body_preconditioners")

    def get_body_preconditioners(self):
        """(Minv (M, 3nb, 3nb), N (M, 6, 6), KTKinv (M, 6, 6)); each block as
        stored (column-major), returned transposed into row-major numpy order."""
        n3 = 3 * self.nb
        Minv = np.zeros(self.M * n3 * n3)
        N = np.zeros(36 * self.M)
        K = np.zeros(36 * self.M)
        self._c(self.L.fcm_get_body_preconditioners(self.h, Minv.ctypes.data, N.ctypes.data, K.ctypes.data),
                "fcm_get_body_preconditioners")
        return (Minv.reshape(self.M, n3, n3).transpose(0, 2, 1), N.reshape(self.M, 6, 6).transpose(0, 2, 1),
                K.reshape(self.M, 6, 6).transpose(0, 2, 1))

    def assemble_RHS(self):
        self._c(self.L.fcm_assemble_RHS(self.h), "fcm_assemble_RHS")

    def get_RHS(self, out=None):
        r, p = _out(out, self.n)
        self._c(self.L.fcm_get_RHS(self.h, p), "fcm_get_RHS")
        return r

    def set_RHS(self, r):
        k, p = _in(r, self.n)
        self._c(self.L.fcm_set_RHS(self.h, p), "fcm_set_RHS")

    def multiply_by_Pinv(self, v, out=None):
        k, pi = _in(v, self.n)
        o, po = _out(out, self.n)
        self._c(self.L.fcm_multiply_by_Pinv(self.h, pi, po), "fcm_multiply_by_Pinv")
        return o

    def multiply_by_saddle_point_matrix(self, v, out=None):
        k, pi = _in(v, self.n)
        o, po = _out(out, self.n)
        self._c(self.L.fcm_multiply_by_saddle_point_matrix(self.h, pi, po), "fcm_multiply_by_saddle_point_matrix")
        return o

    def invert_saddle_point_system(self, out=None):
        """Returns (status, solution, iterations, relative residual); status is
        FCM_OK or FCM_ERR_NOT_CONVERGED (the iterate is still returned)."""
        o, po = _out(out, self.n)
        it = ctypes.c_int32(0)
        rel = ctypes.c_double(0.0)
        st = self.L.fcm_invert_saddle_point_system(self.h, po, ctypes.byref(it), ctypes.byref(rel))
        self._c(st, "fcm_invert_saddle_point_system", ok=(0, 5))
        return st, o, it.value, rel.value

    # -------------------------------------------------- time step
    def step(self, seed, step_index):
        """One time step (main.cpp:222-451); returns (status, FcmStepInfo);
        status FCM_ERR_OVERLAP means the step was rejected and bodies restored."""
        info = FcmStepInfo()
        st = self.L.fcm_step(self.h, seed, step_index, ctypes.byref(info))
        self._c(st, "fcm_step", ok=(0, 7))
        return st, info

    def step_async(self, seed, step_index):
        """Issue a step without waiting (a CUDA-graph launch after the first step)."""
        self._c(self.L.fcm_step_async(self.h, seed, step_index), "fcm_step_async")

    def step_wait(self):
        """Wait for the step issued by step_async; returns (status, FcmStepInfo)."""
        info = FcmStepInfo()
        st = self.L.fcm_step_wait(self.h, ctypes.byref(info))
        self._c(st, "fcm_step_wait", ok=(0, 7))
        return st, info


class Batch:
    """Many independent suspensions stepped together (fcm_batch_*): members[i]
    is a Suspension view of member i (owned by the batch)."""

    def __init__(self, members, stream=None):
        """members: list of (FcmParams, blob_ref_pos)."""
        self.L = capi.load()
        n = len(members)
        self.n = n
        self._params = (FcmParams * n)(*[p.copy() for p, _ in members])
        self._refs = [np.ascontiguousarray(r, dtype=np.float64).ravel() for _, r in members]
        ptrs = (ctypes.c_void_p * n)(*[r.ctypes.data for r in self._refs])
        h = ctypes.c_void_p()
        capi.check(self.L.fcm_batch_create(n, self._params, ptrs, ctypes.byref(h)), "fcm_batch_create")
        self.h = h
        self.members = [Suspension(p, r, _handle=self.L.fcm_batch_member(h, i))
                        for i, (p, r) in enumerate(members)]
        if stream is not None:
            self.set_stream(stream)

    def set_stream(self, stream):
        s = getattr(stream, "cuda_stream", stream)
        capi.check(self.L.fcm_batch_set_stream(self.h, ctypes.c_void_p(int(s))), "fcm_batch_set_stream")

    def step(self, seeds, step_index):
        """One step of every member; returns the list of FcmStepInfo."""
        sd = (ctypes.c_uint64 * self.n)(*[int(x) for x in seeds])
        infos = (FcmStepInfo * self.n)()
        capi.check(self.L.fcm_batch_step(self.h, sd, step_index, infos), "fcm_batch_step")
        return list(infos)

    def last_rounds(self):
        """(lockstep GMRES iterations, refinement sweeps) of the last graph step."""
        r = (ctypes.c_int32 * 2)()
        capi.check(self.L.fcm_batch_last_rounds(self.h, r), "fcm_batch_last_rounds")
        return int(r[0]), int(r[1])

    def close(self):
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None
            self.L.fcm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def step_many(suspensions, seeds, step_index):
    """One step of each suspension (fcm_step_many): all issued, then all awaited.
    Returns the list of FcmStepInfo."""
    n = len(suspensions)
    L = suspensions[0].L if n else capi.load()
    hs = (ctypes.c_void_p * n)(*[s.h.value for s in suspensions])
    sd = (ctypes.c_uint64 * n)(*[int(x) for x in seeds])
    infos = (FcmStepInfo * n)()
    st = L.fcm_step_many(hs, n, sd, step_index, infos)
    capi.check(st, "fcm_step_many", (0,))
    return list(infos)


class fft_solver:
    """fft_solver.hpp:10-31 on the GPU (in-place transforms of padded arrays)."""

    def __init__(self, nx, ny, nz):
        self.L = capi.load()
        self.nx, self.ny, self.nz = nx, ny, nz
        h = ctypes.c_void_p()
        capi.check(self.L.fcm_fft_create(nx, ny, nz, ctypes.byref(h)), "fcm_fft_create")
        self.h = h
        a = [ctypes.c_int32() for _ in range(4)]
        tot = ctypes.c_int64()
        pad = ctypes.c_int32()
        capi.check(self.L.fcm_fft_local_sizes(self.h, *[ctypes.byref(x) for x in a], ctypes.byref(tot),
                                              ctypes.byref(pad)), "fcm_fft_local_sizes")
        (self.local_nx, self.local_x_start, self.local_ny_after_transpose,
         self.local_y_start_after_transpose) = [x.value for x in a]
        self.total_local_size = tot.value
        self.pad = pad.value

    def transform(self, arr):
        assert arr.dtype == np.float64 and arr.flags.c_contiguous and arr.size == self.total_local_size
        capi.check(self.L.fcm_fft_transform(self.h, ctypes.c_void_p(arr.ctypes.data)), "fcm_fft_transform")

    def inverse_transform(self, arr):
        assert arr.dtype == np.float64 and arr.flags.c_contiguous and arr.size == self.total_local_size
        capi.check(self.L.fcm_fft_inverse_transform(self.h, ctypes.c_void_p(arr.ctypes.data)),
                   "fcm_fft_inverse_transform")

    def __del__(self):
        try:
            if self.h:
                self.L.fcm_fft_destroy(self.h)
                self.h = None
        except Exception:
            pass
