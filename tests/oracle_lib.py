"""ctypes wrapper of the CPU FP64 oracle (oracle/liboracle.so), test side only.

The oracle is the checker: a CPU restatement of the reference's FCM path (see
oracle/fcm_oracle.cpp).  Method names follow the reference's classes.
"""
import ctypes
import os
import subprocess

import numpy as np

from timstochrigidbodiessim_b200.params import FcmMcmcState, FcmParams, FcmStepInfo

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")

_lib = None

D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)


def build_oracle():
    subprocess.run(["make", "-s", "-C", ORACLE_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = ctypes.CDLL(ORACLE_SO)
        vp = ctypes.c_void_p
        sig = {
            "orc_set_threads": (None, [ctypes.c_int]),
            "orc_get_threads": (ctypes.c_int, []),
            "orc_fft_transform": (ctypes.c_int, [ctypes.c_int] * 3 + [D]),
            "orc_fft_inverse_transform": (ctypes.c_int, [ctypes.c_int] * 3 + [D]),
            "orc_create": (vp, [ctypes.POINTER(FcmParams), D]),
            "orc_destroy": (None, [vp]),
            "orc_set_bodies": (None, [vp, D, D]),
            "orc_get_bodies": (None, [vp, D, D]),
            "orc_get_midstep_bodies": (None, [vp, D, D]),
            "orc_set_external_forces": (None, [vp, D]),
            "orc_fill_all_blob_pos": (None, [vp, ctypes.c_int]),
            "orc_set_all_blob_pos": (None, [vp, D]),
            "orc_get_all_blob_pos": (None, [vp, D]),
            "orc_multiply_by_K_at_midstep": (None, [vp, D, D]),
            "orc_multiply_by_KT_at_midstep": (None, [vp, D, D]),
            "orc_calculate_forces": (None, [vp]),
            "orc_get_blob_forces": (None, [vp, D]),
            "orc_set_blob_forces": (None, [vp, D]),
            "orc_advance_to_midstep": (ctypes.c_int, [vp, D]),
            "orc_calculate_divU": (ctypes.c_double, [vp]),
            "orc_end_of_step_update": (ctypes.c_int, [vp, D, ctypes.c_double]),
            "orc_reset_to_start_of_step": (None, [vp]),
            "orc_check_for_overlap": (ctypes.c_int, [vp]),
            "orc_list_populate": (None, [vp]),
            "orc_list_get_cells": (None, [vp, I32]),
            "orc_list_get_pairs": (ctypes.c_int64, [vp, I32, ctypes.c_int64]),
            "orc_apply_barrier_forces": (None, [vp, D]),
            "orc_set_up_gaussians": (None, [vp, D]),
            "orc_get_gaussians": (None, [vp, I32, D]),
            "orc_inject_random_stress": (None, [vp, D, D, D, D, D, D]),
            "orc_produce_random_velocity_field": (None, [vp, ctypes.c_uint64, ctypes.c_uint64]),
            "orc_calculate_random_blob_velocities": (None, [vp, D]),
            "orc_set_up_force_distribution": (None, [vp, D]),
            "orc_produce_deterministic_velocity_field": (None, [vp]),
            "orc_calculate_deterministic_blob_velocities": (None, [vp, D]),
            "orc_set_up_dipole_distribution": (None, [vp, D, D, D]),
            "orc_calculate_potential": (ctypes.c_double, [vp]),
            "orc_produce_shear_velocity_field": (None, [vp, ctypes.c_double, ctypes.c_double]),
            "orc_calculate_shear_blob_velocities": (None, [vp, D]),
            "orc_fluid_x_velocity_in_y": (None, [vp, D, D]),
            "orc_mcmc_run": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(FcmMcmcState)]),
            "orc_calculate_deterministic_blob_rotations": (None, [vp, D, D]),
            "orc_get_V": (None, [vp, D]),
            "orc_get_grid": (None, [vp, ctypes.c_int, D]),
            "orc_produce_reference_matrices": (None, [vp]),
            "orc_get_reference_matrices": (None, [vp, D, D, D]),
            "orc_set_reference_matrices": (None, [vp, D, D]),
            "orc_set_body_shapes": (None, [vp, D]),
            "orc_set_body_preconditioners": (None, [vp, D, D]),
            "orc_get_body_preconditioners": (None, [vp, D, D, D]),
            "orc_produce_body_preconditioners": (None, [vp]),
            "orc_set_sequential_noise": (None, [vp, ctypes.c_int, ctypes.c_uint64, ctypes.c_uint64]),
            "orc_assemble_RHS": (None, [vp]),
            "orc_get_RHS": (None, [vp, D]),
            "orc_set_RHS": (None, [vp, D]),
            "orc_multiply_by_Pinv": (None, [vp, D, D]),
            "orc_multiply_by_saddle_point_matrix": (None, [vp, D, D]),
            "orc_invert_saddle_point_system": (ctypes.c_int, [vp, D, I32, D]),
            "orc_step": (ctypes.c_int, [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(FcmStepInfo)]),
            "orc_step_injected": (ctypes.c_int, [vp, D, ctypes.POINTER(FcmStepInfo)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(D)


def _f64(a, n=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if n is not None:
        assert a.size == n, (a.size, n)
    return a


def fft_transform(nx, ny, nz, arr):
    """fft_solver::transform on a padded real array (returns a new array)."""
    a = _f64(arr).copy()
    lib().orc_fft_transform(nx, ny, nz, _dp(a))
    return a


def fft_inverse_transform(nx, ny, nz, arr):
    a = _f64(arr).copy()
    lib().orc_fft_inverse_transform(nx, ny, nz, _dp(a))
    return a


class Oracle:
    """One suspension on the CPU oracle."""

    def __init__(self, params: FcmParams, blob_ref_pos):
        self.p = params
        self.ref = _f64(blob_ref_pos, 3 * params.blobs_per_body)
        self.h = lib().orc_create(ctypes.byref(params), _dp(self.ref))
        if not self.h:
            raise ValueError("orc_create rejected the parameters")
        self.M = params.num_bodies
        self.nb = params.blobs_per_body
        self.Nb = params.num_blobs
        self.n = params.system_size
        self.P = params.nx * params.ny * params.pad

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # collection_of_rigid_bodies
    def set_bodies(self, x, q):
        lib().orc_set_bodies(self.h, _dp(_f64(x, 3 * self.M)), _dp(_f64(q, 4 * self.M)))

    def get_bodies(self):
        x = np.zeros(3 * self.M); q = np.zeros(4 * self.M)
        lib().orc_get_bodies(self.h, _dp(x), _dp(q))
        return x, q

    def get_midstep_bodies(self):
        x = np.zeros(3 * self.M); q = np.zeros(4 * self.M)
        lib().orc_get_midstep_bodies(self.h, _dp(x), _dp(q))
        return x, q

    def set_external_forces(self, fe):
        if fe is None:
            lib().orc_set_external_forces(self.h, None)
        else:
            lib().orc_set_external_forces(self.h, _dp(_f64(fe, 6 * self.M)))

    def fill_all_blob_pos(self, at_midstep=False):
        lib().orc_fill_all_blob_pos(self.h, int(at_midstep))

    def set_all_blob_pos(self, Y):
        lib().orc_set_all_blob_pos(self.h, _dp(_f64(Y, 3 * self.Nb)))

    def get_all_blob_pos(self):
        Y = np.zeros(3 * self.Nb)
        lib().orc_get_all_blob_pos(self.h, _dp(Y))
        return Y

    def multiply_by_K_at_midstep(self, U):
        out = np.zeros(3 * self.Nb)
        lib().orc_multiply_by_K_at_midstep(self.h, _dp(_f64(U, 6 * self.M)), _dp(out))
        return out

    def multiply_by_KT_at_midstep(self, lam):
        out = np.zeros(6 * self.M)
        lib().orc_multiply_by_KT_at_midstep(self.h, _dp(_f64(lam, 3 * self.Nb)), _dp(out))
        return out

    def calculate_forces(self):
        lib().orc_calculate_forces(self.h)

    def get_blob_forces(self):
        F = np.zeros(3 * self.Nb)
        lib().orc_get_blob_forces(self.h, _dp(F))
        return F

    def set_blob_forces(self, F):
        lib().orc_set_blob_forces(self.h, _dp(_f64(F, 3 * self.Nb)))

    def advance_to_midstep(self, V=None):
        return lib().orc_advance_to_midstep(self.h, None if V is None else _dp(_f64(V, 3 * self.Nb)))

    def calculate_divU(self):
        return lib().orc_calculate_divU(self.h)

    def end_of_step_update(self, U, nu=1.0):
        return lib().orc_end_of_step_update(self.h, _dp(_f64(U, 6 * self.M)), float(nu))

    def reset_to_start_of_step(self):
        lib().orc_reset_to_start_of_step(self.h)

    def check_for_overlap(self):
        return lib().orc_check_for_overlap(self.h)

    # linked_list
    def list_populate(self):
        lib().orc_list_populate(self.h)

    def list_get_cells(self):
        c = np.zeros(self.Nb, dtype=np.int32)
        lib().orc_list_get_cells(self.h, c.ctypes.data_as(I32))
        return c

    def list_get_pairs(self):
        n = lib().orc_list_get_pairs(self.h, None, 0)
        out = np.zeros(2 * max(n, 1), dtype=np.int32)
        lib().orc_list_get_pairs(self.h, out.ctypes.data_as(I32), n)
        return out[: 2 * n].reshape(-1, 2)

    def apply_barrier_forces(self, F=None):
        F = np.zeros(3 * self.Nb) if F is None else _f64(F, 3 * self.Nb).copy()
        lib().orc_apply_barrier_forces(self.h, _dp(F))
        return F

    # fcm_fluid_solver
    def set_up_gaussians(self, Y=None):
        lib().orc_set_up_gaussians(self.h, None if Y is None else _dp(_f64(Y, 3 * self.Nb)))

    def get_gaussians(self):
        W = self.p.ngauss
        ind = np.zeros(self.Nb * 3 * W, dtype=np.int32)
        w = np.zeros(self.Nb * 3 * W)
        lib().orc_get_gaussians(self.h, ind.ctypes.data_as(I32), _dp(w))
        return ind.reshape(self.Nb, 3, W), w.reshape(self.Nb, 3, W)

    def inject_random_stress(self, s6):
        s6 = [_f64(s, self.P) for s in s6]
        lib().orc_inject_random_stress(self.h, *[_dp(s) for s in s6])

    def produce_random_velocity_field(self, seed, counter):
        lib().orc_produce_random_velocity_field(self.h, seed, counter)

    def set_sequential_noise(self, on, seed=0, stream=0):
        """Noise from one stream continued across calls (the SPRNG stream of one
        reference rank); on=False returns to per-plane streams."""
        lib().orc_set_sequential_noise(self.h, int(bool(on)), seed, stream)

    def calculate_random_blob_velocities(self):
        V = np.zeros(3 * self.Nb)
        lib().orc_calculate_random_blob_velocities(self.h, _dp(V))
        return V

    def set_up_force_distribution(self, F):
        lib().orc_set_up_force_distribution(self.h, _dp(_f64(F, 3 * self.Nb)))

    def produce_deterministic_velocity_field(self):
        lib().orc_produce_deterministic_velocity_field(self.h)

    def calculate_deterministic_blob_velocities(self):
        V = np.zeros(3 * self.Nb)
        lib().orc_calculate_deterministic_blob_velocities(self.h, _dp(V))
        return V

    def calculate_potential(self):
        return lib().orc_calculate_potential(self.h)

    def get_V(self):
        V = np.zeros(3 * self.Nb)
        lib().orc_get_V(self.h, _dp(V))
        return V

    def produce_shear_velocity_field(self, scale=1.0, wavenumber=1.0):
        """fcm_fluid_solver.cpp:703-842 with SHEAR_FORCE_SCALE and SHEAR_WAVENUMBER."""
        lib().orc_produce_shear_velocity_field(self.h, float(scale), float(wavenumber))

    def calculate_shear_blob_velocities(self):
        Vs = np.zeros(3 * self.Nb)
        lib().orc_calculate_shear_blob_velocities(self.h, _dp(Vs))
        return Vs

    def fluid_x_velocity_in_y(self, F):
        prof = np.zeros(self.p.ny)
        lib().orc_fluid_x_velocity_in_y(self.h, _dp(_f64(F, 3 * self.Nb)), _dp(prof))
        return prof

    def mcmc_run(self, seed, n_steps, state=None):
        """Metropolis steps (main.cpp:113-210); state defaults to the reference's start."""
        if state is None:
            state = FcmMcmcState(scale=0.1 * self.p.blob_radius, acceptance_ratio=0.5)
        st = lib().orc_mcmc_run(self.h, seed, n_steps, ctypes.byref(state))
        return st, state

    def set_up_dipole_distribution(self, F=None, T=None, S=None):
        """Forces, torques and stresslets (9 per blob) spread together (no reference code)."""
        arr = [None if v is None else _f64(v, (9 if k == 2 else 3) * self.Nb) for k, v in enumerate((F, T, S))]
        lib().orc_set_up_dipole_distribution(self.h, *[None if a is None else _dp(a) for a in arr])

    def calculate_deterministic_blob_rotations(self):
        """(Omega (3Nb), E (9Nb)) of the deterministic field."""
        Om = np.zeros(3 * self.Nb)
        E = np.zeros(9 * self.Nb)
        lib().orc_calculate_deterministic_blob_rotations(self.h, _dp(Om), _dp(E))
        return Om, E

    def apply_mobility(self, F):
        self.set_up_force_distribution(F)
        self.produce_deterministic_velocity_field()
        return self.calculate_deterministic_blob_velocities()

    def get_grid(self, which):
        g = np.zeros(self.P)
        lib().orc_get_grid(self.h, which, _dp(g))
        return g

    def produce_reference_matrices(self):
        lib().orc_produce_reference_matrices(self.h)

    def get_reference_matrices(self):
        n3 = 3 * self.p.blobs_per_body
        Minv = np.zeros(n3 * n3); N = np.zeros(36); KTKinv = np.zeros(36)
        lib().orc_get_reference_matrices(self.h, _dp(Minv), _dp(N), _dp(KTKinv))
        return (Minv.reshape(n3, n3, order="F"), N.reshape(6, 6, order="F"),
                KTKinv.reshape(6, 6, order="F"))

    def set_reference_matrices(self, Minv, N):
        lib().orc_set_reference_matrices(self.h, _dp(_f64(np.asarray(Minv).ravel(order="F"))),
                                         _dp(_f64(np.asarray(N).ravel(order="F"))))

    # gmres_solver
    def set_body_shapes(self, shapes):
        lib().orc_set_body_shapes(self.h, _dp(_f64(shapes, 3 * self.nb * self.M)))

    def produce_body_preconditioners(self):
        lib().orc_produce_body_preconditioners(self.h)

    def set_body_preconditioners(self, Minv=None, N=None):
        n3 = 3 * self.nb
        m = _f64(Minv, n3 * n3 * self.M) if Minv is not None else None
        n = _f64(N, 36 * self.M) if N is not None else None
        lib().orc_set_body_preconditioners(self.h, _dp(m) if m is not None else None,
                                           _dp(n) if n is not None else None)

    def get_body_preconditioners(self):
        """(Minv, N, KTKinv) as flat column-major blocks, body after body."""
        n3 = 3 * self.nb
        Minv = np.zeros(n3 * n3 * self.M)
        N = np.zeros(36 * self.M)
        K = np.zeros(36 * self.M)
        lib().orc_get_body_preconditioners(self.h, _dp(Minv), _dp(N), _dp(K))
        return Minv, N, K

    def assemble_RHS(self):
        lib().orc_assemble_RHS(self.h)

    def get_RHS(self):
        r = np.zeros(self.n)
        lib().orc_get_RHS(self.h, _dp(r))
        return r

    def set_RHS(self, r):
        lib().orc_set_RHS(self.h, _dp(_f64(r, self.n)))

    def multiply_by_Pinv(self, v):
        out = np.zeros(self.n)
        lib().orc_multiply_by_Pinv(self.h, _dp(_f64(v, self.n)), _dp(out))
        return out

    def multiply_by_saddle_point_matrix(self, v):
        out = np.zeros(self.n)
        lib().orc_multiply_by_saddle_point_matrix(self.h, _dp(_f64(v, self.n)), _dp(out))
        return out

    def invert_saddle_point_system(self):
        soln = np.zeros(self.n)
        it = ctypes.c_int32(0)
        rel = ctypes.c_double(0.0)
        st = lib().orc_invert_saddle_point_system(self.h, _dp(soln), ctypes.byref(it), ctypes.byref(rel))
        return st, soln, it.value, rel.value

    def step(self, seed, step_index):
        info = FcmStepInfo()
        st = lib().orc_step(self.h, seed, step_index, ctypes.byref(info))
        return st, info

    def step_injected(self, s6):
        s = np.concatenate([_f64(x, self.P) for x in s6])
        info = FcmStepInfo()
        st = lib().orc_step_injected(self.h, _dp(s), ctypes.byref(info))
        return st, info
