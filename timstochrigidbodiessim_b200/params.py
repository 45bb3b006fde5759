"""ctypes mirror of ``fcm_params`` / ``fcm_step_info`` (include/fcm_b200.h).

The fields are the runtime replacements of the reference's compile-time macros
(config.hpp:8-116); defaults follow config.hpp with SLIP_CHANNEL false and
SIMULATION_ALGORITHM 2 (Euler-Maruyama).
"""
import ctypes
import math

PI = 3.14159265358979323846264338327950288  # config.hpp:86


class FcmParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("ngauss", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("blob_radius", ctypes.c_double),
        ("viscosity", ctypes.c_double),
        ("kT", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("num_bodies", ctypes.c_int32),
        ("blobs_per_body", ctypes.c_int32),
        ("ncells", ctypes.c_int32),
        ("potential", ctypes.c_int32),
        ("steric_fs", ctypes.c_double),
        ("steric_rc", ctypes.c_double),
        ("gmres_max_iter", ctypes.c_int32),
        ("gmres_tol", ctypes.c_double),
        ("fd_delta", ctypes.c_double),
        ("algorithm", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("noise", ctypes.c_int32),
        ("skip_on_overlap", ctypes.c_int32),
        ("slip_channel", ctypes.c_int32),
    ]

    @classmethod
    def defaults(cls, **kw):
        """config.hpp defaults (DX = a/(1.86 sqrt(pi)), DT = pi eta a^3/kT/100)."""
        a, eta, kT = 1.0, 1.0, 1.0
        p = cls(nx=256, ny=256, nz=256, ngauss=20,
                dx=a * 0.3033277330901916, blob_radius=a, viscosity=eta, kT=kT,
                dt=(PI * eta * a ** 3 / kT) / 100.0,
                num_bodies=3, blobs_per_body=22, ncells=6, potential=0,
                steric_fs=40.0 * kT / a, steric_rc=2.2 * a,
                gmres_max_iter=40, gmres_tol=1e-3, fd_delta=1e-5,
                algorithm=2, precision=0, noise=1, skip_on_overlap=0, slip_channel=0)
        for k, v in kw.items():
            if not hasattr(p, k):
                raise AttributeError(k)
            setattr(p, k, v)
        return p

    def copy(self, **kw):
        q = FcmParams()
        ctypes.pointer(q)[0] = self
        for k, v in kw.items():
            if not hasattr(q, k):
                raise AttributeError(k)
            setattr(q, k, v)
        return q

    @property
    def box(self):
        return (self.dx * self.nx, self.dx * self.ny, self.dx * self.nz)

    @property
    def num_blobs(self):
        return self.num_bodies * self.blobs_per_body

    @property
    def system_size(self):
        return 3 * self.num_blobs + 6 * self.num_bodies

    @property
    def pad(self):
        return 2 * (self.nz // 2 + 1)

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FcmMcmcState(ctypes.Structure):
    """fcm_mcmc_state: a Metropolis run's state, carried across calls."""
    _fields_ = [
        ("scale", ctypes.c_double),
        ("acceptance_ratio", ctypes.c_double),
        ("potential", ctypes.c_double),
        ("steps", ctypes.c_int64),
        ("attempts", ctypes.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class FcmStepInfo(ctypes.Structure):
    _fields_ = [
        ("gmres_iters", ctypes.c_int32),
        ("refinement_sweeps", ctypes.c_int32),
        ("gmres_rel_residual", ctypes.c_double),
        ("divU", ctypes.c_double),
        ("overlap", ctypes.c_int32),
        ("status", ctypes.c_int32),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


# status codes (enum fcm_status)
FCM_OK = 0
FCM_ERR_INVALID = 1
FCM_ERR_CUDA = 2
FCM_ERR_CUFFT = 3
FCM_ERR_STATE = 4
FCM_ERR_NOT_CONVERGED = 5
FCM_ERR_NONFINITE = 6
FCM_ERR_OVERLAP = 7
FCM_ERR_NOMEM = 8
FCM_ERR_CAPACITY = 9

STATUS_NAMES = {
    0: "FCM_OK", 1: "FCM_ERR_INVALID", 2: "FCM_ERR_CUDA", 3: "FCM_ERR_CUFFT",
    4: "FCM_ERR_STATE", 5: "FCM_ERR_NOT_CONVERGED", 6: "FCM_ERR_NONFINITE",
    7: "FCM_ERR_OVERLAP", 8: "FCM_ERR_NOMEM", 9: "FCM_ERR_CAPACITY",
}


def rod_reference_positions(n_blobs=6, spacing=2.2, a=1.0):
    """Straight rod of ``n_blobs`` touching blobs along the body x-axis, centred:
    r_m = ((m - (n-1)/2) * spacing * a, 0, 0).  (The reference's own rods are the
    22-blob twisted pairs of collection_of_rigid_bodies.cpp:56-70; the geometry is
    data, so this shape is just another blob_ref_pos.)"""
    out = []
    for m in range(n_blobs):
        out += [(m - 0.5 * (n_blobs - 1)) * spacing * a, 0.0, 0.0]
    return out


def reference_rod_positions(blobs_per_body=22, a=1.0):
    """The reference's rod shape, collection_of_rigid_bodies.cpp:56-70: pairs of
    blobs at x = sqrt(2) a (pair - nb/4 + 1/2), rotated by 90 degrees per pair."""
    out = [0.0] * (3 * blobs_per_body)
    pair = 0
    for blob_id in range(0, blobs_per_body, 2):
        theta = pair * 0.5 * PI
        x = math.sqrt(2.0) * a * (pair - 0.25 * blobs_per_body + 0.5)
        out[3 * blob_id:3 * blob_id + 3] = [x, a * math.cos(theta), a * math.sin(theta)]
        out[3 * blob_id + 3:3 * blob_id + 6] = [x, -a * math.cos(theta), -a * math.sin(theta)]
        pair += 1
    return out
