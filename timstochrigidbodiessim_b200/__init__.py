"""B200-native fluctuating force-coupling-method (FCM) mobility solve.

Drop-in for the FCM path of timwestwood/TimStochRigidBodiesSim: Gaussian
spreading, spectral Stokes solve with the fluctuating stress, interpolation, the
rigid-body saddle-point GMRES with its block-diagonal preconditioner, cell-list
steric forces and Philox noise, as hand-written sm_100a kernels behind the
C-ABI of include/fcm_b200.h.
"""
from .params import (FcmParams, FcmStepInfo, rod_reference_positions, reference_rod_positions,
                     STATUS_NAMES, FCM_OK, FCM_ERR_NOT_CONVERGED, FCM_ERR_OVERLAP)

__all__ = ["FcmParams", "FcmStepInfo", "rod_reference_positions", "reference_rod_positions",
           "STATUS_NAMES", "FCM_OK", "FCM_ERR_NOT_CONVERGED", "FCM_ERR_OVERLAP", "Suspension", "fft_solver"]


def __getattr__(name):
    # The GPU classes load libfcm_b200.so on first use and fail loudly if it is
    # missing; the parameter helpers above need no GPU.
    if name in ("Suspension", "fft_solver"):
        from . import fcm
        return getattr(fcm, name)
    raise AttributeError(name)
