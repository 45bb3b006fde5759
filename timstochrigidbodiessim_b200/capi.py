"""ctypes binding of the C-ABI in include/fcm_b200.h (libfcm_b200.so).

The library is loaded from the package directory; if it is missing the import
fails loudly (build it with ``python -m timstochrigidbodiessim_b200.build``).
There is no CPU fallback.  With FCM_B200_BOUNDS_CHECK=1 in the environment the
bounds-checked build of the same library (libfcm_b200_debug.so) is loaded
instead; fcm_debug_bounds reports what its index checks found.
"""
import ctypes
import os

from .params import FcmMcmcState, FcmParams, FcmStepInfo

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
DEBUG_LIB_PATH = os.path.join(PKG_DIR, "libfcm_b200_debug.so")
LIB_PATH = DEBUG_LIB_PATH if os.environ.get("FCM_B200_BOUNDS_CHECK") == "1" else os.path.join(PKG_DIR,
                                                                                               "libfcm_b200.so")

D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)
I64 = ctypes.POINTER(ctypes.c_int64)
VP = ctypes.c_void_p

# name -> (restype, argtypes); every function of include/fcm_b200.h
SIGNATURES = {
    "fcm_default_params": (None, [ctypes.POINTER(FcmParams)]),
    "fcm_last_error": (ctypes.c_char_p, []),
    "fcm_version": (ctypes.c_char_p, []),
    "fcm_kernel_launch_count": (ctypes.c_int64, []),
    "fcm_debug_bounds": (ctypes.c_int, [I32, I64, I32, I64, I64, ctypes.c_int32]),
    "fcm_fft_create": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.POINTER(VP)]),
    "fcm_fft_destroy": (ctypes.c_int, [VP]),
    "fcm_fft_local_sizes": (ctypes.c_int, [VP, I32, I32, I32, I32, I64, I32]),
    "fcm_fft_transform": (ctypes.c_int, [VP, VP]),
    "fcm_fft_inverse_transform": (ctypes.c_int, [VP, VP]),
    "fcm_create": (ctypes.c_int, [ctypes.POINTER(FcmParams), VP, ctypes.POINTER(VP)]),
    "fcm_destroy": (ctypes.c_int, [VP]),
    "fcm_set_stream": (ctypes.c_int, [VP, VP]),
    "fcm_get_params": (ctypes.c_int, [VP, ctypes.POINTER(FcmParams)]),
    "fcm_set_bodies": (ctypes.c_int, [VP, VP, VP]),
    "fcm_get_bodies": (ctypes.c_int, [VP, VP, VP]),
    "fcm_get_midstep_bodies": (ctypes.c_int, [VP, VP, VP]),
    "fcm_set_external_forces": (ctypes.c_int, [VP, VP]),
    "fcm_fill_all_blob_pos": (ctypes.c_int, [VP, ctypes.c_int32]),
    "fcm_set_all_blob_pos": (ctypes.c_int, [VP, VP]),
    "fcm_get_all_blob_pos": (ctypes.c_int, [VP, VP]),
    "fcm_multiply_by_K_at_midstep": (ctypes.c_int, [VP, VP, VP]),
    "fcm_multiply_by_KT_at_midstep": (ctypes.c_int, [VP, VP, VP]),
    "fcm_calculate_forces": (ctypes.c_int, [VP]),
    "fcm_get_blob_forces": (ctypes.c_int, [VP, VP]),
    "fcm_set_blob_forces": (ctypes.c_int, [VP, VP]),
    "fcm_advance_to_midstep": (ctypes.c_int, [VP, VP, I32]),
    "fcm_calculate_divU": (ctypes.c_int, [VP, D]),
    "fcm_end_of_step_update": (ctypes.c_int, [VP, VP, ctypes.c_double, I32]),
    "fcm_reset_to_start_of_step": (ctypes.c_int, [VP]),
    "fcm_check_for_overlap": (ctypes.c_int, [VP, I32]),
    "fcm_check_for_channel_wall_overlap": (ctypes.c_int, [VP, I32]),
    "fcm_list_populate": (ctypes.c_int, [VP]),
    "fcm_list_get_cells": (ctypes.c_int, [VP, VP]),
    "fcm_list_get_pairs": (ctypes.c_int, [VP, VP, ctypes.c_int64, I64]),
    "fcm_apply_barrier_forces": (ctypes.c_int, [VP, VP]),
    "fcm_set_up_gaussians": (ctypes.c_int, [VP, VP]),
    "fcm_get_gaussians": (ctypes.c_int, [VP, ctypes.c_int32, VP, VP]),
    "fcm_set_body_shapes": (ctypes.c_int, [VP, VP]),
    "fcm_set_body_preconditioners": (ctypes.c_int, [VP, VP, VP]),
    "fcm_get_body_preconditioners": (ctypes.c_int, [VP, VP, VP, VP]),
    "fcm_produce_random_velocity_field": (ctypes.c_int, [VP, ctypes.c_uint64, ctypes.c_uint64]),
    "fcm_inject_random_stress": (ctypes.c_int, [VP, VP, VP, VP, VP, VP, VP]),
    "fcm_calculate_random_blob_velocities": (ctypes.c_int, [VP, VP]),
    "fcm_set_up_force_distribution": (ctypes.c_int, [VP, VP]),
    "fcm_produce_deterministic_velocity_field": (ctypes.c_int, [VP]),
    "fcm_calculate_deterministic_blob_velocities": (ctypes.c_int, [VP, VP]),
    "fcm_get_V": (ctypes.c_int, [VP, VP]),
    "fcm_get_velocity_field": (ctypes.c_int, [VP, ctypes.c_int32, VP, VP, VP]),
    "fcm_apply_mobility": (ctypes.c_int, [VP, VP, VP]),
    "fcm_set_up_dipole_distribution": (ctypes.c_int, [VP, VP, VP, VP]),
    "fcm_calculate_deterministic_blob_rotations": (ctypes.c_int, [VP, VP, VP]),
    "fcm_produce_shear_velocity_field": (ctypes.c_int, [VP, ctypes.c_double, ctypes.c_double]),
    "fcm_calculate_shear_blob_velocities": (ctypes.c_int, [VP, VP]),
    "fcm_fluid_x_velocity_in_y": (ctypes.c_int, [VP, VP, VP]),
    "fcm_spread": (ctypes.c_int, [VP, ctypes.c_int32, VP]),
    "fcm_stokes_solve": (ctypes.c_int, [VP, ctypes.c_int32]),
    "fcm_interp": (ctypes.c_int, [VP, ctypes.c_int32, VP]),
    "fcm_get_variants": (ctypes.c_int, [VP, VP]),
    "fcm_set_variants": (ctypes.c_int, [VP, VP]),
    "fcm_autotune": (ctypes.c_int, [VP, ctypes.c_int32, VP, VP]),
    "fcm_produce_reference_matrices": (ctypes.c_int, [VP]),
    "fcm_get_reference_matrices": (ctypes.c_int, [VP, VP, VP, VP]),
    "fcm_set_reference_matrices": (ctypes.c_int, [VP, VP, VP]),
    "fcm_assemble_RHS": (ctypes.c_int, [VP]),
    "fcm_get_RHS": (ctypes.c_int, [VP, VP]),
    "fcm_set_RHS": (ctypes.c_int, [VP, VP]),
    "fcm_multiply_by_Pinv": (ctypes.c_int, [VP, VP, VP]),
    "fcm_multiply_by_saddle_point_matrix": (ctypes.c_int, [VP, VP, VP]),
    "fcm_invert_saddle_point_system": (ctypes.c_int, [VP, VP, I32, D]),
    "fcm_step": (ctypes.c_int, [VP, ctypes.c_uint64, ctypes.c_uint64, ctypes.POINTER(FcmStepInfo)]),
    "fcm_calculate_potential": (ctypes.c_int, [VP, D]),
    "fcm_mcmc_state_init": (ctypes.c_int, [VP, ctypes.POINTER(FcmMcmcState)]),
    "fcm_mcmc_run": (ctypes.c_int, [VP, ctypes.c_uint64, ctypes.c_int64, ctypes.POINTER(FcmMcmcState)]),
    "fcm_batch_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(FcmParams), ctypes.POINTER(VP),
                                        ctypes.POINTER(VP)]),
    "fcm_batch_destroy": (ctypes.c_int, [VP]),
    "fcm_batch_member": (VP, [VP, ctypes.c_int32]),
    "fcm_batch_set_stream": (ctypes.c_int, [VP, VP]),
    "fcm_batch_last_rounds": (ctypes.c_int, [VP, ctypes.POINTER(ctypes.c_int32)]),
    "fcm_batch_step": (ctypes.c_int, [VP, ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint64,
                                      ctypes.POINTER(FcmStepInfo)]),
    "fcm_step_async": (ctypes.c_int, [VP, ctypes.c_uint64, ctypes.c_uint64]),
    "fcm_step_wait": (ctypes.c_int, [VP, ctypes.POINTER(FcmStepInfo)]),
    "fcm_step_many": (ctypes.c_int, [ctypes.POINTER(VP), ctypes.c_int32, ctypes.POINTER(ctypes.c_uint64),
                                     ctypes.c_uint64, ctypes.POINTER(FcmStepInfo)]),
    "fcm_interp_noalloc": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int32, ctypes.c_int32, VP, VP, VP, VP]),
}

_lib = None


class FcmError(RuntimeError):
    def __init__(self, status, where, message):
        from .params import STATUS_NAMES
        self.status = status
        super().__init__("%s failed: %s (%s)" % (where, STATUS_NAMES.get(status, status), message))


def load(path=LIB_PATH):
    """Load libfcm_b200.so; raises if it is missing (no fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError("libfcm_b200.so not built (%s); run python -m timstochrigidbodiessim_b200.build" % path)
    L = ctypes.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


BOUNDS_SITES = {0: "none", 1: "grid point", 2: "blob id", 3: "tile id", 4: "list slot", 5: "partial",
                6: "cell id", 7: "spectrum index", 8: "Krylov column"}


def debug_bounds(reset=False):
    """fcm_debug_bounds: (checked, violations, first site name, index, limit) on
    the current device; checked is False for the release build."""
    L = load()
    chk, site = ctypes.c_int32(0), ctypes.c_int32(0)
    cnt, idx, lim = ctypes.c_int64(0), ctypes.c_int64(0), ctypes.c_int64(0)
    check(L.fcm_debug_bounds(ctypes.byref(chk), ctypes.byref(cnt), ctypes.byref(site), ctypes.byref(idx),
                             ctypes.byref(lim), 1 if reset else 0), "fcm_debug_bounds")
    return bool(chk.value), int(cnt.value), BOUNDS_SITES.get(site.value, str(site.value)), int(idx.value), \
        int(lim.value)


def check(status, where, ok=(0,)):
    if status not in ok:
        msg = load().fcm_last_error()
        raise FcmError(status, where, msg.decode() if msg else "")
    return status
