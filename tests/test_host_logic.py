"""Host-side logic that needs no GPU: parameters, workloads, the C-ABI library
(loads and exports every symbol of include/fcm_b200.h)."""
import ctypes
import os
import re

import numpy as np
import pytest

from tests.conftest import ROOT
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.params import FcmParams, reference_rod_positions, rod_reference_positions

HEADER = os.path.join(ROOT, "include", "fcm_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(fcm_[a-zA-Z0-9_]+)\s*\(", txt)))


def test_params_struct_matches_header_defaults():
    from timstochrigidbodiessim_b200 import build
    p = FcmParams.defaults()
    assert p.nx == 256 and p.ngauss == 20 and p.ncells == 6 and p.gmres_max_iter == 40
    assert abs(p.dx - 0.3033277330901916) < 1e-16
    assert p.system_size == 3 * 66 + 18


def test_library_exports_every_header_symbol():
    from timstochrigidbodiessim_b200 import build
    lib_path = build.LIB
    if not os.path.exists(lib_path):
        build.build()
    lib = ctypes.CDLL(lib_path)
    syms = header_symbols()
    assert len(syms) >= 50
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    from timstochrigidbodiessim_b200 import capi
    assert sorted(capi.SIGNATURES) == syms


def test_default_params_from_library_match_python():
    from timstochrigidbodiessim_b200 import build, capi
    if not os.path.exists(build.LIB):
        build.build()
    lib = capi.load()
    p = FcmParams()
    lib.fcm_default_params(ctypes.byref(p))
    assert p.as_dict() == FcmParams.defaults().as_dict()


def test_invalid_params_rejected_without_gpu():
    """Parameter validation runs before any device call."""
    from timstochrigidbodiessim_b200 import build, capi
    if not os.path.exists(build.LIB):
        build.build()
    lib = capi.load()
    p = FcmParams.defaults(ncells=2)
    h = ctypes.c_void_p()
    ref = (ctypes.c_double * 66)()
    st = lib.fcm_create(ctypes.byref(p), ctypes.cast(ref, ctypes.c_void_p), ctypes.byref(h))
    assert st == 1 and b"ncells" in lib.fcm_last_error()
    p = FcmParams.defaults(algorithm=0)
    st = lib.fcm_create(ctypes.byref(p), ctypes.cast(ref, ctypes.c_void_p), ctypes.byref(h))
    assert st == 1


def test_rod_shapes():
    r = np.array(rod_reference_positions(6, 2.2)).reshape(-1, 3)
    assert np.allclose(np.diff(r[:, 0]), 2.2) and abs(r[:, 0].sum()) < 1e-12
    r22 = np.array(reference_rod_positions(22)).reshape(-1, 3)
    assert r22.shape == (22, 3) and np.allclose(r22.sum(0), 0.0, atol=1e-12)


@pytest.mark.parametrize("name", ["rods32_L64_g64"])
def test_workload_is_overlap_free(name):
    p, ref, x, q, fe = configs.workload(name)
    L = p.box[0]
    R = configs.rotation_matrices(q.reshape(-1, 4))
    Y = (x.reshape(-1, 1, 3) + np.einsum("nij,mj->nmi", R, ref.reshape(-1, 3))) % L
    Y = Y.reshape(-1, 3)
    body = np.repeat(np.arange(p.num_bodies), p.blobs_per_body)
    d = Y[:, None, :] - Y[None, :, :]
    d -= L * np.round(d / L)
    r2 = (d ** 2).sum(-1)
    other = body[:, None] != body[None, :]
    assert r2[other].min() >= 4.0
    assert np.allclose(np.linalg.norm(q.reshape(-1, 4), axis=1), 1.0)
    assert np.all(fe.reshape(-1, 6)[:, 2] == -1.0)


def test_volume_fraction_box():
    L = configs.box_for_volume_fraction(12288, 0.10)
    assert abs(L - 80.141) < 0.001


def test_ensemble_members_are_valid():
    """Batched-ensemble instances: body counts in [50, 500], volume fraction in
    [0.05, 0.20], grids 2^k or 3*2^k in [64, 128], no inter-body overlap."""
    from scipy.spatial import cKDTree
    for i in (0, 8):  # instance 8 is dense enough to need the compression path
        p, ref, x, q, fe = configs.ensemble(1, seed0=i)[0]
        assert 50 <= p.num_bodies <= 500 and p.nx in (64, 96, 128)
        L = p.box[0]
        phi = p.num_blobs * 4.0 / 3.0 * np.pi / L ** 3
        assert 0.05 <= phi <= 0.20
        R = configs.rotation_matrices(q.reshape(-1, 4))
        Y = ((x.reshape(-1, 1, 3) + np.einsum("nij,mj->nmi", R, ref.reshape(-1, 3))) % L).reshape(-1, 3)
        body = np.repeat(np.arange(p.num_bodies), p.blobs_per_body)
        pr = cKDTree(Y, boxsize=L).query_pairs(2.0, output_type="ndarray")
        assert not len(pr) or np.all(body[pr[:, 0]] == body[pr[:, 1]])
    assert configs.nearest_fft_size(117) == 128 and configs.nearest_fft_size(40) == 64
    assert configs.nearest_fft_size(100) == 96


def test_array_sizes_match_header():
    """The Python mirror's array sizes of the variant calls equal the header's
    (fcm_get/set_variants, fcm_autotune: 16 timings per precision)."""
    from timstochrigidbodiessim_b200.fcm import Suspension
    txt = open(HEADER).read()
    defs = dict(re.findall(r"#define\s+(FCM_[A-Z_]+)\s+(\d+)", txt))
    assert int(defs["FCM_NUM_VARIANTS"]) == Suspension.NUM_VARIANTS == 6
    assert int(defs["FCM_NUM_TUNE_TIMES"]) == Suspension.NUM_TUNE_TIMES == 32
