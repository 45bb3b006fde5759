"""Kernel variants of the grid stages and their autotuner (no reference
counterpart).  The four spread kernels (persistent pipelined; one CTA per tile
staging 16, 8 or 32 blobs per round) sum every grid point's blobs in the same
order with the same products, and so does the one-warp-per-tile spread (variant
4), so M F is the same bit for bit whichever runs; the Stokes-solve variants
(cuFFT 3D + projection, cuFFT (y, z) + fused x-transform, the library's (y, z)
kernels + fused x-transform) and the three interpolation kernels (64 threads per
tile with the shuffle reduction; one warp per tile, two y-rows per lane, with the
shuffle or a shared-memory reduction) agree with the oracle
within 1e-10 (FP64) and 1e-6 (FP32) relative.  fcm_autotune times what the grid
allows, keeps the fastest by its own timings, and the results after tuning still
match the oracle."""
import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.capi import FcmError
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu

TOL = {0: 1e-10, 1: 1e-6}


def _setup(n=(64, 64, 64), nbodies=40):
    nx, ny, nz = n
    p = FcmParams.defaults(nx=nx, ny=ny, nz=nz, ngauss=12, dx=1.0, num_bodies=nbodies, blobs_per_body=1, ncells=3,
                           precision=1)
    rng = np.random.default_rng(3)
    Y = (rng.uniform(0, 1, (nbodies, 3)) * np.array([nx, ny, nz])).ravel()
    F = rng.standard_normal(3 * nbodies)
    g, o = Suspension(p, [0, 0, 0]), Oracle(p.copy(precision=0), [0, 0, 0])
    for s in (g, o):
        s.set_up_gaussians(Y)
    return g, o.apply_mobility(F), F


def _mf(g, F, prec):
    g.spread(F, prec)
    g.stokes_solve(prec)
    return g.interp(prec)


def test_variants_agree(gpu):
    g, Vo, F = _setup()
    v0 = g.get_variants()
    assert v0 == [0, 1, 4, 2, 1, 1]  # the defaults on a 64^3 grid
    for prec in (0, 1):
        for sv in ((0, 1) if prec == 0 else (0, 1, 2)):
            out = []
            for sp in (0, 1, 2, 3, 4):
                v = g.get_variants()
                v[2 * prec], v[2 * prec + 1] = sp, sv
                g.set_variants(v)
                out.append(_mf(g, F, prec))
            for o_ in out[1:]:
                assert np.array_equal(out[0], o_), (prec, sv)
            assert rel_err(out[0], Vo) < TOL[prec], (prec, sv)
        if prec == 1:  # the tensor-core spread agrees with the FMA kernels to FP32 rounding
            v = g.get_variants()
            v[2], v[3] = 5, 0
            g.set_variants(v)
            assert rel_err(_mf(g, F, prec), Vo) < TOL[prec]
        for iv in ((0, 1, 2) if prec == 0 else (0, 1, 2, 3)):
            v = g.get_variants()
            v[4 + prec] = iv
            g.set_variants(v)
            assert g.get_variants()[4 + prec] == iv
            assert rel_err(_mf(g, F, prec), Vo) < TOL[prec], (prec, iv)


def test_autotune_keeps_the_fastest(gpu):
    g, Vo, F = _setup()
    v, us = g.autotune(reps=3)
    # FP64 has no library (y, z) variant and no tensor-core spread or interpolation
    assert np.all(us[0:5] > 0) and us[5] == -1 and np.all(us[6:8] > 0) and us[8] == -1
    assert np.all(us[9:12] > 0) and np.all(us[12:16] == -1)
    assert np.all(us[16:29] > 0) and np.all(us[29:32] == -1)
    for P in (0, 1):
        t = us[16 * P:16 * P + 16]
        spread, solve, interp = t[0:5 + P], t[6:9], t[9:12 + P]
        assert v[2 * P] == int(np.argmin(spread))
        best = min((x, i) for i, x in enumerate(solve) if x >= 0)[1]
        assert v[2 * P + 1] == best
        assert v[4 + P] == int(np.argmin(interp))
    assert g.get_variants() == v
    for prec in (0, 1):
        assert rel_err(_mf(g, F, prec), Vo) < TOL[prec], prec


def test_variants_refused_where_the_grid_does_not_allow_them(gpu):
    g, _, _ = _setup()
    with pytest.raises(FcmError):
        g.set_variants([0, 2, 1, 2, 0, 0])  # no library (y, z) variant in FP64
    with pytest.raises(FcmError):
        g.set_variants([5, 1, 1, 2, 0, 0])  # no tensor-core spread in FP64
    with pytest.raises(FcmError):
        g.set_variants([0, 1, 6, 2, 0, 0])  # out of range
    with pytest.raises(FcmError):
        g.set_variants([0, 1, 1, 2, 3, 0])  # no tensor-core interpolation in FP64
    with pytest.raises(FcmError):
        g.set_variants([0, 1, 1, 2, 0, 4])  # out of range
    # 20 points along x: no fused x-transform, so only the 3D solve; not tiled, so
    # the spread and interpolation variants are not timed
    h, Vo, F = _setup((20, 24, 16), nbodies=12)
    assert h.get_variants()[1] == 0 and h.get_variants()[3] == 0
    with pytest.raises(FcmError):
        h.set_variants([0, 1, 1, 0, 0, 0])
    v, us = h.autotune(reps=2)
    assert us[6] > 0 and us[7] == -1 and us[8] == -1 and us[22] > 0 and us[23] == -1 and us[24] == -1
    assert np.all(us[0:6] == -1) and np.all(us[9:16] == -1) and np.all(us[16:22] == -1) and np.all(us[25:32] == -1)
    assert v[1] == 0 and v[3] == 0
    for prec in (0, 1):
        assert rel_err(_mf(h, F, prec), Vo) < TOL[prec], prec


@pytest.mark.parametrize("n", [(384, 32, 32), (512, 32, 32), (32, 512, 32), (32, 32, 512), (32, 384, 384),
                               (512, 64, 64), (256, 256, 64)])
def test_long_transforms(gpu, n):
    """The long lengths (384 = 16 x 24, 512 = 32 x 16) of the fused x-transform and
    of the library's y and z passes (64 KB of shared memory per y CTA at 512), in
    both precisions against the 3D transforms and the oracle, on thin boxes; the
    last two boxes give the persistent FP32 x-transform CTAs (one per SM) more than
    one block each.  FP64 keeps the 3D transforms by default beyond 256 points along
    x; the fused path is a tunable variant."""
    g, Vo, F = _setup(n, nbodies=24)
    assert g.get_variants()[1] == (0 if n[0] > 256 else 1)
    for prec in (0, 1):
        out = []
        for sv in ((0, 1) if prec == 0 else (0, 1, 2)):
            v = g.get_variants()
            v[2 * prec + 1] = sv
            g.set_variants(v)
            out.append(_mf(g, F, prec))
            assert rel_err(out[-1], Vo) < TOL[prec], (prec, sv)
        for o_ in out[1:]:
            assert rel_err(o_, out[0]) < TOL[prec], prec
