"""Tiled spreading and interpolation against the CPU FP64 oracle where the tile
lists are long and ragged: dense blobs (many staging rounds per tile), a cluster
packed into one tile, blobs on tile faces and on the periodic boundary.  Also the
one-stage C-ABI calls (fcm_spread / fcm_stokes_solve / fcm_interp) on the FP64
and FP32 grids.

Tolerances: FP64 force grids and blob velocities 1e-10 relative (norm-wise), as
the rest of the parity suite; FP32 grids 1e-5 relative.
"""
import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _blobs(L, n, rng):
    Y = rng.uniform(0.0, L, (n, 3))
    # a cluster inside one tile (DX = 1: the tile [16, 24)^3)
    Y[:200] = rng.uniform(16.0, 24.0, (200, 3))
    # on tile faces, on the periodic boundary and just below L
    Y[200] = (8.0, 16.0, 24.0)
    Y[201] = (0.0, 0.0, 0.0)
    Y[202] = (L - 1e-9, L - 1e-9, L - 1e-9)
    Y[203] = (L - 1e-9, 0.0, 32.0)
    Y[204] = (7.999999, 8.0, 8.000001)
    return Y.ravel()


def _params(n, precision=0, N=64, L=64.0):
    return FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=20, dx=L / N, blob_radius=1.0, viscosity=1.0,
                              num_bodies=n, blobs_per_body=1, ncells=3, precision=precision)


@pytest.fixture(scope="module")
def dense():
    n = 1500
    Y = _blobs(64.0, n, np.random.default_rng(11))
    F = np.random.default_rng(12).standard_normal(3 * n)
    o = Oracle(_params(n), [0, 0, 0])
    o.set_up_gaussians(Y)
    o.set_up_force_distribution(F)
    fgrid = [o.get_grid(c).copy() for c in range(3)]
    o.produce_deterministic_velocity_field()
    V = o.calculate_deterministic_blob_velocities()
    return n, Y, F, fgrid, V


def test_dense_spread_grid_fp64(gpu, dense):
    n, Y, F, fgrid, _ = dense
    g = Suspension(_params(n), [0, 0, 0])
    g.set_up_gaussians(Y)
    g.spread(F, 0)
    fg = g.get_velocity_field(0)
    for c in range(3):
        assert rel_err(fg[c], fgrid[c]) < TOL


def test_dense_mobility_fp64_stages(gpu, dense):
    n, Y, F, _, V = dense
    g = Suspension(_params(n), [0, 0, 0])
    g.set_up_gaussians(Y)
    g.spread(F, 0)
    g.stokes_solve(0)
    assert rel_err(g.interp(0), V) < TOL
    # the reference-named sequence gives the same
    assert rel_err(g.apply_mobility(F), V) < TOL


def test_dense_mobility_fp32_stages(gpu, dense):
    import torch
    n, Y, F, _, V = dense
    g = Suspension(_params(n, precision=1), [0, 0, 0])
    g.set_up_gaussians(Y)
    Fd = torch.tensor(F, device="cuda")
    Vd = torch.full((3 * n,), float("nan"), dtype=torch.float64, device="cuda")
    g.spread(Fd, 1)
    g.stokes_solve(1)
    g.interp(1, out=Vd)
    torch.cuda.synchronize()
    assert rel_err(Vd.cpu().numpy(), V) < 1e-5
    # host buffers through the same calls
    g.spread(F, 1)
    g.stokes_solve(1)
    assert rel_err(g.interp(1), V) < 1e-5


def test_stage_precision_checks(gpu):
    from timstochrigidbodiessim_b200.capi import FcmError
    n = 8
    g = Suspension(_params(n), [0, 0, 0])
    with pytest.raises(FcmError):
        g.spread(np.zeros(3 * n), 0)  # no Gaussians yet
    g.set_up_gaussians(np.random.default_rng(0).uniform(0, 64, 3 * n))
    with pytest.raises(FcmError):
        g.spread(np.zeros(3 * n), 1)  # FP32 grid on an FP64 context
    with pytest.raises(FcmError):
        g.stokes_solve(2)


def test_dense_tensor_core_fp32_stages(gpu, dense):
    """The tensor-core spread (FP32 variant 5) and interpolation (variant 3), each
    alone beside the FMA kernels and both together, on the dense ragged tile lists:
    within 1e-6 of the FMA kernels' velocities (both FP32; 3xTF32 keeps every
    product to FP32 rounding) and within 1e-5 of the FP64 oracle, on two calls."""
    n, Y, F, _, V = dense
    g = Suspension(_params(n, precision=1), [0, 0, 0])
    g.set_up_gaussians(Y)

    def mf(sp, ip):
        v = g.get_variants()
        v[2], v[5] = sp, ip
        g.set_variants(v)
        g.spread(F, 1)
        g.stokes_solve(1)
        return g.interp(1)

    V_fma = mf(4, 1)
    assert rel_err(V_fma, V) < 1e-5
    for sp, ip in ((5, 1), (4, 3), (5, 3), (5, 3)):
        Vt = mf(sp, ip)
        assert rel_err(Vt, V_fma) < 1e-6, (sp, ip)
        assert rel_err(Vt, V) < 1e-5, (sp, ip)
