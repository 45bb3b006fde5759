"""The allocation-free interpolation entry point (fcm_interp_noalloc), for callers
that cannot allocate device memory (a time-step loop that must not stall the
device, or an application whose device memory belongs to its own allocator).
It must give the same blob velocities as the context's own interpolation
(fcm_calculate_deterministic_blob_velocities) on the same grid and positions, on
consecutive calls that reuse its static scratch array.  Collected last so that a
run stopping at the first failure has run everything else."""
import ctypes

import numpy as np
import pytest

from tests.conftest import rel_err
from timstochrigidbodiessim_b200 import capi, configs
from timstochrigidbodiessim_b200.fcm import Suspension

pytestmark = pytest.mark.gpu


def _unpadded_grid(s, p):
    import torch
    ux, uy, uz = s.get_velocity_field(0)
    g = np.stack([u.reshape(p.nx, p.ny, p.pad)[:, :, :p.nz] for u in (ux, uy, uz)]).ravel()
    return torch.tensor(g, dtype=torch.float64, device="cuda")


def test_interp_noalloc_matches_context_interpolation(gpu):
    import torch
    lib = capi.load()
    p, ref, x, q, fe = configs.workload("rods32_L64_g64")
    s = Suspension(p, ref)
    s.set_bodies(x, q)
    s.fill_all_blob_pos()
    s.set_up_gaussians()
    Nb = p.num_blobs
    Y = torch.tensor(s.get_all_blob_pos(), dtype=torch.float64, device="cuda")
    rng = np.random.default_rng(17)
    for call in range(2):  # two calls in a row share (and must reset) the scratch array
        F = rng.standard_normal(3 * Nb)
        s.set_up_force_distribution(F)
        s.produce_deterministic_velocity_field()
        V_ref = s.calculate_deterministic_blob_velocities()
        grid = _unpadded_grid(s, p)
        V = torch.full((3 * Nb,), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.fcm_interp_noalloc(p.nx, p.ny, p.nz, p.dx, p.blob_radius, p.ngauss, Nb,
                                    ctypes.c_void_p(Y.data_ptr()), ctypes.c_void_p(grid.data_ptr()),
                                    ctypes.c_void_p(V.data_ptr()), None)
        assert st == 0, lib.fcm_last_error()
        torch.cuda.synchronize()
        assert rel_err(V.cpu().numpy(), V_ref) < 1e-13, call


def _free_blobs(n, grid, L, W, seed):
    """A context of n single-blob bodies at random positions on a grid^3 box of
    side L with stencil width W, its Gaussians set up, and Y as a CUDA tensor."""
    import torch
    from timstochrigidbodiessim_b200.params import FcmParams
    p = FcmParams.defaults(nx=grid, ny=grid, nz=grid, ngauss=W, dx=L / grid, num_bodies=n, blobs_per_body=1,
                           ncells=3)
    Y = np.random.default_rng(seed).uniform(0.0, L, 3 * n)
    s = Suspension(p, [0.0, 0.0, 0.0])
    s.set_up_gaussians(Y)
    return s, p, torch.tensor(Y, dtype=torch.float64, device="cuda")


def test_interp_noalloc_at_its_limits_then_smaller(gpu):
    """The largest input the scratch array accepts (8192 blobs, a 24-point stencil,
    a 256^3 grid), then a call with fewer blobs at other positions on another grid:
    the second call must not see the first call's tile lists or partials."""
    import torch
    lib = capi.load()
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    for n, grid, L, W, seed in ((8192, 256, 160.0, 24, 3), (5000, 128, 60.0, 16, 4)):
        s, p, Y = _free_blobs(n, grid, L, W, seed)
        F = np.random.default_rng(seed + 10).standard_normal(3 * n)
        s.set_up_force_distribution(F)
        s.produce_deterministic_velocity_field()
        V_ref = s.calculate_deterministic_blob_velocities()
        g = _unpadded_grid(s, p)
        V = torch.full((3 * n,), float("nan"), dtype=torch.float64, device="cuda")
        st = lib.fcm_interp_noalloc(p.nx, p.ny, p.nz, p.dx, p.blob_radius, p.ngauss, n, ptr(Y), ptr(g), ptr(V),
                                    None)
        assert st == 0, lib.fcm_last_error()
        torch.cuda.synchronize()
        assert rel_err(V.cpu().numpy(), V_ref) < 1e-13, (n, grid)
        s.close()
        del g


def test_interp_noalloc_rejects_out_of_range_inputs(gpu):
    import torch
    lib = capi.load()
    Y = torch.zeros(3 * 9000, dtype=torch.float64, device="cuda")
    grid = torch.zeros(3 * 64 ** 3, dtype=torch.float64, device="cuda")
    V = torch.zeros(3 * 9000, dtype=torch.float64, device="cuda")
    ptr = lambda t: ctypes.c_void_p(t.data_ptr())
    # too many blobs
    assert lib.fcm_interp_noalloc(64, 64, 64, 1.0, 1.0, 20, 9000, ptr(Y), ptr(grid), ptr(V), None) == 1
    assert b"nblobs" in lib.fcm_last_error()
    # grid not a multiple of 8
    assert lib.fcm_interp_noalloc(60, 64, 64, 1.0, 1.0, 20, 10, ptr(Y), ptr(grid), ptr(V), None) == 1
    # host pointer
    h = np.zeros(30)
    assert lib.fcm_interp_noalloc(64, 64, 64, 1.0, 1.0, 20, 10, ctypes.c_void_p(h.ctypes.data), ptr(grid),
                                  ptr(V), None) == 1
    assert b"device pointers" in lib.fcm_last_error()
    # a 9-tile-per-side grid beyond 32768 tiles (264^3 = 35937 tiles)
    assert lib.fcm_interp_noalloc(264, 264, 264, 1.0, 1.0, 20, 10, ptr(Y), ptr(grid), ptr(V), None) == 1
    assert b"tiles" in lib.fcm_last_error()
    # stencil wider than 24 points
    assert lib.fcm_interp_noalloc(64, 64, 64, 1.0, 1.0, 25, 10, ptr(Y), ptr(grid), ptr(V), None) == 1
    assert b"ngauss" in lib.fcm_last_error()
