"""GPU path (through the C-ABI) against the CPU FP64 oracle on identical inputs.

Tolerances (FP64): blob velocities, RHS, K/K^T, P^-1 and saddle-point products
1e-10 relative (norm-wise); positions, Gaussian indices, cell ids and pair sets
bit-exact; body states after several steps 1e-9 absolute.
"""
import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle, fft_inverse_transform, fft_transform
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Suspension, fft_solver
from timstochrigidbodiessim_b200.params import FcmParams, rod_reference_positions

pytestmark = pytest.mark.gpu

TOL = 1e-10


def pair(p, ref, x=None, q=None, fe=None):
    g = Suspension(p, ref)
    o = Oracle(p, ref)
    if x is not None:
        g.set_bodies(x, q)
        o.set_bodies(x, q)
    if fe is not None:
        g.set_external_forces(fe)
        o.set_external_forces(fe)
    return g, o


@pytest.fixture(scope="module")
def cfg0():
    return configs.workload("rods32_L64_g64", gmres_tol=1e-12)


@pytest.mark.parametrize("shape", [(8, 8, 8), (12, 6, 10), (16, 24, 9), (64, 64, 64), (24, 12, 48)])
def test_fft_solver(gpu, shape):
    nx, ny, nz = shape
    rng = np.random.default_rng(7)
    f = fft_solver(nx, ny, nz)
    assert f.pad == 2 * (nz // 2 + 1) and f.local_nx == nx and f.local_x_start == 0
    a = np.zeros((nx, ny, f.pad))
    a[:, :, :nz] = rng.standard_normal((nx, ny, nz))
    a = a.ravel()
    ref = fft_transform(nx, ny, nz, a)
    g = a.copy()
    f.transform(g)
    assert rel_err(g, ref) < 1e-13
    spec = rng.standard_normal(f.total_local_size)  # non-Hermitian input
    ref = fft_inverse_transform(nx, ny, nz, spec).reshape(nx, ny, f.pad)[:, :, :nz]
    g = spec.copy()
    f.inverse_transform(g)
    assert rel_err(g.reshape(nx, ny, f.pad)[:, :, :nz], ref) < 1e-13


def test_positions_cells_pairs_bitexact(gpu, cfg0):
    p, ref, x, q, fe = cfg0
    g, o = pair(p, ref, x, q)
    g.fill_all_blob_pos()
    o.fill_all_blob_pos()
    Yg, Yo = g.get_all_blob_pos(), o.get_all_blob_pos()
    assert np.array_equal(Yg, Yo)
    g.list_populate()
    o.list_populate()
    assert np.array_equal(g.list_get_cells(), o.list_get_cells())
    assert np.array_equal(g.list_get_pairs(), o.list_get_pairs())


def test_cells_and_pairs_soft_sphere_dense(gpu):
    """Type-0 soft sphere (no cutoff): every pair of the 27-cell neighbourhood
    counts, so the pair set is large; bit-exact set, forces to 1e-12."""
    nb, M, L = 3, 300, 30.0
    ref = np.array(rod_reference_positions(nb, 2.2))
    p = FcmParams.defaults(nx=32, ny=32, nz=32, ngauss=8, dx=L / 32, num_bodies=M, blobs_per_body=nb, ncells=6,
                           potential=0)
    rng = np.random.default_rng(11)
    Y = rng.uniform(0, L, 3 * M * nb)
    g, o = pair(p, ref)
    g.set_all_blob_pos(Y)
    o.set_all_blob_pos(Y)
    g.list_populate()
    o.list_populate()
    assert np.array_equal(g.list_get_cells(), o.list_get_cells())
    pg, po = g.list_get_pairs(), o.list_get_pairs()
    assert len(po) > 10000 and np.array_equal(pg, po)
    Fg = g.apply_barrier_forces(np.ones(3 * M * nb))
    Fo = o.apply_barrier_forces(np.ones(3 * M * nb))
    assert rel_err(Fg, Fo) < 1e-12
    assert g.check_for_overlap() == bool(o.check_for_overlap())


@pytest.mark.parametrize("potential", [1, 2, 3])
def test_steric_potentials(gpu, potential):
    nb, M, L = 2, 200, 20.0
    ref = np.array(rod_reference_positions(nb, 2.2))
    p = FcmParams.defaults(nx=16, ny=16, nz=16, ngauss=4, dx=L / 16, num_bodies=M, blobs_per_body=nb, ncells=5,
                           potential=potential, steric_fs=40.0, steric_rc=2.2)
    rng = np.random.default_rng(potential)
    Y = rng.uniform(0, L, 3 * M * nb)
    g, o = pair(p, ref)
    g.set_all_blob_pos(Y)
    o.set_all_blob_pos(Y)
    g.list_populate()
    o.list_populate()
    assert rel_err(g.apply_barrier_forces(), o.apply_barrier_forces()) < 1e-12


def test_mobility_parity_cfg0(gpu, cfg0):
    p, ref, x, q, fe = cfg0
    g, o = pair(p, ref, x, q)
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    F = np.random.default_rng(1).standard_normal(3 * p.num_blobs)
    for s in (g, o):
        s.set_up_force_distribution(F)
        s.produce_deterministic_velocity_field()
    Vg = g.calculate_deterministic_blob_velocities()
    Vo = o.calculate_deterministic_blob_velocities()
    assert rel_err(Vg, Vo) < TOL
    # velocity grids in the reference's padded layout
    ug = g.get_velocity_field(0)
    for c in range(3):
        assert rel_err(ug[c], o.get_grid(3 + c)) < TOL
    # one-call M F
    assert rel_err(g.apply_mobility(F), Vo) < TOL


def test_mobility_parity_golden_noncubic(gpu, golden):
    N = golden["mobility2_N"]
    dx, a, eta, W = golden["mobility2_params"]
    Y = golden["mobility2_Y"]
    p = FcmParams.defaults(nx=int(N[0]), ny=int(N[1]), nz=int(N[2]), ngauss=int(W), dx=float(dx), blob_radius=float(a),
                           viscosity=float(eta), num_bodies=len(Y) // 3, blobs_per_body=1, ncells=3)
    g = Suspension(p, [0, 0, 0])
    g.set_up_gaussians(Y)
    assert rel_err(g.apply_mobility(golden["mobility2_F"]), golden["mobility2_V"]) < TOL


def test_random_field_injected_parity(gpu, cfg0):
    p, ref, x, q, fe = cfg0
    g, o = pair(p, ref, x, q)
    rng = np.random.default_rng(3)
    s6 = [rng.standard_normal(p.nx * p.ny * p.pad) for _ in range(6)]
    for s in (g, o):
        s.inject_random_stress(s6)
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    assert rel_err(g.calculate_random_blob_velocities(), o.calculate_random_blob_velocities()) < TOL
    ug = g.get_velocity_field(1)
    for c in range(3):
        assert rel_err(ug[c], o.get_grid(6 + c)) < TOL


def test_random_field_golden(gpu, golden):
    N = golden["random_N"]
    Y = golden["random_Y"]
    p = FcmParams.defaults(nx=int(N[0]), ny=int(N[1]), nz=int(N[2]), ngauss=8, dx=1.0, num_bodies=len(Y) // 3,
                           blobs_per_body=1, ncells=3)
    g = Suspension(p, [0, 0, 0])
    P = int(N[0] * N[1] * (2 * (N[2] // 2 + 1)))
    g.inject_random_stress(golden["random_s6"].reshape(6, P))
    g.set_up_gaussians(Y)
    assert rel_err(g.calculate_random_blob_velocities(), golden["random_V"]) < TOL


def test_K_KT_Pinv_saddle_parity(gpu, cfg0):
    p, ref, x, q, fe = cfg0
    g, o = pair(p, ref, x, q)
    o.produce_reference_matrices()
    Minv, N, _ = o.get_reference_matrices()
    g.set_reference_matrices(Minv, N)
    rng = np.random.default_rng(4)
    U = rng.standard_normal(6 * p.num_bodies)
    lam = rng.standard_normal(3 * p.num_blobs)
    assert rel_err(g.multiply_by_K_at_midstep(U), o.multiply_by_K_at_midstep(U)) < TOL
    assert rel_err(g.multiply_by_KT_at_midstep(lam), o.multiply_by_KT_at_midstep(lam)) < TOL
    v = rng.standard_normal(p.system_size)
    assert rel_err(g.multiply_by_Pinv(v), o.multiply_by_Pinv(v)) < TOL
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    assert rel_err(g.multiply_by_saddle_point_matrix(v), o.multiply_by_saddle_point_matrix(v)) < TOL


def test_reference_matrices_parity(gpu, cfg0):
    p, ref, x, q, fe = cfg0
    g, o = pair(p, ref, x, q)
    g.produce_reference_matrices()
    o.produce_reference_matrices()
    Mg, Ng, Kg = g.get_reference_matrices()
    Mo, No, Ko = o.get_reference_matrices()
    assert rel_err(Mg, Mo) < 1e-9
    assert rel_err(Ng, No) < 1e-9
    assert rel_err(Kg, Ko) < 1e-14


def test_gmres_parity(gpu, cfg0):
    p, ref, x, q, fe = cfg0
    g, o = pair(p, ref, x, q, fe)
    o.produce_reference_matrices()
    Minv, N, _ = o.get_reference_matrices()
    g.set_reference_matrices(Minv, N)
    rng = np.random.default_rng(5)
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        s.calculate_forces()
    assert rel_err(g.get_blob_forces(), o.get_blob_forces()) < 1e-12
    V = rng.standard_normal(3 * p.num_blobs) * 0.01
    # RHS from V and forces (gmres_solver.cpp:58-70): inject V through set_RHS
    for s in (g, o):
        s.assemble_RHS()
    assert rel_err(g.get_RHS(), o.get_RHS()) < TOL
    b = o.get_RHS()
    b[: 3 * p.num_blobs] = -V
    for s in (g, o):
        s.set_RHS(b)
    sg, xg, itg, relg = g.invert_saddle_point_system()
    so, xo, ito, relo = o.invert_saddle_point_system()
    assert sg == 0 and so == 0
    assert abs(itg - ito) <= 1
    assert rel_err(xg, xo) < 1e-9


def _em_step_manual(s, s6, gdc=False):
    """main.cpp:222-451 driven through the reference-named methods with the
    stress injected (the reference's noise array)."""
    s.fill_all_blob_pos()
    s.inject_random_stress(s6)
    s.set_up_gaussians()
    V = s.calculate_random_blob_velocities()
    nu = 1.0
    if gdc:
        s.advance_to_midstep(V)
        divU = s.calculate_divU()
        nu = 1.0 + 0.5 * s.p.dt * divU
        s.fill_all_blob_pos(True)
        s.set_up_gaussians()
        s.calculate_random_blob_velocities()
    s.calculate_forces()
    s.assemble_RHS()
    st, soln, it, rel = s.invert_saddle_point_system()
    s.end_of_step_update(soln[3 * s.Nb:], nu)
    return st, it, nu


@pytest.mark.parametrize("algorithm", [2, 1])
def test_steps_with_injected_noise(gpu, cfg0, algorithm):
    p, ref, x, q, fe = cfg0
    p = p.copy(algorithm=algorithm)
    g, o = pair(p, ref, x, q, fe)
    o.produce_reference_matrices()
    Minv, N, _ = o.get_reference_matrices()
    g.set_reference_matrices(Minv, N)
    rng = np.random.default_rng(6)
    for step in range(3):
        s6 = [rng.standard_normal(p.nx * p.ny * p.pad) * 0.05 for _ in range(6)]
        rg = _em_step_manual(g, s6, gdc=(algorithm == 1))
        ro = _em_step_manual(o, s6, gdc=(algorithm == 1))
        assert rg[0] == 0 and ro[0] == 0
        if algorithm == 1:
            assert abs(rg[2] - ro[2]) < 1e-9 * max(1.0, abs(ro[2]))
        xg, qg = g.get_bodies()
        xo, qo = o.get_bodies()
        assert np.abs(xg - xo).max() < 1e-9
        assert np.abs(qg - qo).max() < 1e-9


def test_fcm_step_noise_off_parity(gpu, cfg0):
    """Ten deterministic EM steps through the one-call fcm_step."""
    p, ref, x, q, fe = cfg0
    p = p.copy(noise=0)
    g, o = pair(p, ref, x, q, fe)
    o.produce_reference_matrices()
    Minv, N, _ = o.get_reference_matrices()
    g.set_reference_matrices(Minv, N)
    for step in range(10):
        sg, ig = g.step(1234, step)
        so, io = o.step(1234, step)
        assert sg == 0 and so == 0
        assert abs(ig.gmres_iters - io.gmres_iters) <= 1
    xg, qg = g.get_bodies()
    xo, qo = o.get_bodies()
    assert np.abs(xg - xo).max() < 1e-9
    assert np.abs(qg - qo).max() < 1e-9
    # the bodies moved: sedimentation under (0,0,-1)
    assert np.abs(xg - x).max() > 1e-4


@pytest.mark.parametrize("precision", [0, 1])
def test_steps_repeat_bit_for_bit(gpu, cfg0, precision):
    """Determinism: two contexts on the same inputs take the same noisy EM steps
    bit for bit (fixed reduction orders, no atomics on tiled grids), FP64 and
    mixed precision; host-driven steps against host-driven, graph steps against
    graph steps."""
    p, ref, x, q, fe = cfg0
    p = p.copy(precision=precision)
    runs = []
    for graph in (False, False, True, True):
        s = Suspension(p, ref)
        s.set_bodies(x, q)
        s.set_external_forces(fe)
        s.produce_reference_matrices()
        for step in range(3):
            if graph:
                s.step_async(77, step)
                assert s.step_wait()[0] == 0
            else:
                assert s.step(77, step)[0] == 0
        runs.append(s.get_bodies())
        s.close()
    for (xa, qa), (xb, qb) in ((runs[0], runs[1]), (runs[2], runs[3])):
        assert np.array_equal(xa, xb) and np.array_equal(qa, qb)
    assert np.abs(runs[0][0] - x).max() > 1e-6


def test_device_pointers_through_the_abi(gpu, cfg0):
    """The same call with CUDA tensors (device pointers) gives the same result."""
    import torch
    p, ref, x, q, fe = cfg0
    g = Suspension(p, ref)
    g.set_bodies(torch.tensor(x, device="cuda"), torch.tensor(q, device="cuda"))
    g.fill_all_blob_pos()
    g.set_up_gaussians()
    F = np.random.default_rng(9).standard_normal(3 * p.num_blobs)
    Vh = g.apply_mobility(F)
    Vd = torch.zeros(3 * p.num_blobs, dtype=torch.float64, device="cuda")
    g.apply_mobility(torch.tensor(F, device="cuda"), out=Vd)
    torch.cuda.synchronize()
    assert rel_err(Vd.cpu().numpy(), Vh) < 1e-13


def test_mobility_parity_long_x_grid(gpu):
    """nx = 384: the FP32 Stokes solve takes the fused x-transform, the FP64 one the
    3D transforms (the fused kernel is used for FP64 only up to 256 points)."""
    from timstochrigidbodiessim_b200.params import FcmParams
    p = FcmParams.defaults(nx=384, ny=16, nz=16, ngauss=8, dx=0.5, num_bodies=24, blobs_per_body=1, ncells=3,
                           precision=1)
    rng = np.random.default_rng(4)
    Y = (rng.uniform(0, 1, (24, 3)) * np.array([192.0, 8.0, 8.0])).ravel()
    F = rng.standard_normal(72)
    g, o = Suspension(p, [0, 0, 0]), Oracle(p.copy(precision=0), [0, 0, 0])
    for s in (g, o):
        s.set_up_gaussians(Y)
    Vo = o.apply_mobility(F)
    g.spread(F, 0)
    g.stokes_solve(0)
    assert rel_err(g.interp(0), Vo) < TOL
    g.spread(F, 1)
    g.stokes_solve(1)
    assert rel_err(g.interp(1), Vo) < 1e-6


@pytest.mark.parametrize("shape", [(16, 16, 16), (32, 24, 16), (48, 64, 32), (96, 96, 96), (128, 64, 96),
                                   (24, 128, 128), (16, 192, 192), (12, 256, 256), (256, 16, 32)])
def test_stokes_solve_both_precisions(gpu, shape):
    """M F through the stage calls on both grids against the oracle: FP64 within
    1e-10, FP32 within 1e-6 (relative, norm-wise).  These grids take the fused
    x-transform in both precisions and, in FP32, the library's own (y, z)
    transforms, with factors 2, 3, 4, 6, 8, 12, 16 and non-cubic shapes: square
    (y, z) planes up to 96 points by one CTA per plane, the others (and the
    square 128, 192, 256-point planes) by separate z and y passes."""
    from timstochrigidbodiessim_b200.params import FcmParams
    nx, ny, nz = shape
    p = FcmParams.defaults(nx=nx, ny=ny, nz=nz, ngauss=8, dx=1.0, num_bodies=20, blobs_per_body=1, ncells=3,
                           precision=1)
    rng = np.random.default_rng(2)
    Y = (rng.uniform(0, 1, (20, 3)) * np.array([nx, ny, nz])).ravel()
    F = rng.standard_normal(60)
    g, o = Suspension(p, [0, 0, 0]), Oracle(p.copy(precision=0), [0, 0, 0])
    for s in (g, o):
        s.set_up_gaussians(Y)
    Vo = o.apply_mobility(F)
    for prec, tol in ((0, TOL), (1, 1e-6)):
        g.spread(F, prec)
        g.stokes_solve(prec)
        assert rel_err(g.interp(prec), Vo) < tol, prec
