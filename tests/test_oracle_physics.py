"""Known-answer and identity checks of the CPU oracle (pinning its physics)."""
import math

import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.params import FcmParams, rod_reference_positions


@pytest.mark.parametrize("L,N", [(32.0, 96), (48.0, 128)])
def test_single_blob_hasimoto(L, N):
    """Self-mobility of one blob in a periodic cube: 1/(6 pi eta a) times
    Hasimoto's correction 1 - 2.837297 a/L + 4.19 (a/L)^3 (sigma = a/sqrt(pi)
    gives the Stokes drag 6 pi eta a of FCM)."""
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=20, dx=L / N, num_bodies=1, blobs_per_body=1, ncells=3)
    o = Oracle(p, [0, 0, 0])
    o.set_bodies([L / 2 + 0.123, L / 2 - 0.2, L / 2 + 0.05], [1, 0, 0, 0])
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    V = o.apply_mobility([1.0, 0, 0])
    mu0 = 1 / (6 * math.pi)
    x = 1.0 / L
    hasimoto = mu0 * (1 - 2.837297 * x + 4.19 * x ** 3)
    assert abs(V[0] - hasimoto) / hasimoto < 2e-5
    assert abs(V[1]) < 1e-10 * mu0 and abs(V[2]) < 1e-10 * mu0


@pytest.mark.parametrize("shape", [(16, 16, 16), (12, 18, 10), (10, 9, 15)])
def test_stokes_solve_is_the_spectral_projection(shape):
    """The oracle's Stokes solve against the spectral solution computed here with
    numpy's FFT: every mode with no Nyquist index satisfies
    u(q) = (f(q) - q (q.f(q)) / |q|^2) / (eta |q|^2), so u is divergence-free
    (q.u = 0) and f - eta |q|^2 u is a pure pressure gradient (parallel to q); the
    mean flow is zero.  (At Nyquist indices the reference's one-sided wavenumber
    and the C2R's Hermitian part differ from this symmetric form.)"""
    nx, ny, nz = shape
    dx = 0.9
    p = FcmParams.defaults(nx=nx, ny=ny, nz=nz, ngauss=8, dx=dx, num_bodies=5, blobs_per_body=1, ncells=3,
                           viscosity=1.7)
    o = Oracle(p, [0, 0, 0])
    rng = np.random.default_rng(11)
    o.set_up_gaussians((rng.uniform(0, 1, (5, 3)) * np.array([nx, ny, nz]) * dx).ravel())
    o.set_up_force_distribution(rng.standard_normal(15))
    grid = lambda c: o.get_grid(c).reshape(nx, ny, p.pad)[:, :, :nz].copy()
    Fh = np.array([np.fft.fftn(grid(c)) for c in range(3)])  # before the in-place transforms
    o.produce_deterministic_velocity_field()
    Uh = np.array([np.fft.fftn(grid(c)) for c in range(3, 6)])
    qs = np.meshgrid(*[2 * np.pi * np.fft.fftfreq(n, d=dx) for n in (nx, ny, nz)], indexing="ij")
    q = np.array(qs)
    q2 = (q ** 2).sum(0)
    keep = np.ones((nx, ny, nz), bool)
    for ax, n in enumerate((nx, ny, nz)):
        if n % 2 == 0:
            idx = [slice(None)] * 3
            idx[ax] = n // 2
            keep[tuple(idx)] = False
    keep[0, 0, 0] = False
    qf = (q * Fh).sum(0)
    expect = (Fh - q * qf / np.where(q2 > 0, q2, 1)) / (p.viscosity * np.where(q2 > 0, q2, 1))
    scale = np.abs(expect[:, keep]).max()
    assert np.abs(Uh[:, keep] - expect[:, keep]).max() < 1e-12 * scale
    assert np.abs((q * Uh).sum(0)[keep]).max() < 1e-12 * scale * np.sqrt(q2.max())
    assert np.abs(Uh[:, 0, 0, 0]).max() < 1e-12 * scale


def _small_suspension(M=4, nb=3, N=24, L=24.0, seed=3):
    ref = np.array(rod_reference_positions(nb, 2.2))
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=12, dx=L / N, num_bodies=M, blobs_per_body=nb, ncells=4,
                           potential=3, gmres_tol=1e-12, gmres_max_iter=200, dt=0.01)
    rng = np.random.default_rng(seed)
    x, q = configs.seed_bodies(rng, M, ref, L)
    return p, ref, x, q


def test_mobility_symmetric_positive_definite():
    p, ref, x, q = _small_suspension()
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    n = 3 * o.Nb
    Mm = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        Mm[:, j] = o.apply_mobility(e)
    assert np.abs(Mm - Mm.T).max() < 1e-12 * np.abs(Mm).max()
    assert np.linalg.eigvalsh(0.5 * (Mm + Mm.T)).min() > 0


def test_K_KT_adjoint():
    p, ref, x, q = _small_suspension()
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    rng = np.random.default_rng(1)
    U = rng.standard_normal(6 * o.M)
    lam = rng.standard_normal(3 * o.Nb)
    assert abs(lam @ o.multiply_by_K_at_midstep(U) - U @ o.multiply_by_KT_at_midstep(lam)) < 1e-12 * np.abs(lam).sum()


def test_quaternion_update_keeps_unit_norm():
    p, ref, x, q = _small_suspension()
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    rng = np.random.default_rng(2)
    for _ in range(20):
        o.end_of_step_update(rng.standard_normal(6 * o.M), 1.0)
    _, q2 = o.get_bodies()
    assert np.abs(np.linalg.norm(q2.reshape(-1, 4), axis=1) - 1).max() < 1e-13


def test_preconditioner_exact_for_isolated_body():
    """With a single body at the box centre, q = 1, the block-diagonal
    preconditioner is the exact inverse of the saddle-point matrix."""
    nb = 4
    ref = np.array([1.1, 0.3, 0.0, -1.1, 0.3, 0.0, 0.0, -0.6, 0.9, 0.2, 0.1, -1.0])
    p = FcmParams.defaults(nx=24, ny=24, nz=24, ngauss=12, dx=1.0, num_bodies=1, blobs_per_body=nb, ncells=3)
    o = Oracle(p, ref)
    o.produce_reference_matrices()
    o.set_bodies([12.0, 12.0, 12.0], [1, 0, 0, 0])
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    rng = np.random.default_rng(4)
    v = rng.standard_normal(o.n)
    w = o.multiply_by_saddle_point_matrix(o.multiply_by_Pinv(v))
    assert rel_err(w, v) < 1e-10


def test_gmres_solves_saddle_point_system():
    p, ref, x, q = _small_suspension()
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    o.produce_reference_matrices()
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    rng = np.random.default_rng(5)
    # consistent right-hand side: straight rods make the axial-torque row of
    # -K^T lambda identically zero, so b must lie in the range of A
    b = o.multiply_by_saddle_point_matrix(rng.standard_normal(o.n))
    o.set_RHS(b)
    st, xs, it, rel = o.invert_saddle_point_system()
    assert st == 0 and rel < 1e-12
    r = o.multiply_by_saddle_point_matrix(xs) - b
    # rods are straight: the axial spin is a null mode of A, so measure the residual
    assert np.linalg.norm(r) < 1e-9 * np.linalg.norm(b)


def test_reference_rod_shape_keeps_full_rank():
    """The reference's own twisted 22-blob rods (collection_of_rigid_bodies.cpp:56-70)
    have an invertible K^T K (no pseudo-inverse is needed)."""
    from timstochrigidbodiessim_b200.params import reference_rod_positions
    ref = np.array(reference_rod_positions(22))
    p = FcmParams.defaults(nx=16, ny=16, nz=16, ngauss=4, dx=4.0, num_bodies=1, blobs_per_body=22, ncells=3)
    o = Oracle(p, ref)
    _, _, KTKinv = o.get_reference_matrices()
    K = np.zeros((66, 6))
    for m in range(22):
        r = ref[3 * m:3 * m + 3]
        K[3 * m:3 * m + 3, :3] = np.eye(3)
        K[3 * m:3 * m + 3, 3:] = np.array([[0, r[2], -r[1]], [-r[2], 0, r[0]], [r[1], -r[0], 0]])
    assert rel_err(KTKinv, np.linalg.inv(K.T @ K)) < 1e-12
