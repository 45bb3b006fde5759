"""Fluctuation-dissipation at the level of the rigid bodies.

An Euler-Maruyama step solves the saddle-point system with the random blob
velocities on the right-hand side (gmres_solver.cpp:58-70, :148-306; main.cpp:
308-312).  With no forces the body velocities are U = N K^T M^-1 V_rand, with
N = (K^T M^-1 K)^-1, so <U U^T> = N K^T M^-1 <V V^T> M^-1 K N = (2 kT/dt) N when
the random field satisfies <V V^T> = (2 kT/dt) M.  N itself is measured through
the same solve: the right-hand side [0 ; -e_j] gives U = N e_j.  The sampled
covariance must match (2 kT/dt) N within the sampling error of S samples,
E|C - T|_F^2 = sum_ij (T_ii T_jj + T_ij^2) / S, in FP64 and in mixed precision.
"""
import numpy as np
import pytest

from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu


def _three_clusters():
    """Three bodies of one compact 4-blob cluster shape (not collinear, so N is
    regular) in a 32^3 box (dx = 0.4a, sigma/dx = 1.41), every inter-body blob
    pair farther apart than the steric cut-off."""
    rng = np.random.default_rng(5)
    ref = configs.random_walk_cluster(rng, 4, draws=8)
    x = np.array([[3.5, 4.0, 6.0], [9.0, 8.5, 4.5], [6.0, 9.5, 10.0]])
    q = configs.random_unit_quaternions(rng, 3)
    R = configs.rotation_matrices(q)
    Y = x[:, None, :] + np.einsum("mij,nj->mni", R, ref)
    for a in range(3):
        for b in range(a + 1, 3):
            assert np.linalg.norm(Y[a][:, None, :] - Y[b][None, :, :], axis=2).min() > 2.5
    return ref.ravel(), x.ravel(), q.ravel()


@pytest.mark.parametrize("precision", [0, 1])
def test_body_velocity_covariance_is_2kT_over_dt_N(gpu, precision):
    ref, x, q = _three_clusters()
    M, nb = 3, 4
    p = FcmParams.defaults(nx=32, ny=32, nz=32, ngauss=16, dx=0.4, num_bodies=M, blobs_per_body=nb, ncells=3,
                           kT=1.0, dt=0.01, potential=3, steric_fs=40.0, steric_rc=2.2, gmres_tol=1e-11,
                           gmres_max_iter=100, precision=precision, noise=1)
    s = Suspension(p, ref)
    s.set_bodies(x, q)
    s.produce_reference_matrices()
    s.fill_all_blob_pos()
    s.set_up_gaussians()
    Nb, n6 = M * nb, 6 * M
    # N column by column: RHS [0 ; -e_j] gives U = N e_j
    Nmat = np.zeros((n6, n6))
    for j in range(n6):
        b = np.zeros(3 * Nb + n6)
        b[3 * Nb + j] = -1.0
        s.set_RHS(b)
        st, soln, it, rel = s.invert_saddle_point_system()
        assert st == 0
        Nmat[:, j] = soln[3 * Nb:]
    assert np.abs(Nmat - Nmat.T).max() < 1e-6 * np.abs(Nmat).max()
    T = (2.0 * p.kT / p.dt) * 0.5 * (Nmat + Nmat.T)
    # samples: Philox random field, no forces, one saddle-point solve each
    s.set_blob_forces(np.zeros(3 * Nb))
    S = 3000
    Us = np.zeros((S, n6))
    for i in range(S):
        s.produce_random_velocity_field(4321, i)
        s.calculate_random_blob_velocities()
        s.assemble_RHS()
        st, soln, it, rel = s.invert_saddle_point_system()
        assert st == 0
        Us[i] = soln[3 * Nb:]
    s.close()
    C = Us.T @ Us / S
    se_mean = np.sqrt(np.diag(T) / S)
    assert np.all(np.abs(Us.mean(0)) < 5 * se_mean)
    expected = np.sqrt(np.sum(np.outer(np.diag(T), np.diag(T)) + T ** 2) / S)
    err = np.linalg.norm(C - T)
    assert err < 3.0 * expected, (err / np.linalg.norm(T), expected / np.linalg.norm(T))
