"""Per-body shapes in the CPU oracle (no counterpart in the reference, whose
bodies share one blob_ref_pos, collection_of_rigid_bodies.hpp:24).

- The analytic free-space FCM blob-blob mobility that forms the per-body
  preconditioner equals the oracle's probed FCM body mobility
  (fcm_fluid_solver.cpp:842-881) up to the periodic images, whose leading term is
  the uniform Hasimoto shift -2.837297/(6 pi eta L) on every 3x3 block.
- A collection whose bodies are all given the same shape through the per-body
  path reproduces the single-shape oracle bit for bit (positions, K, K^T, the
  preconditioner with the same blocks, the rigid projection).
- With distinct shapes K and K^T stay adjoint and a saddle-point solve converges.
"""
import numpy as np
import pytest

from tests.oracle_lib import Oracle, lib
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.params import FcmParams


def test_analytic_body_mobility_matches_probed_fcm():
    lib().orc_set_threads(8)
    ref = configs.random_walk_cluster(np.random.default_rng(3), 4, draws=4)
    p = FcmParams.defaults(nx=128, ny=128, nz=128, ngauss=14, dx=0.5, num_bodies=1, blobs_per_body=4, ncells=3)
    o = Oracle(p, ref.ravel())
    o.produce_reference_matrices()
    Minv, _, _ = o.get_reference_matrices()
    M_fcm = np.linalg.inv(Minv.reshape(12, 12).T)
    o.set_body_shapes(ref.ravel())
    o.produce_body_preconditioners()
    Ma, _, _ = o.get_body_preconditioners()
    M_an = np.linalg.inv(Ma.reshape(12, 12).T)
    L = p.nx * p.dx
    shift = 2.837297 / (6.0 * np.pi * p.viscosity * L)
    assert abs(M_an[0, 0] * 6.0 * np.pi * p.blob_radius - 1.0) < 1e-12  # self-mobility 1/(6 pi eta a)
    rel = np.linalg.norm(M_fcm - M_an + shift * np.kron(np.ones((4, 4)), np.eye(3))) / np.linalg.norm(M_an)
    assert rel < 1e-3, rel
    o.close()


def _rods(M=12, seed=4):
    p, ref, x, q, fe = configs.rod_suspension(M=M, grid=32, L=24.0, nb=3, seed=seed, gmres_tol=1e-12, noise=0,
                                              ngauss=12)
    return p, ref, x, q, fe


def test_per_body_path_with_one_shape_equals_the_shared_shape():
    p, ref, x, q, fe = _rods()
    ref = np.asarray(ref).ravel()
    a, b = Oracle(p, ref), Oracle(p, ref)
    b.set_body_shapes(np.tile(ref, p.num_bodies))
    rng = np.random.default_rng(1)
    Minv = np.linalg.inv(np.eye(9) + 0.1 * np.ones((9, 9)))
    N = np.linalg.inv(np.eye(6) * 2.0 + 0.05)
    a.set_reference_matrices(Minv.T.ravel(), N.T.ravel())
    b.set_body_preconditioners(np.tile(Minv.T.ravel(), p.num_bodies), np.tile(N.T.ravel(), p.num_bodies))
    for s in (a, b):
        s.set_bodies(x, q)
        s.fill_all_blob_pos()
    assert np.array_equal(a.get_all_blob_pos(), b.get_all_blob_pos())
    U = rng.standard_normal(6 * p.num_bodies)
    lam = rng.standard_normal(3 * p.num_blobs)
    assert np.array_equal(a.multiply_by_K_at_midstep(U), b.multiply_by_K_at_midstep(U))
    assert np.array_equal(a.multiply_by_KT_at_midstep(lam), b.multiply_by_KT_at_midstep(lam))
    v = rng.standard_normal(p.system_size)
    assert np.array_equal(a.multiply_by_Pinv(v), b.multiply_by_Pinv(v))
    V = rng.standard_normal(3 * p.num_blobs) * 0.01
    a.advance_to_midstep(V)
    b.advance_to_midstep(V)
    assert np.array_equal(a.get_midstep_bodies()[0], b.get_midstep_bodies()[0])
    assert np.array_equal(a.get_midstep_bodies()[1], b.get_midstep_bodies()[1])
    a.close()
    b.close()


def test_distinct_shapes_adjoint_and_solve():
    lib().orc_set_threads(8)
    M, nb = 10, 5
    rng = np.random.default_rng(9)
    shapes = np.concatenate([configs.random_walk_cluster(rng, nb, draws=1).ravel() for _ in range(M)])
    p = FcmParams.defaults(nx=32, ny=32, nz=32, ngauss=12, dx=0.8, num_bodies=M, blobs_per_body=nb, ncells=3,
                           potential=3, gmres_tol=1e-12, gmres_max_iter=200, noise=0)
    o = Oracle(p, shapes[:3 * nb])
    o.set_body_shapes(shapes)
    o.produce_body_preconditioners()
    x = np.array([[(i % 3) * 8.0 + 4.0, (i // 3 % 3) * 8.0 + 4.0, (i // 9) * 8.0 + 4.0] for i in range(M)]).ravel()
    q = configs.random_unit_quaternions(rng, M).ravel()
    o.set_bodies(x, q)
    o.fill_all_blob_pos()
    # every body's blobs sit at its own shape: distances within a body are the shape's
    Y = o.get_all_blob_pos().reshape(M, nb, 3)
    for n in range(M):
        S = shapes[3 * nb * n:3 * nb * (n + 1)].reshape(nb, 3)
        dY = Y[n][:, None, :] - Y[n][None, :, :]
        dY -= p.dx * p.nx * np.round(dY / (p.dx * p.nx))
        assert np.allclose(np.linalg.norm(dY, axis=2), np.linalg.norm(S[:, None] - S[None], axis=2), atol=1e-12)
    U = rng.standard_normal(6 * M)
    lam = rng.standard_normal(3 * M * nb)
    lhs = lam @ o.multiply_by_K_at_midstep(U)
    rhs = U @ o.multiply_by_KT_at_midstep(lam)
    assert abs(lhs - rhs) < 1e-12 * abs(lhs)
    o.set_up_gaussians()
    b = rng.standard_normal(p.system_size)
    o.set_RHS(b)
    st, soln, it, rel = o.invert_saddle_point_system()
    assert st == 0 and rel < 1e-12
    r = o.multiply_by_saddle_point_matrix(soln) - b
    assert np.linalg.norm(r) < 1e-9 * np.linalg.norm(b)
    o.close()
