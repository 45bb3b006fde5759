"""Per-body shapes on the GPU (fcm_set_body_shapes) against the CPU oracle's
per-body restatement.  No counterpart in the reference: its bodies share one
blob_ref_pos (collection_of_rigid_bodies.hpp:24); the per-body path applies the
reference's formulas (collection_of_rigid_bodies.cpp:155-193, :566-621,
:707-757; gmres_solver.cpp:85-146) with each body's own shape and blocks.

Tolerances as for the shared shape: positions bit-exact; K, K^T, P^-1 and
saddle-point products 1e-10; preconditioner blocks 1e-12; GMRES solutions 1e-9;
bodies after three steps with injected stress 1e-9.
"""
import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from tests.test_gpu_parity import _em_step_manual
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.capi import FcmError
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _clusters(M=27, nb=6, grid=48, dx=0.5, algorithm=2, precision=0, seed=12):
    """M bodies of M distinct random-walk shapes of nb blobs, one per cell of a
    3x3x3 lattice in a grid^3 box; params, shapes (3*nb*M), x, q, forces."""
    rng = np.random.default_rng(seed)
    shapes = np.concatenate([configs.random_walk_cluster(rng, nb, draws=4).ravel() for _ in range(M)])
    L = grid * dx
    side = round(M ** (1 / 3))
    ijk = np.array([[i, j, k] for i in range(side) for j in range(side) for k in range(side)])[:M]
    x = ((ijk + 0.5) * (L / side)).ravel()
    q = configs.random_unit_quaternions(rng, M).ravel()
    p = FcmParams.defaults(nx=grid, ny=grid, nz=grid, ngauss=12, dx=dx, num_bodies=M, blobs_per_body=nb, ncells=3,
                           potential=3, steric_fs=40.0, steric_rc=2.2, gmres_tol=1e-12, gmres_max_iter=200,
                           algorithm=algorithm, precision=precision, noise=0)
    fe = np.zeros(6 * M)
    fe[2::6] = -1.0
    return p, shapes, x, q, fe


def _pair(p, shapes, x, q, fe):
    nb = p.blobs_per_body
    g = Suspension(p, shapes[:3 * nb])
    o = Oracle(p.copy(precision=0), shapes[:3 * nb])
    g.set_body_shapes(shapes)
    o.set_body_shapes(shapes)
    o.produce_body_preconditioners()
    for s in (g, o):
        s.set_bodies(x, q)
        s.set_external_forces(fe)
    return g, o


def test_body_preconditioners_match_the_oracle(gpu):
    p, shapes, x, q, fe = _clusters()
    g, o = _pair(p, shapes, x, q, fe)
    Mg, Ng, Kg = g.get_body_preconditioners()
    Mo, No, Ko = o.get_body_preconditioners()
    n3 = 3 * p.blobs_per_body
    # the library returns each block row-major; the oracle's flat blocks are column-major
    assert rel_err(Mg.transpose(0, 2, 1).ravel(), Mo) < 1e-12
    assert rel_err(Ng.transpose(0, 2, 1).ravel(), No) < 1e-12
    assert rel_err(Kg.transpose(0, 2, 1).ravel(), Ko) < 1e-12
    assert Mg.shape == (p.num_bodies, n3, n3)
    # single-shape calls are refused once the bodies have their own shapes
    with pytest.raises(FcmError):
        g.produce_reference_matrices()
    g.close()
    o.close()


def test_per_body_products_and_solve(gpu):
    p, shapes, x, q, fe = _clusters()
    g, o = _pair(p, shapes, x, q, fe)
    for s in (g, o):
        s.fill_all_blob_pos()
    assert np.array_equal(g.get_all_blob_pos(), o.get_all_blob_pos())
    rng = np.random.default_rng(2)
    U = rng.standard_normal(6 * p.num_bodies)
    lam = rng.standard_normal(3 * p.num_blobs)
    assert rel_err(g.multiply_by_K_at_midstep(U), o.multiply_by_K_at_midstep(U)) < TOL
    assert rel_err(g.multiply_by_KT_at_midstep(lam), o.multiply_by_KT_at_midstep(lam)) < TOL
    v = rng.standard_normal(p.system_size)
    assert rel_err(g.multiply_by_Pinv(v), o.multiply_by_Pinv(v)) < TOL
    for s in (g, o):
        s.set_up_gaussians()
    assert rel_err(g.multiply_by_saddle_point_matrix(v), o.multiply_by_saddle_point_matrix(v)) < TOL
    for s in (g, o):
        s.calculate_forces()
        s.assemble_RHS()
    assert rel_err(g.get_RHS(), o.get_RHS()) < TOL
    sg, xg, itg, _ = g.invert_saddle_point_system()
    so, xo, ito, _ = o.invert_saddle_point_system()
    assert sg == 0 and so == 0 and abs(itg - ito) <= 1
    assert rel_err(xg, xo) < 1e-9
    g.close()
    o.close()


@pytest.mark.parametrize("algorithm", [2, 1])
def test_per_body_steps_with_injected_noise(gpu, algorithm):
    """Three EM or GDC steps (the GDC midstep uses each body's own ref_KTKinv)."""
    p, shapes, x, q, fe = _clusters(algorithm=algorithm)
    g, o = _pair(p, shapes, x, q, fe)
    rng = np.random.default_rng(6)
    for step in range(3):
        s6 = [rng.standard_normal(p.nx * p.ny * p.pad) * 0.05 for _ in range(6)]
        rg = _em_step_manual(g, s6, gdc=(algorithm == 1))
        ro = _em_step_manual(o, s6, gdc=(algorithm == 1))
        assert rg[0] == 0 and ro[0] == 0
        xg, qg = g.get_bodies()
        xo, qo = o.get_bodies()
        assert np.abs(xg - xo).max() < 1e-9, step
        assert np.abs(qg - qo).max() < 1e-9, step
    assert np.abs(xg - x).max() > 1e-4
    g.close()
    o.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_per_body_graph_steps_equal_host_steps(gpu, precision):
    """Noise-on steps: host-driven and device-resident graph steps of the same
    per-body suspension agree bit for bit (FP64 and mixed precision)."""
    p, shapes, x, q, fe = _clusters(precision=precision)
    p = p.copy(noise=1, gmres_tol=1e-10 if precision == 0 else 1e-8)
    runs = []
    for graph in (False, True):
        s = Suspension(p, shapes[:3 * p.blobs_per_body])
        s.set_body_shapes(shapes)
        s.set_bodies(x, q)
        s.set_external_forces(fe)
        for k in range(3):
            if graph:
                s.step_async(5, k)
                assert s.step_wait()[0] == 0
            else:
                assert s.step(5, k)[0] == 0
        runs.append(s.get_bodies())
        s.close()
    assert np.array_equal(runs[0][0], runs[1][0]) and np.array_equal(runs[0][1], runs[1][1])


def test_per_body_metropolis_matches_the_oracle(gpu):
    """Metropolis steps with per-body shapes (the rotation scale is the largest blob
    distance over all shapes): same decisions and bodies as the oracle."""
    p, shapes, x, q, fe = _clusters()
    g, o = _pair(p, shapes, x, q, fe)
    sg = g.mcmc_run(77, 60)
    _, so = o.mcmc_run(77, 60)
    assert sg.steps == so.steps and sg.attempts == so.attempts
    assert abs(sg.acceptance_ratio - so.acceptance_ratio) < 1e-12
    assert np.abs(g.get_bodies()[0] - o.get_bodies()[0]).max() < 1e-12
    assert np.abs(g.get_bodies()[1] - o.get_bodies()[1]).max() < 1e-12
    g.close()
    o.close()


def test_one_shape_through_the_per_body_path_is_the_shared_shape(gpu):
    """Every body given the same shape: the per-body kernels produce the shared
    shape's positions, K, K^T and P^-1 bit for bit (same blocks)."""
    p, ref, x, q, fe = configs.rod_suspension(M=16, grid=32, L=24.0, nb=4, seed=3, noise=0, ngauss=12)
    ref = np.asarray(ref).ravel()
    a = Suspension(p, ref)
    b = Suspension(p, ref)
    b.set_body_shapes(np.tile(ref, p.num_bodies))
    Mb, Nb_, _ = b.get_body_preconditioners()
    a.set_reference_matrices(Mb[0].T.ravel(), Nb_[0].T.ravel())
    for s in (a, b):
        s.set_bodies(x, q)
        s.fill_all_blob_pos()
    assert np.array_equal(a.get_all_blob_pos(), b.get_all_blob_pos())
    rng = np.random.default_rng(0)
    U = rng.standard_normal(6 * p.num_bodies)
    lam = rng.standard_normal(3 * p.num_blobs)
    v = rng.standard_normal(p.system_size)
    assert np.array_equal(a.multiply_by_K_at_midstep(U), b.multiply_by_K_at_midstep(U))
    assert np.array_equal(a.multiply_by_KT_at_midstep(lam), b.multiply_by_KT_at_midstep(lam))
    assert np.array_equal(a.multiply_by_Pinv(v), b.multiply_by_Pinv(v))
    a.close()
    b.close()
