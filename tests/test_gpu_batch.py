"""Batches (fcm_batch_*): many suspensions stepped together, the solves in
lockstep as batched kernels inside one CUDA graph per step.  Every member must
follow the trajectory of the same suspension stepped alone with fcm_step: the
batched kernels run each member's arithmetic in the single-suspension order
(its own reduction grids included), so the only possible difference is cuFFT's
choice of kernels for a batch of transforms; positions and quaternions must
agree to 1e-9 absolute (FP64) or 1e-8 (mixed, refined to 1e-8), and the GMRES
iteration counts to within one."""
import numpy as np
import pytest

from timstochrigidbodiessim_b200 import capi, configs
from timstochrigidbodiessim_b200.capi import FcmError
from timstochrigidbodiessim_b200.fcm import Batch, Suspension

pytestmark = pytest.mark.gpu


def _solo(p, ref, x, q, fe):
    s = Suspension(p, ref)
    s.set_bodies(x, q)
    s.set_external_forces(fe)
    s.produce_reference_matrices()
    return s


def _batch(insts):
    b = Batch([(p, ref) for p, ref, *_ in insts])
    for m, (p, ref, x, q, fe) in zip(b.members, insts):
        m.set_bodies(x, q)
        m.set_external_forces(fe)
        m.produce_reference_matrices()
    return b


@pytest.mark.parametrize("precision,algorithm", [(1, 2), (0, 2), (1, 1)])
def test_batch_members_follow_single_steps(gpu, precision, algorithm):
    insts = []
    for p, ref, x, q, fe in configs.ensemble(3, seed0=11):
        pp = p.copy(precision=precision, algorithm=algorithm)
        if precision == 1:
            pp.gmres_tol = 1e-8
        insts.append((pp, ref, x, q, fe))
    solo = [_solo(*i) for i in insts]
    b = _batch(insts)
    seeds = [11, 12, 13]
    for k in range(3):  # the first batch step is host-driven, the others run the graph
        infos = b.step(seeds, k)
        for i, s in enumerate(solo):
            st, inf = s.step(seeds[i], k)
            assert abs(inf.gmres_iters - infos[i].gmres_iters) <= 1, (k, i)
            assert infos[i].status in (0, 5)
    # FP64 solves (tol 1e-10) agree to 1e-9; mixed solves, refined to 1e-8, whose
    # FP32 arithmetic in the batched kernels rounds differently, to 1e-8
    tol = 1e-8 if precision == 1 else 1e-9
    for s, m in zip(solo, b.members):
        xs, qs = s.get_bodies()
        xm, qm = m.get_bodies()
        assert np.max(np.abs(xs - xm)) <= tol
        assert np.max(np.abs(qs - qm)) <= tol
    b.close()


def test_batch_refuses_bad_members(gpu):
    raw = configs.ensemble(2, seed0=2)
    p0, r0 = raw[0][0], raw[0][1]
    p1 = raw[1][0].copy(precision=1 - raw[1][0].precision)
    with pytest.raises(FcmError):
        Batch([(p0, r0), (p1, raw[1][1])])  # mixed precisions
    b = Batch([(p0, r0)])
    assert capi.load().fcm_destroy(b.members[0].h) != 0  # members belong to the batch
    b.close()


def test_batch_long_x_grid_mixed_paths(gpu):
    """Members with nx = 384, whose FP32 solves use the fused x-transform and whose
    FP64 residuals the 3D transforms with k_b_project: batch steps follow single
    steps (mixed precision, 1e-8)."""
    from timstochrigidbodiessim_b200.params import FcmParams, rod_reference_positions
    ref = np.array(rod_reference_positions(3, 2.2))
    insts = []
    for seed in (1, 2):
        p = FcmParams.defaults(nx=384, ny=16, nz=16, ngauss=8, dx=0.5, num_bodies=8, blobs_per_body=3, ncells=3,
                               potential=3, gmres_tol=1e-8, gmres_max_iter=100, precision=1, dt=0.01)
        rng = np.random.default_rng(seed)
        x = np.column_stack([20.0 * np.arange(8) + rng.uniform(0, 5, 8), rng.uniform(3, 5, 8),
                             rng.uniform(3, 5, 8)]).ravel()
        q = configs.random_unit_quaternions(rng, 8).ravel()
        fe = np.zeros(48)
        fe[2::6] = -1.0
        insts.append((p, ref, x, q, fe))
    solo = [_solo(*i) for i in insts]
    b = _batch(insts)
    for k in range(3):
        infos = b.step([3, 4], k)
        for i, s in enumerate(solo):
            st, inf = s.step([3, 4][i], k)
            assert st == 0 and infos[i].status == 0
            assert abs(inf.gmres_iters - infos[i].gmres_iters) <= 1
    for s, m in zip(solo, b.members):
        assert np.max(np.abs(s.get_bodies()[0] - m.get_bodies()[0])) <= 1e-8
        assert np.max(np.abs(s.get_bodies()[1] - m.get_bodies()[1])) <= 1e-8
    b.close()


def test_batch_members_against_the_oracle(gpu):
    """A three-member FP64 batch of uneven suspensions (64^3, 96^3 and 128^3 grids,
    50 / 150 / 300 rods) against each member's own CPU oracle, not against a solo
    GPU step: M F through the member context within 1e-10, then three
    deterministic EM steps of the batch (the lockstep batched spread, projection,
    interpolation and GMRES kernels inside the step graph from the second step on)
    against the oracle's steps, bodies within 1e-9 and GMRES iterations within one
    (gmres_solver.cpp:148-306, fcm_fluid_solver.cpp:363-424, :552-701)."""
    import os

    from tests.conftest import rel_err
    from tests.oracle_lib import Oracle, lib
    lib().orc_set_threads(os.cpu_count() or 1)
    insts = []
    for M, grid, phi, seed in ((50, 64, 0.05, 21), (150, 96, 0.10, 22), (300, 128, 0.15, 23)):
        insts.append(configs.rod_suspension(M=M, grid=grid, phi=phi, seed=seed, gmres_tol=1e-10, noise=0))
    b = _batch(insts)
    oracles = []
    for m, (p, ref, x, q, fe) in zip(b.members, insts):
        o = Oracle(p, ref)
        o.set_bodies(x, q)
        o.set_external_forces(fe)
        Minv, N, _ = m.get_reference_matrices()
        o.set_reference_matrices(Minv, N)  # the same preconditioner on both sides
        oracles.append(o)
    rng = np.random.default_rng(3)
    for m, o, (p, *_rest) in zip(b.members, oracles, insts):
        F = rng.standard_normal(3 * p.num_blobs)
        for s in (m, o):
            s.fill_all_blob_pos()
            s.set_up_gaussians()
        assert rel_err(m.apply_mobility(F), o.apply_mobility(F)) < 1e-10
    for k in range(3):
        infos = b.step([0, 0, 0], k)
        for i, o in enumerate(oracles):
            so, io = o.step(0, k)
            assert so == 0 and infos[i].status == 0
            assert abs(io.gmres_iters - infos[i].gmres_iters) <= 1, (k, i)
            xm, qm = b.members[i].get_bodies()
            xo, qo = o.get_bodies()
            assert np.abs(xm - xo).max() < 1e-9, (k, i)
            assert np.abs(qm - qo).max() < 1e-9, (k, i)
    for o, (p, ref, x, q, fe) in zip(oracles, insts):
        assert np.abs(o.get_bodies()[0] - x).max() > 1e-5  # the bodies moved
        o.close()
    b.close()
