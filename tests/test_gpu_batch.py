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
