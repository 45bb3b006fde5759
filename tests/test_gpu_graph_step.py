"""Device-resident steps (fcm_step_async / fcm_step_wait / fcm_step_many): the
whole step as one CUDA graph with the GMRES iterations and refinement sweeps as
device-side conditional loops.  The same kernels run in the same order as in
the host-driven fcm_step, so trajectories must agree to round-off (1e-12
absolute on positions and quaternions; they are expected to be identical), and
the step records (iterations, sweeps, residual, divU) must agree."""
import numpy as np
import pytest

from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Suspension, step_many

pytestmark = pytest.mark.gpu


def _make(p, ref, x, q, fe):
    s = Suspension(p, ref)
    s.set_bodies(x, q)
    s.set_external_forces(fe)
    s.produce_reference_matrices()
    return s


@pytest.mark.parametrize("algorithm,precision", [(2, 0), (2, 1), (1, 0), (1, 1)])
def test_graph_steps_match_host_steps(gpu, algorithm, precision):
    p, ref, x, q, fe = configs.workload("rods32_L64_g64", algorithm=algorithm, precision=precision,
                                        gmres_tol=1e-8 if precision else 1e-10)
    a = _make(p, ref, x, q, fe)
    b = _make(p, ref, x, q, fe)
    for i in range(4):
        st_a, ia = a.step(1234, i)
        b.step_async(1234, i)
        st_b, ib = b.step_wait()
        assert st_a == st_b == 0
        assert ia.gmres_iters == ib.gmres_iters, i
        assert ia.refinement_sweeps == ib.refinement_sweeps, i
        assert abs(ia.gmres_rel_residual - ib.gmres_rel_residual) <= 1e-12 * max(1.0, ia.gmres_rel_residual)
        assert abs(ia.divU - ib.divU) <= 1e-12 * max(1.0, abs(ia.divU))
    xa, qa = a.get_bodies()
    xb, qb = b.get_bodies()
    assert np.max(np.abs(xa - xb)) <= 1e-12
    assert np.max(np.abs(qa - qb)) <= 1e-12


def test_graph_step_not_converged_and_refusals(gpu):
    p, ref, x, q, fe = configs.workload("rods32_L64_g64", gmres_max_iter=3)
    a = _make(p, ref, x, q, fe)
    b = _make(p, ref, x, q, fe)
    for i in range(3):
        st_a, ia = a.step(7, i)
        b.step_async(7, i)
        st_b, ib = b.step_wait()
        assert st_a == st_b == 0
        assert ia.status == ib.status == 5  # FCM_ERR_NOT_CONVERGED recorded, step taken
        assert ia.gmres_iters == ib.gmres_iters == 3
    assert np.max(np.abs(a.get_bodies()[0] - b.get_bodies()[0])) <= 1e-12
    from timstochrigidbodiessim_b200.capi import FcmError
    b.step_async(7, 3)
    with pytest.raises(FcmError):
        b.step_async(7, 4)  # one step in flight per context
    with pytest.raises(FcmError):
        b.step(7, 4)
    b.step_wait()
    with pytest.raises(FcmError):
        b.step_wait()  # nothing in flight


def test_step_many_matches_single_steps(gpu):
    import torch
    insts = configs.ensemble(3, seed0=5)
    solo = [_make(p, ref, x, q, fe) for p, ref, x, q, fe in insts]
    many = [_make(p, ref, x, q, fe) for p, ref, x, q, fe in insts]
    streams = [torch.cuda.Stream() for _ in many]
    for s, st in zip(many, streams):
        s.set_stream(st)
    seeds = [5 + i for i in range(3)]
    for k in range(3):
        infos = step_many(many, seeds, k)
        for i, s in enumerate(solo):
            st, inf = s.step(seeds[i], k)
            assert inf.gmres_iters == infos[i].gmres_iters
    for a, b in zip(solo, many):
        assert np.max(np.abs(a.get_bodies()[0] - b.get_bodies()[0])) <= 1e-12
        assert np.max(np.abs(a.get_bodies()[1] - b.get_bodies()[1])) <= 1e-12
