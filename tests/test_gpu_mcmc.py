"""Pair potential and Metropolis Monte Carlo on the GPU (fcm_calculate_potential,
fcm_mcmc_run: the whole run is one CUDA graph with the loop on the device)
against the oracle on the same inputs and the same Philox uniforms.  The
potentials agree to 1e-12 relative; the runs take the same decisions (a flip
would need an energy difference within round-off of a uniform), so the final
bodies agree to 1e-12 and the scale, acceptance ratio and counters exactly
up to round-off of the energies."""
import numpy as np
import pytest

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Suspension

pytestmark = pytest.mark.gpu


def _close_rods(potential, skip=0):
    p, ref, x, q, fe = configs.rod_suspension(M=32, grid=32, L=24.0, seed=3)
    return p.copy(potential=potential, ncells=3, skip_on_overlap=skip), ref, x, q, fe


@pytest.mark.parametrize("potential", [0, 1, 2, 3])
def test_potential_matches_oracle(gpu, potential):
    p, ref, x, q, fe = _close_rods(potential)
    g, o = Suspension(p, ref), Oracle(p, ref)
    for s in (g, o):
        s.set_bodies(x, q)
    Ug, Uo = g.calculate_potential(), o.calculate_potential()
    assert abs(Ug - Uo) <= 1e-12 * max(1.0, abs(Uo))


@pytest.mark.parametrize("potential,skip", [(0, 0), (3, 0), (0, 1)])
def test_mcmc_matches_oracle(gpu, potential, skip):
    p, ref, x, q, fe = _close_rods(potential, skip)
    g, o = Suspension(p, ref), Oracle(p, ref)
    for s in (g, o):
        s.set_bodies(x, q)
    sg = g.mcmc_run(7, 150)
    _, so = o.mcmc_run(7, 150)
    assert (sg.steps, sg.attempts) == (so.steps, so.attempts)
    assert abs(sg.scale - so.scale) <= 1e-12 * so.scale
    assert abs(sg.acceptance_ratio - so.acceptance_ratio) <= 1e-12
    assert abs(sg.potential - so.potential) <= 1e-10 * max(1.0, abs(so.potential))
    xg, qg = g.get_bodies()
    xo, qo = o.get_bodies()
    assert np.max(np.abs(xg - xo)) <= 1e-12 and np.max(np.abs(qg - qo)) <= 1e-12


def test_mcmc_continues_across_calls(gpu):
    p, ref, x, q, fe = _close_rods(0)
    a, b = Suspension(p, ref), Suspension(p, ref)
    for s in (a, b):
        s.set_bodies(x, q)
    sa = a.mcmc_run(11, 100)
    sb = b.mcmc_run(11, 40)
    sb = b.mcmc_run(11, 60, sb)
    assert sa.attempts == sb.attempts and sa.scale == sb.scale
    assert np.array_equal(a.get_bodies()[0], b.get_bodies()[0])
    assert abs(sa.potential - a.calculate_potential()) <= 1e-12 * max(1.0, abs(sa.potential))
