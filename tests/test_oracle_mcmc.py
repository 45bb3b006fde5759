"""Pair potential and Metropolis Monte Carlo in the oracle (main.cpp:113-210,
collection_of_rigid_bodies.cpp:666-705, linked_list.cpp:283-360).  The
potential must equal the sum of the pair energies over the reference's pair set
(the half-shell cell traversal, checked bit-for-bit elsewhere), computed here
with numpy from the same pairs; and for the cut-off polynomial potential the sum
over all inter-body pairs (brute force, minimum image).  A Metropolis run must
keep the reference's bookkeeping: one step per accepted or rejected proposal,
the acceptance ratio as a 20-step running mean, the scale moving by 2%."""
import numpy as np
import pytest

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200 import configs


def energy(r, p):
    a, kT = p.blob_radius, p.kT
    if p.potential == 3:
        rc, fs = p.steric_rc, p.steric_fs
        s = np.linspace(0.0, 1.0, 4001)
        out = np.zeros_like(r)
        for i, ri in enumerate(r):
            if ri < rc:
                x = ri + (rc - ri) * s
                f = fs * ((rc * rc - x * x) / (rc * rc - 4 * a * a)) ** 4
                out[i] = np.trapezoid(f, x)
        return out
    U0, b = 20.0 * kT, 0.5 * a
    e = np.where(r < 2 * a, U0 + U0 * (2 * a - r) / b, U0 * np.exp((2 * a - r) / b))
    if p.potential in (1, 2):
        A, lam = 5.0 * kT, 0.5 * a
        t = A * np.exp(-(a / lam) ** 2)
        inside = -t + 2 * a * (2 * a - r) * t / lam ** 2
        outside = -A * np.exp(-((r - 3 * a) / lam) ** 2)
        if p.potential == 2:
            t2 = A * np.exp(-(1.5 * a / lam) ** 2)
            inside = inside + t2 - 3 * a * (2 * a - r) * t2 / lam ** 2
            outside = outside + A * np.exp(-((r - 3.5 * a) / lam) ** 2)
        e = e + np.where(r < 2 * a, inside, outside)
    return e


def _close_rods(potential):
    # 32 rods in a small box so that many pairs interact
    p, ref, x, q, fe = configs.rod_suspension(M=32, grid=32, L=24.0, seed=3)
    p = p.copy(potential=potential, ncells=max(3, int(24.0 // 7.0)))
    return p, ref, x, q, fe


@pytest.mark.parametrize("potential", [0, 1, 2, 3])
def test_potential_is_the_pair_sum(potential):
    p, ref, x, q, fe = _close_rods(potential)
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    U = o.calculate_potential()
    Y = o.get_all_blob_pos().reshape(-1, 3)
    pairs = o.list_get_pairs()
    d = Y[pairs[:, 0]] - Y[pairs[:, 1]]
    L = p.box
    d -= np.array(L) * np.trunc(2.0 * d / np.array(L))
    r = np.linalg.norm(d, axis=1)
    tol = 1e-6 if potential == 3 else 1e-12
    assert abs(U - energy(r, p).sum()) <= tol * max(1.0, abs(U))
    if potential == 3:  # cut-off below the cell width: every close pair is in the set
        n = len(Y)
        body = np.arange(n) // p.blobs_per_body
        i, j = np.triu_indices(n, 1)
        keep = body[i] != body[j]
        dd = Y[i[keep]] - Y[j[keep]]
        dd -= np.array(L) * np.round(dd / np.array(L))
        assert abs(U - energy(np.linalg.norm(dd, axis=1), p).sum()) <= 1e-6 * max(1.0, abs(U))


def test_mcmc_bookkeeping():
    p, ref, x, q, fe = _close_rods(0)
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    U0 = o.calculate_potential()
    st, state = o.mcmc_run(42, 300)
    assert st == 0 and state.steps == 300 and state.attempts == 300
    assert 0.0 < state.acceptance_ratio < 1.0
    assert abs(state.potential - o.calculate_potential()) <= 1e-12 * max(1.0, abs(U0))
    # the scale is the start value times 1.02^up * 0.98^down with up + down = 300
    k = np.log(state.scale / (0.1 * p.blob_radius))
    up = (k - 300 * np.log(0.98)) / (np.log(1.02) - np.log(0.98))
    assert abs(up - round(up)) < 1e-6
    # continuing a run reproduces one long run
    o2 = Oracle(p, ref)
    o2.set_bodies(x, q)
    st2, s2 = o2.mcmc_run(42, 120)
    st2, s2 = o2.mcmc_run(42, 180, s2)
    assert s2.attempts == state.attempts and s2.scale == state.scale
    xa, qa = o.get_bodies()
    xb, qb = o2.get_bodies()
    assert np.array_equal(xa, xb) and np.array_equal(qa, qb)
