"""GPU path against the CPU FP64 oracle at the size of the plain-FP64 benchmark:
2048 straight 6-blob rods (12,288 blobs) at volume fraction 0.10 on a 256^3 grid
(rods2048_phi0.10_g256), plus a reduced box at the blob density of the 512^3
cluster suspension (about 57 blobs meet each 8^3 tile).

Checks, as the target states them:
- cell ids, the inter-body pair set and the Gaussian stencil indices bit-exact
  (linked_list.cpp:74-102, :192-281; fcm_fluid_solver.cpp:131-165);
- M F and the random velocities from six injected 256^3 stress arrays within
  1e-10 relative, blob velocities and velocity grids (fcm_fluid_solver.cpp:167-424,
  :552-701);
- one full FP64 Euler-Maruyama step with the stress injected: bodies within 1e-9
  (main.cpp:222-340, gmres_solver.cpp:148-306);
- the mixed-precision solve (FP32 grids inside FP64 refinement to 1e-8) against
  the oracle's FP64 solve of the same right-hand side within 1e-6 relative.
The oracle runs on every host thread; its solve is done once per module.
"""
import os

import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle, lib
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _injected_stress(p, seed):
    """Six real stress arrays in the reference's padded layout, N(0,1) scaled as
    fcm_fluid_solver.cpp:169-170 scales them (var2 on the diagonal, var1 off it)."""
    var1 = np.sqrt(2.0 * p.kT * p.viscosity / (p.dx ** 3 * p.dt))
    var2 = np.sqrt(2.0) * var1
    rng = np.random.default_rng(seed)
    P = p.nx * p.ny * p.pad
    return [rng.standard_normal(P) * v for v in (var2, var2, var2, var1, var1, var1)]


@pytest.fixture(scope="module")
def cfg1(gpu):
    lib().orc_set_threads(os.cpu_count() or 1)
    p, ref, x, q, fe = configs.workload("rods2048_phi0.10_g256")
    g = Suspension(p, ref)
    o = Oracle(p, ref)
    for s in (g, o):
        s.set_bodies(x, q)
        s.set_external_forces(fe)
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    yield p, ref, x, q, fe, g, o
    g.close()
    o.close()


def test_config1_blob_positions_cells_pairs_bitexact(cfg1):
    p, ref, x, q, fe, g, o = cfg1
    assert np.array_equal(g.get_all_blob_pos(), o.get_all_blob_pos())
    g.list_populate()
    o.list_populate()
    assert np.array_equal(g.list_get_cells(), o.list_get_cells())
    pg, po = g.list_get_pairs(), o.list_get_pairs()
    assert len(po) > 1000
    assert np.array_equal(pg, po)


def test_config1_gaussian_indices_bitexact(cfg1):
    p, ref, x, q, fe, g, o = cfg1
    ig, wg = g.get_gaussians()
    io, wo = o.get_gaussians()
    assert np.array_equal(ig, io)
    # the weights are exp() of the same argument: CUDA's and the host's exp agree
    # to within an ulp or two
    assert np.abs(wg - wo).max() <= 4e-16 * np.abs(wo).max()


def test_config1_mobility_and_grids(cfg1):
    p, ref, x, q, fe, g, o = cfg1
    F = np.random.default_rng(21).standard_normal(3 * p.num_blobs)
    for s in (g, o):
        s.set_up_force_distribution(F)
        s.produce_deterministic_velocity_field()
    Vg = g.calculate_deterministic_blob_velocities()
    Vo = o.calculate_deterministic_blob_velocities()
    assert rel_err(Vg, Vo) < TOL
    ug = g.get_velocity_field(0)
    for c in range(3):
        assert rel_err(ug[c], o.get_grid(3 + c)) < TOL


def test_config1_random_velocities_from_injected_stress(cfg1):
    p, ref, x, q, fe, g, o = cfg1
    s6 = _injected_stress(p, 31)
    for s in (g, o):
        s.inject_random_stress(s6)
    assert rel_err(g.calculate_random_blob_velocities(), o.calculate_random_blob_velocities()) < TOL
    ug = g.get_velocity_field(1)
    for c in range(3):
        assert rel_err(ug[c], o.get_grid(6 + c)) < TOL


@pytest.fixture(scope="module")
def cfg1_step(cfg1):
    """One EM step with injected stress on both sides.  The preconditioner's
    reference matrices are the GPU's, handed to the oracle, so both solve with the
    same preconditioner.  Returns the oracle's FP64 solve and RHS as well."""
    p, ref, x, q, fe, g, o = cfg1
    g.produce_reference_matrices()
    Minv, N, _ = g.get_reference_matrices()
    o.set_reference_matrices(Minv, N)
    s6 = _injected_stress(p, 41)
    out = {}
    for tag, s in (("gpu", g), ("oracle", o)):
        s.set_bodies(x, q)
        s.fill_all_blob_pos()
        s.inject_random_stress(s6)
        s.set_up_gaussians()
        s.calculate_random_blob_velocities()
        s.calculate_forces()
        s.assemble_RHS()
        rhs = s.get_RHS()
        st, soln, it, rel = s.invert_saddle_point_system()
        s.end_of_step_update(soln[3 * p.num_blobs:], 1.0)
        out[tag] = dict(status=st, soln=soln, iters=it, rel=rel, rhs=rhs, bodies=s.get_bodies())
    return out, Minv, N


def test_config1_em_step_injected_noise(cfg1, cfg1_step):
    p = cfg1[0]
    out, _, _ = cfg1_step
    G, O = out["gpu"], out["oracle"]
    assert G["status"] == 0 and O["status"] == 0
    assert rel_err(G["rhs"], O["rhs"]) < TOL
    assert abs(G["iters"] - O["iters"]) <= 1
    assert rel_err(G["soln"], O["soln"]) < 1e-9
    (xg, qg), (xo, qo) = G["bodies"], O["bodies"]
    assert np.abs(xg - xo).max() < 1e-9
    assert np.abs(qg - qo).max() < 1e-9
    assert np.abs(xg - cfg1[2]).max() > 1e-6  # the bodies moved


def test_config1_mixed_precision_solve_vs_oracle(cfg1, cfg1_step):
    """The FP32-grid solve with FP64 refinement to 1e-8 of the oracle's RHS:
    body and blob velocities within 1e-6 of the oracle's FP64 solve."""
    p, ref, x, q, fe = cfg1[:5]
    out, Minv, N = cfg1_step
    O = out["oracle"]
    pm = p.copy(precision=1, gmres_tol=1e-8)
    m = Suspension(pm, ref)
    m.set_bodies(x, q)
    m.set_external_forces(fe)
    m.set_reference_matrices(Minv, N)
    m.fill_all_blob_pos()
    m.set_up_gaussians()
    m.set_RHS(O["rhs"])
    st, soln, it, rel = m.invert_saddle_point_system()
    m.close()
    assert st == 0
    Nb = p.num_blobs
    err_U = rel_err(soln[3 * Nb:], O["soln"][3 * Nb:])
    err_l = rel_err(soln[:3 * Nb], O["soln"][:3 * Nb])
    assert err_U < 1e-6 and err_l < 1e-6, (err_U, err_l)


def test_dense_tiles_at_cluster_density(gpu):
    """A 64^3 box at the grid spacing and volume fraction of the 512^3 cluster
    suspension (DX = 0.394a, phi = 0.20, 12-blob clusters): about 57 blobs meet
    each 8^3 tile, so every tile takes several staging rounds.  Both FP64 spread
    kernels (persistent pipelined and one CTA per tile) give the oracle's grid and
    the three tiled interpolation kernels its velocities within 1e-10; the FP32
    grid within 1e-6."""
    lib().orc_set_threads(os.cpu_count() or 1)
    grid, phi, nb = 64, 0.20, 12
    dx = configs.box_for_volume_fraction(393216, 0.20) / 512
    L = grid * dx
    M = int(round(phi * L ** 3 / (4.0 / 3.0 * np.pi) / nb))
    rng = np.random.default_rng(8)
    ref = configs.random_walk_cluster(rng, nb, draws=1)
    Y = np.concatenate([(rng.uniform(0, L, 3) + ref) % L for _ in range(M)]).ravel()
    p = FcmParams.defaults(nx=grid, ny=grid, nz=grid, ngauss=20, dx=dx, num_bodies=M, blobs_per_body=nb, ncells=3,
                           precision=1)
    g = Suspension(p, ref.ravel())
    o = Oracle(p.copy(precision=0), ref.ravel())
    for s in (g, o):
        s.set_up_gaussians(Y)
    ind, _ = g.get_gaussians()
    tiles = {}
    for b in range(M * nb):
        ts = [set(ind[b, d] // 8) for d in range(3)]
        for tx in ts[0]:
            for ty in ts[1]:
                for tz in ts[2]:
                    tiles[(tx, ty, tz)] = tiles.get((tx, ty, tz), 0) + 1
    assert np.mean(list(tiles.values())) > 45, np.mean(list(tiles.values()))
    F = rng.standard_normal(3 * M * nb)
    o.set_up_force_distribution(F)
    o.produce_deterministic_velocity_field()
    Vo = o.calculate_deterministic_blob_velocities()
    for variant in (0, 1, 2, 3):
        v = g.get_variants()
        g.set_variants([variant, v[1], variant, v[3], min(variant, 2), min(variant, 2)])
        g.set_up_force_distribution(F)
        g.produce_deterministic_velocity_field()
        assert rel_err(g.calculate_deterministic_blob_velocities(), Vo) < TOL, variant
        ug = g.get_velocity_field(0)
        for c in range(3):
            assert rel_err(ug[c], o.get_grid(3 + c)) < TOL
        g.spread(F, 1)
        g.stokes_solve(1)
        assert rel_err(g.interp(1), Vo) < 1e-6, variant
    g.close()
    o.close()
