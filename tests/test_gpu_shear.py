"""Shear forcing on the GPU (fcm_produce_shear_velocity_field,
fcm_calculate_shear_blob_velocities, fcm_fluid_x_velocity_in_y: the
SHEARING_FORCES paths of fcm_fluid_solver.cpp:703-842 and :489-550,
gmres_solver.cpp:62-64 and main.cpp:270-272, :371-433) against the oracle on the
same inputs: the imposed flow, Vshear and the x-velocity profile within 1e-10
relative, and GDC / EM steps with the flow on -- host-driven, as graph steps and
as a batch -- on the oracle's trajectory (1e-9 absolute)."""
import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Batch, Suspension

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _pair(p, ref, x, q, fe=None):
    out = []
    for cls in (Suspension, Oracle):
        s = cls(p, ref)
        s.set_bodies(x, q)
        if fe is not None:
            s.set_external_forces(fe)
        out.append(s)
    return out


@pytest.mark.parametrize("scale,w", [(1.0, 1.0), (2.5, 0.75)])
def test_shear_flow_matches_oracle(gpu, scale, w):
    # w = 0.75 is not periodic on the grid: the forcing then has every y mode
    p, ref, x, q, fe = configs.workload("rods32_L64_g64")
    g, o = _pair(p, ref, x, q)
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        s.produce_shear_velocity_field(scale, w)
    shape = (p.nx, p.ny, p.pad)
    ug = g.get_velocity_field(2)
    for c in range(3):
        a = ug[c].reshape(shape)[:, :, :p.nz]
        b = o.get_grid(3 + c).reshape(shape)[:, :, :p.nz]
        if c == 0:
            assert rel_err(a, b) < TOL
        else:  # no y or z flow: round-off only
            assert np.abs(a - b).max() < 1e-12 * np.abs(ug[0]).max()
    assert rel_err(g.calculate_shear_blob_velocities(), o.calculate_shear_blob_velocities()) < TOL
    F = np.random.default_rng(3).standard_normal(3 * p.num_blobs)
    assert rel_err(g.fluid_x_velocity_in_y(F), o.fluid_x_velocity_in_y(F)) < TOL
    assert rel_err(g.fluid_x_velocity_in_y(np.zeros_like(F)), o.fluid_x_velocity_in_y(np.zeros_like(F))) < TOL


def test_shear_rhs_matches_oracle(gpu):
    p, ref, x, q, fe = configs.workload("rods32_L64_g64")
    g, o = _pair(p, ref, x, q, fe)
    rng = np.random.default_rng(6)
    s6 = [rng.standard_normal(p.nx * p.ny * p.pad) * 0.05 for _ in range(6)]
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        s.inject_random_stress(s6)  # the same fluctuating stress on both sides
        s.calculate_random_blob_velocities()
        s.produce_shear_velocity_field(1.0, 1.0)
        s.calculate_shear_blob_velocities()
        s.calculate_forces()
        s.assemble_RHS()
    assert rel_err(g.get_RHS(), o.get_RHS()) < TOL
    # fcm.V is the random velocities still, Vshear went into the RHS beside it
    assert rel_err(g.get_V(), o.get_V()) < TOL


@pytest.mark.parametrize("algorithm", [1, 2])
def test_steps_with_shear_match_oracle(gpu, algorithm):
    # noise off: the oracle's fluctuations are drawn in real space, the library's in
    # Fourier space, so only deterministic steps can follow one trajectory
    p, ref, x, q, fe = configs.workload("rods32_L64_g64", algorithm=algorithm, gmres_tol=1e-12, noise=0)
    g, o = _pair(p, ref, x, q, fe)
    o.produce_reference_matrices()
    Minv, N, _ = o.get_reference_matrices()
    g.set_reference_matrices(Minv, N)
    for s in (g, o):
        s.produce_shear_velocity_field(2.0, 1.0)
    for step in range(3):
        sg, ig = g.step(99, step)
        so, io = o.step(99, step)
        assert sg == 0 and so == 0
    xg, qg = g.get_bodies()
    xo, qo = o.get_bodies()
    assert np.abs(xg - xo).max() < 1e-9
    assert np.abs(qg - qo).max() < 1e-9


def test_shear_in_graph_and_batch_steps(gpu):
    """Turning the flow on after graph steps recaptures the graphs: graph steps,
    batch steps and host-driven steps stay on one trajectory."""
    p, ref, x, q, fe = configs.workload("rods32_L64_g64", algorithm=1, gmres_tol=1e-10)

    def make(s):
        s.set_bodies(x, q)
        s.set_external_forces(fe)
        s.produce_reference_matrices()
        return s

    host = make(Suspension(p, ref))
    graph = make(Suspension(p, ref))
    batch = Batch([(p, ref)])
    make(batch.members[0])
    for k in range(2):  # graph captured without the flow
        host.step(5, k)
        graph.step_async(5, k)
        graph.step_wait()
        batch.step([5], k)
    for s in (host, graph, batch.members[0]):
        s.produce_shear_velocity_field(3.0, 2.0)
    for k in range(2, 5):
        host.step(5, k)
        graph.step_async(5, k)
        graph.step_wait()
        batch.step([5], k)
    xh, qh = host.get_bodies()
    # graph steps run the host-driven kernels in order; a batch may differ by
    # cuFFT's kernel choice for a batch of transforms
    for s, tol in ((graph, 1e-12), (batch.members[0], 1e-9)):
        xs, qs = s.get_bodies()
        assert np.abs(xs - xh).max() < tol
        assert np.abs(qs - qh).max() < tol
    # and the flow made a difference
    ref_run = make(Suspension(p, ref))
    for k in range(5):
        ref_run.step(5, k)
    assert np.abs(ref_run.get_bodies()[0] - xh).max() > 1e-6
    batch.close()
