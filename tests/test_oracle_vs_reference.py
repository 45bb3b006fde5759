"""The oracle against the reference itself.

The fixtures tests/golden/ref_<config>.npz were computed by the reference's own
classes, compiled unchanged from its sources with the project-written stand-ins
of oracle/ref_shim (tests/golden/make_ref_golden.py; recipe `make -C oracle
ref`).  The oracle, given the same compile-time parameters, bodies and noise
stream, must reproduce them:
- blob positions, cell ids and Gaussian stencil indices bit for bit, stencil
  weights to 1e-15, steric forces to 1e-13;
- M F, K, K^T, P^-1 and the saddle-point product to 1e-12;
- the probed reference matrices (3 nb full FCM solves) to 1e-9;
- random velocities from the same SPRNG stream to 1e-12;
- whole time steps (Euler-Maruyama in a periodic box; the generalised
  drifter-corrector in the reference's default slip channel), bodies to 1e-10
  and the GDC factor nu to 1e-9;
- the Metropolis-mode pair potential (soft sphere, hydrophilic) to 1e-12.
The fixtures hold the reference's numbers; nothing of the reference is needed
to run this test.
"""
import os

import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle, lib
from timstochrigidbodiessim_b200.params import FcmParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(config):
    path = os.path.join(GOLDEN, "ref_%s.npz" % config)
    if not os.path.exists(path):
        pytest.fail("missing fixture %s (tests/golden/make_ref_golden.py)" % path)
    return dict(np.load(path))


def _params(c, M, nb):
    """FcmParams of a reference build's compile-time parameters (ref_harness rh_config)."""
    return FcmParams.defaults(nx=int(c[2]), ny=int(c[3]), nz=int(c[4]), dx=float(c[5]), blob_radius=float(c[6]),
                              viscosity=float(c[7]), kT=float(c[8]), dt=float(c[9]), gmres_tol=float(c[10]),
                              gmres_max_iter=int(c[11]), ngauss=int(c[12]), ncells=int(c[13]),
                              slip_channel=int(c[14]), algorithm=int(c[15]) if int(c[15]) else 2,
                              potential=int(c[16]), fd_delta=float(c[17]), skip_on_overlap=int(c[18]),
                              num_bodies=M, blobs_per_body=nb, precision=0, noise=1)


def _oracle(g):
    c = g["cfg"]
    M, nb = int(c[0]), int(c[1])
    o = Oracle(_params(c, M, nb), g["blob_ref_pos"])
    return o, M, nb


@pytest.mark.parametrize("config", ["em_tetra", "gdc_rods_slip"])
def test_static_quantities(config):
    lib().orc_set_threads(os.cpu_count() or 1)
    g = _load(config)
    o, M, nb = _oracle(g)
    o.set_bodies(g["x"], g["q"])
    o.fill_all_blob_pos()
    assert np.array_equal(o.get_all_blob_pos(), g["Y"])
    o.list_populate()
    assert np.array_equal(o.list_get_cells(), g["cells"])
    o.set_up_gaussians()
    ind, w = o.get_gaussians()
    assert np.array_equal(ind, g["gauss_ind"])
    assert np.abs(w - g["gauss_w"]).max() <= 1e-15 * np.abs(g["gauss_w"]).max()
    o.calculate_forces()
    assert rel_err(o.get_blob_forces(), g["forces"]) < 1e-13
    assert rel_err(o.apply_mobility(g["F"]), g["V"]) < 1e-12
    assert rel_err(o.multiply_by_K_at_midstep(g["U"]), g["KU"]) < 1e-12
    assert rel_err(o.multiply_by_KT_at_midstep(g["lam"]), g["KTlam"]) < 1e-12
    o.set_reference_matrices(g["ref_Minv"], g["ref_N"])
    assert rel_err(o.multiply_by_Pinv(g["v"]), g["Pinv_v"]) < 1e-12
    o.fill_all_blob_pos()
    o.set_up_gaussians()
    assert rel_err(o.multiply_by_saddle_point_matrix(g["v"]), g["A_v"]) < 1e-12
    o.set_sequential_noise(True, 77, 0)
    o.produce_random_velocity_field(0, 0)
    assert rel_err(o.calculate_random_blob_velocities(), g["V_random"]) < 1e-12
    o.close()


@pytest.mark.parametrize("config", ["em_tetra", "gdc_rods_slip"])
def test_reference_matrices(config):
    """fcm_fluid_solver.cpp:842-881 with body 0 at the centre (main.cpp's order)."""
    lib().orc_set_threads(os.cpu_count() or 1)
    g = _load(config)
    o, M, nb = _oracle(g)
    o.produce_reference_matrices()
    Minv, N, KTKinv = o.get_reference_matrices()
    assert rel_err(Minv, g["ref_Minv"]) < 1e-9
    assert rel_err(N, g["ref_N"]) < 1e-9
    assert rel_err(KTKinv, g["ref_KTKinv"]) < 1e-13
    o.close()


@pytest.mark.parametrize("config", ["em_tetra", "gdc_rods_slip"])
def test_time_steps(config):
    """main.cpp:222-340: noise from the same stream, forces, GMRES, update (and
    the GDC midstep and div(U) drift in the slip channel)."""
    lib().orc_set_threads(os.cpu_count() or 1)
    g = _load(config)
    o, M, nb = _oracle(g)
    o.set_reference_matrices(g["ref_Minv"], g["ref_N"])
    o.set_bodies(g["x"], g["q"])
    o.set_sequential_noise(True, 5, 0)
    for k in range(len(g["step_x"])):
        st, info = o.step(0, k)
        assert st == 0 and int(g["step_status"][k]) == 0
        x, q = o.get_bodies()
        assert np.abs(x - g["step_x"][k]).max() < 1e-10, k
        assert np.abs(q - g["step_q"][k]).max() < 1e-10, k
        if int(g["cfg"][15]) == 1:
            nu = 1.0 + 0.5 * float(g["cfg"][9]) * info.divU
            assert abs(nu - g["step_nu"][k]) < 1e-9, k
    assert np.abs(x - g["x"]).max() > 1e-3  # the bodies moved
    o.close()


@pytest.mark.parametrize("config", ["mcmc_tetra_soft", "mcmc_tetra_philic"])
def test_metropolis_pair_potential(config):
    """collection_of_rigid_bodies.cpp:666-705 / linked_list.cpp:283-360 in a
    Metropolis build, whose pair terms are the energies of linked_list.cpp:362-497."""
    g = _load(config)
    o, M, nb = _oracle(g)
    o.set_bodies(g["x"], g["q"])
    U = o.calculate_potential()
    assert g["potential"][0] > 0
    assert abs(U - g["potential"][0]) <= 1e-12 * abs(g["potential"][0])
    o.close()
