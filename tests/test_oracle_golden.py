"""The CPU oracle against the golden fixtures of tests/golden/make_golden.py
(an independent numpy restatement of the reference's formulas)."""
import numpy as np

from tests.conftest import rel_err
from tests.oracle_lib import Oracle, fft_transform, fft_inverse_transform
from timstochrigidbodiessim_b200.params import FcmParams

TOL = 1e-12


def test_fft_forward_and_nonhermitian_inverse(golden):
    for tag, shape in (("a", (6, 8, 10)), ("b", (8, 6, 9))):
        fwd = fft_transform(*shape, golden["fft_%s_in" % tag])
        assert rel_err(fwd, golden["fft_%s_fwd" % tag]) < TOL
        inv = fft_inverse_transform(*shape, golden["fft_%s_spec" % tag])
        nz = shape[2]
        pad = 2 * (nz // 2 + 1)
        got = inv.reshape(shape[0], shape[1], pad)[:, :, :nz]
        ref = golden["fft_%s_inv" % tag].reshape(shape[0], shape[1], pad)[:, :, :nz]
        assert rel_err(got, ref) < TOL


def _mob_params(N, dx, a, eta, W, nblobs):
    return FcmParams.defaults(nx=int(N[0]), ny=int(N[1]), nz=int(N[2]), ngauss=int(W), dx=float(dx), blob_radius=float(a),
                              viscosity=float(eta), num_bodies=nblobs, blobs_per_body=1, ncells=3)


def test_mobility_golden(golden):
    N = golden["mobility_N"]
    dx, a, eta, W = golden["mobility_params"]
    Y = golden["mobility_Y"]
    o = Oracle(_mob_params(N, dx, a, eta, W, len(Y) // 3), [0, 0, 0])
    o.set_up_gaussians(Y)
    ind, w = o.get_gaussians()
    assert np.array_equal(ind.ravel(), golden["mobility_ind"].astype(np.int32))
    assert rel_err(w.ravel(), golden["mobility_w"]) < TOL
    V = o.apply_mobility(golden["mobility_F"])
    assert rel_err(V, golden["mobility_V"]) < TOL


def test_mobility_golden_noncubic_odd(golden):
    N = golden["mobility2_N"]
    dx, a, eta, W = golden["mobility2_params"]
    Y = golden["mobility2_Y"]
    o = Oracle(_mob_params(N, dx, a, eta, W, len(Y) // 3), [0, 0, 0])
    o.set_up_gaussians(Y)
    V = o.apply_mobility(golden["mobility2_F"])
    assert rel_err(V, golden["mobility2_V"]) < TOL


def test_random_field_injected_golden(golden):
    N = golden["random_N"]
    Y = golden["random_Y"]
    o = Oracle(_mob_params(N, 1.0, 1.0, 1.0, 8, len(Y) // 3), [0, 0, 0])
    P = int(N[0] * N[1] * (2 * (N[2] // 2 + 1)))
    s6 = golden["random_s6"].reshape(6, P)
    o.inject_random_stress(s6)
    o.set_up_gaussians(Y)
    V = o.calculate_random_blob_velocities()
    assert rel_err(V, golden["random_V"]) < TOL


def test_bodies_golden(golden):
    L = float(golden["bodies_L"][0])
    ref = golden["bodies_ref"]
    p = FcmParams.defaults(nx=20, ny=20, nz=20, ngauss=4, dx=L / 20, num_bodies=5, blobs_per_body=3, ncells=3)
    o = Oracle(p, ref)
    o.set_bodies(golden["bodies_x"], golden["bodies_q"])
    o.fill_all_blob_pos()
    assert rel_err(o.get_all_blob_pos(), golden["bodies_Y"]) < TOL
    assert rel_err(o.multiply_by_K_at_midstep(golden["bodies_U"]), golden["bodies_KU"]) < TOL
    assert rel_err(o.multiply_by_KT_at_midstep(golden["bodies_lam"]), golden["bodies_KTl"]) < TOL
    p2 = p.copy(dt=0.37)
    o2 = Oracle(p2, ref)
    o2.set_bodies(golden["bodies_x"], golden["bodies_q"])
    o2.end_of_step_update(golden["bodies_U"], 1.0)
    x2, q2 = o2.get_bodies()
    assert rel_err(x2, golden["bodies_x2"]) < TOL
    assert rel_err(q2, golden["bodies_q2"]) < TOL


def test_cells_golden(golden):
    L = float(golden["cells_L"][0])
    Nc = int(golden["cells_Nc"][0])
    nb = int(golden["cells_nb"][0])
    Y = golden["cells_Y"]
    p = FcmParams.defaults(nx=12, ny=12, nz=12, ngauss=4, dx=L / 12, num_bodies=len(Y) // 3 // nb,
                           blobs_per_body=nb, ncells=Nc, potential=0)
    o = Oracle(p, [0, 0, 0] * nb)
    o.set_all_blob_pos(Y)
    o.list_populate()
    assert np.array_equal(o.list_get_cells(), golden["cells_ids"])
    assert np.array_equal(o.list_get_pairs(), golden["cells_pairs"])
    F = o.apply_barrier_forces()
    assert rel_err(F, golden["cells_F"]) < TOL
