"""The slip channel on the GPU (slip_channel = 1: SLIP_CHANNEL of the
reference) against the oracle on the same inputs: the mirrored force grid and
the truncated interpolation in the mobility and random velocities (1e-10
relative, with the same injected image-symmetric stress), wall forces and the
potential (1e-12), steps without noise on one trajectory (1e-9), wall-contact
rejection, Metropolis runs on the same decisions, and the Fourier-space
image-symmetric noise against fluctuation-dissipation of the channel mobility."""
import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.capi import FcmError
from timstochrigidbodiessim_b200.fcm import Batch, Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _channel(**kw):
    return configs.rod_channel(24, 64, 32.0, nb=3, seed=2, ngauss=16, **kw)


def _pair(p, ref, x, q, fe=None):
    out = []
    for cls in (Suspension, Oracle):
        s = cls(p, ref)
        s.set_bodies(x, q)
        if fe is not None:
            s.set_external_forces(fe)
        out.append(s)
    return out


def _image_stress(p, rng, scale=0.05):
    """Six real-space stress arrays with the image symmetry of
    fcm_fluid_solver.cpp:186-217 (padded [x][y][pad] layout)."""
    h = p.ny // 2
    out = []
    for c in range(6):  # xx, yy, zz, xy, xz, yz
        a = rng.standard_normal((p.nx, p.ny, p.pad)) * scale
        odd = c in (3, 5)
        for j in range(h + 1, p.ny):
            a[:, j, :] = -a[:, p.ny - j, :] if odd else a[:, p.ny - j, :]
        if odd:
            a[:, 0, :] = 0.0
            a[:, h, :] = 0.0
        out.append(a.ravel())
    return out


def test_slip_mobility_and_random_velocities_match_oracle(gpu):
    p, ref, x, q, fe = _channel()
    g, o = _pair(p, ref, x, q)
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    F = np.random.default_rng(1).standard_normal(3 * p.num_blobs)
    assert rel_err(g.apply_mobility(F), o.apply_mobility(F)) < TOL
    ug = g.get_velocity_field(0)
    for c in range(3):
        assert rel_err(ug[c], o.get_grid(3 + c)) < TOL
    s6 = _image_stress(p, np.random.default_rng(2))
    for s in (g, o):
        s.inject_random_stress(s6)
    assert rel_err(g.calculate_random_blob_velocities(), o.calculate_random_blob_velocities()) < TOL


def test_slip_forces_potential_and_reference_matrices(gpu):
    p, ref, x, q, fe = _channel()
    # push some rods into the walls' spring range
    xx = x.reshape(-1, 3).copy()
    xx[:4, 1] = [1.9, 2.3, 14.0, 13.6]
    g, o = _pair(p, ref, xx.ravel(), q)
    for s in (g, o):
        s.fill_all_blob_pos()
        s.calculate_forces()
    Fg, Fo = g.get_blob_forces(), o.get_blob_forces()
    assert np.abs(Fg - Fo).max() <= 1e-12 * max(1.0, np.abs(Fo).max())
    assert np.abs(Fo[1::3]).max() > 1.0  # the walls push
    Ug, Uo = g.calculate_potential(), o.calculate_potential()
    assert abs(Ug - Uo) <= 1e-12 * max(1.0, abs(Uo))
    for s in (g, o):
        s.produce_reference_matrices()
    for a, b in zip(g.get_reference_matrices()[:2], o.get_reference_matrices()[:2]):
        assert rel_err(a, b) < 1e-9


@pytest.mark.parametrize("algorithm", [2, 1])
def test_slip_steps_match_oracle(gpu, algorithm):
    p, ref, x, q, fe = _channel(algorithm=algorithm, gmres_tol=1e-12, noise=0)
    fe = fe.copy()
    fe[1::6] = 0.3  # also drive the rods towards the upper wall
    g, o = _pair(p, ref, x, q, fe)
    o.produce_reference_matrices()
    Minv, N, _ = o.get_reference_matrices()
    g.set_reference_matrices(Minv, N)
    for step in range(3):
        sg, ig = g.step(5, step)
        so, io = o.step(5, step)
        assert sg == so == 0
    xg, qg = g.get_bodies()
    xo, qo = o.get_bodies()
    assert np.abs(xg - xo).max() < 1e-9 and np.abs(qg - qo).max() < 1e-9
    # graph steps are not taken in a slip channel: async steps stay host-driven
    g.step_async(5, 3)
    assert g.step_wait()[0] == 0


def test_slip_wall_contact_rejected(gpu):
    p, ref, x, q, fe = _channel(noise=0)
    g, o = _pair(p, ref, x, q)
    U = np.zeros(6 * p.num_bodies)
    U[1] = 20.0 / p.dt  # the first rod through the upper wall
    for s in (g, o):
        s.fill_all_blob_pos()
    assert g.end_of_step_update(U, 1.0) and o.end_of_step_update(U, 1.0) == 1
    g.reset_to_start_of_step()
    assert np.array_equal(g.get_bodies()[0], x)
    assert not g.end_of_step_update(np.zeros_like(U), 1.0)


def test_slip_mcmc_matches_oracle(gpu):
    p, ref, x, q, fe = _channel()
    p = p.copy(potential=0)
    g, o = _pair(p, ref, x, q)
    sg = g.mcmc_run(3, 120)
    _, so = o.mcmc_run(3, 120)
    assert (sg.steps, sg.attempts) == (so.steps, so.attempts)
    assert abs(sg.potential - so.potential) <= 1e-10 * max(1.0, abs(so.potential))
    xg, qg = g.get_bodies()
    xo, qo = o.get_bodies()
    assert np.max(np.abs(xg - xo)) <= 1e-12 and np.max(np.abs(qg - qo)) <= 1e-12


def test_slip_fourier_noise_fluctuation_dissipation(gpu):
    """The Fourier-space draw of the image-symmetric stress: <V V^T> of random
    blob velocities equals (2 kT/dt) sym(M) of the channel within sampling error,
    with blobs near both walls and mid-channel."""
    N, dx = 32, 0.4
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=16, dx=dx, num_bodies=3, blobs_per_body=1, ncells=3, kT=1.0,
                           dt=0.01, slip_channel=1)
    Y = np.array([[3.1, 1.3, 5.3], [6.6, 3.4, 8.9], [9.7, 5.9, 11.1]]).ravel()
    s = Suspension(p, [0, 0, 0])
    s.set_up_gaussians(Y)
    n = 9
    Mm = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        Mm[:, j] = s.apply_mobility(e)
    T = (2.0 * p.kT / p.dt) * 0.5 * (Mm + Mm.T)
    S = 6000
    Vs = np.zeros((S, n))
    for i in range(S):
        s.produce_random_velocity_field(77, i)
        Vs[i] = s.calculate_random_blob_velocities()
    C = Vs.T @ Vs / S
    expected = np.sqrt(np.sum(np.outer(np.diag(T), np.diag(T)) + T ** 2) / S)
    assert np.linalg.norm(C - T) < 3.0 * expected


def test_slip_shear_flow_and_refusals(gpu):
    p, ref, x, q, fe = _channel()
    g, o = _pair(p, ref, x, q)
    for s in (g, o):
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        s.produce_shear_velocity_field(1.0, 1.0)
    assert rel_err(g.calculate_shear_blob_velocities(), o.calculate_shear_blob_velocities()) < TOL
    with pytest.raises(FcmError):
        g.set_up_dipole_distribution(T=np.zeros(3 * p.num_blobs))
    with pytest.raises(FcmError):
        Batch([(p, ref)])


def test_slip_fp32_tile_variants_match_oracle(gpu):
    """The FP32 tile kernels in the channel, where the force grid is mirrored and
    the interpolation reads nothing at or above the upper wall (ny/2): each FP32
    spread and interpolation variant, the tensor-core ones included, within 1e-5
    of the oracle's FP64 channel mobility."""
    p, ref, x, q, fe = _channel()
    p32 = p.copy(precision=1)
    g = Suspension(p32, ref)
    o = Oracle(p, ref)
    for s in (g, o):
        s.set_bodies(x, q)
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    F = np.random.default_rng(5).standard_normal(3 * p.num_blobs)
    Vo = o.apply_mobility(F)
    for sp in (0, 4, 5):
        for ip in (1, 3):
            v = g.get_variants()
            v[2], v[5] = sp, ip
            g.set_variants(v)
            g.spread(F, 1)
            g.stokes_solve(1)
            assert rel_err(g.interp(1), Vo) < 1e-5, (sp, ip)
