"""The slip channel (SLIP_CHANNEL, the reference's default geometry) in the
oracle: the image system in y (fcm_fluid_solver.cpp:186-217, :387-389,
:602-632), the wall forces and potential (collection_of_rigid_bodies.cpp:640-662,
:679-700) and the wall-contact rejection (:207-239, :611-617, :780-786).

Pinned by: fluctuation-dissipation of the image-symmetric stress against the
slip-channel mobility; the mirror symmetry of the flow (u_y vanishes on the wall
rows up to the reference's one-sided Nyquist wavenumber); the free-slip wall's
effect on a blob (perpendicular mobility lowered, parallel raised); the wall
spring and its energy in closed form; rejection of steps that touch a wall."""
import math

import numpy as np
import pytest

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.params import FcmParams, rod_reference_positions


def _blobs(n, N=16, dx=0.5, W=12, **kw):
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=W, dx=dx, num_bodies=n, blobs_per_body=1, ncells=3,
                           kT=1.0, dt=0.01, slip_channel=1, **kw)
    return Oracle(p, [0, 0, 0]), p


def _mobility(o, n):
    Mm = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        Mm[:, j] = o.apply_mobility(e)
    return Mm


def test_slip_fluctuation_dissipation():
    """<V V^T> of the random velocities equals (2 kT/dt) sym(M) of the channel
    (the truncated Gaussians leave M non-symmetric by about 1%)."""
    o, p = _blobs(2)
    o.set_up_gaussians(np.array([2.1, 1.2, 4.3, 5.6, 2.9, 6.9]))
    Mm = _mobility(o, 6)
    assert np.abs(Mm - Mm.T).max() < 0.03 * np.abs(Mm).max()
    T = (2.0 * p.kT / p.dt) * 0.5 * (Mm + Mm.T)
    S = 1500
    Vs = np.zeros((S, 6))
    for i in range(S):
        o.produce_random_velocity_field(4321, i)
        Vs[i] = o.calculate_random_blob_velocities()
    C = Vs.T @ Vs / S
    expected = np.sqrt(np.sum(np.outer(np.diag(T), np.diag(T)) + T ** 2) / S)
    assert np.linalg.norm(C - T) < 3.0 * expected


def test_slip_flow_mirror_symmetric():
    o, p = _blobs(2)
    o.set_up_gaussians(np.array([2.1, 1.2, 4.3, 5.6, 2.9, 6.9]))
    o.set_up_force_distribution(np.random.default_rng(1).standard_normal(6))
    f = [o.get_grid(c).reshape(p.nx, p.ny, p.pad)[:, :, :p.nz] for c in range(3)]
    h = p.ny // 2
    assert np.all(f[1][:, 0, :] == 0) and np.all(f[1][:, h, :] == 0)
    for j in range(h + 1, p.ny):
        assert np.array_equal(f[0][:, j, :], f[0][:, p.ny - j, :])
        assert np.array_equal(f[1][:, j, :], -f[1][:, p.ny - j, :])
    o.produce_deterministic_velocity_field()
    u = [o.get_grid(3 + c).reshape(p.nx, p.ny, p.pad)[:, :, :p.nz] for c in range(3)]
    # u_y is odd about both walls; only the Nyquist row's one-sided wavenumber
    # (fcm_fluid_solver.cpp:99-111) breaks the symmetry, at the 1e-4 level
    top = np.abs(u[1]).max()
    assert np.abs(u[1][:, 0, :]).max() < 1e-3 * top and np.abs(u[1][:, h, :]).max() < 1e-3 * top
    assert np.abs(u[0] - u[0][:, (p.ny - np.arange(p.ny)) % p.ny, :]).max() < 1e-3 * np.abs(u[0]).max()


def test_free_slip_wall_mobility():
    """Near a free-slip wall a blob moves more easily along it and less easily
    towards it than in the middle of the channel."""
    o, p = _blobs(1, N=32, dx=0.5, W=16)
    H = 0.5 * p.ny * p.dx  # channel height 8
    mob = {}
    for y in (2.5, 0.5 * H):
        o.set_up_gaussians(np.array([4.1, y, 4.3]))
        mob[y] = np.diag(_mobility(o, 3))
    near, mid = mob[2.5], mob[0.5 * H]
    assert near[0] > mid[0] and near[2] > mid[2]  # parallel
    assert near[1] < mid[1]                        # perpendicular


def test_wall_forces_and_potential():
    o, p = _blobs(3, N=32, potential=3)  # cut off at 2.2a: the blobs below do not interact
    H = 0.5 * p.ny * p.dx
    L = 2.2 * p.blob_radius
    ys = np.array([1.0, 0.5 * H, H - 0.7])
    Y = np.column_stack([[1.0, 4.0, 7.0], ys, [2.0, 5.0, 6.5]]).ravel()
    o.set_bodies(Y, np.tile([1.0, 0, 0, 0], 3))
    o.fill_all_blob_pos()
    o.calculate_forces()
    F = o.get_blob_forces().reshape(3, 3)
    K = (40.0 * p.kT / p.blob_radius) / L
    assert F[0, 1] == pytest.approx(K * (L - ys[0]), rel=1e-15)
    assert F[1, 1] == 0.0
    assert F[2, 1] == pytest.approx(-K * (L - H + ys[2]), rel=1e-15)
    U = o.calculate_potential()
    Ke = 40.0 * p.kT / (L * p.blob_radius)
    assert U == pytest.approx(0.5 * Ke * ((L - ys[0]) ** 2 + (L - H + ys[2]) ** 2), rel=1e-14)


def test_steps_rejected_on_wall_contact():
    """A rod pushed through the upper wall: the end-of-step update reports the
    contact and the step is undone (main.cpp:316-328); an MCMC run keeps every
    blob strictly inside the channel."""
    ref = rod_reference_positions(3, 2.2)
    p = FcmParams.defaults(nx=16, ny=16, nz=16, ngauss=12, dx=0.5, num_bodies=1, blobs_per_body=3, ncells=3,
                           kT=1.0, dt=0.01, slip_channel=1, noise=0)
    o = Oracle(p, ref)
    x0 = np.array([4.0, 3.5, 4.0])
    q0 = np.array([1.0, 0.0, 0.0, 0.0])
    o.set_bodies(x0, q0)
    H = 0.5 * p.ny * p.dx
    U = np.array([0.0, (H - 3.5 + 0.1) / p.dt, 0.0, 0.0, 0.0, 0.0])
    assert o.end_of_step_update(U, 1.0) == 1
    o.reset_to_start_of_step()
    assert np.array_equal(o.get_bodies()[0], x0)
    assert o.end_of_step_update(np.zeros(6), 1.0) == 0
    q2 = FcmParams.defaults(nx=16, ny=16, nz=16, ngauss=12, dx=0.5, num_bodies=4, blobs_per_body=3, ncells=3,
                            kT=1.0, dt=0.5, slip_channel=1, potential=0)
    o2 = Oracle(q2, ref)
    xs = np.array([[2.0, 2.0, 2.0], [6.0, 2.0, 6.0], [2.0, 2.0, 6.0], [6.0, 2.0, 2.0]]).ravel()
    o2.set_bodies(xs, np.tile([1.0, 0, 0, 0], 4))
    st, state = o2.mcmc_run(5, 300)
    assert st == 0
    o2.fill_all_blob_pos()
    Yb = o2.get_all_blob_pos().reshape(-1, 3)
    assert np.all(Yb[:, 1] > 0) and np.all(Yb[:, 1] < H)
