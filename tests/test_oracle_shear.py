"""Shear forcing in the oracle (fcm_fluid_solver.cpp:703-842, :489-550;
gmres_solver.cpp:62-64; main.cpp:270-272, :371-433).  Pinned by known answers:
the body force fx = S kT sin(k y)/a with k = 2 pi w / L_y (w an integer below
Ny/2) is one Fourier mode, so the periodic Stokes flow is exactly
u_x = S kT sin(k y) / (a eta k^2), u_y = u_z = 0, on the grid; a Gaussian
envelope of width sigma = a/sqrt(pi) sees sin(k Y) exp(-k^2 sigma^2 / 2) of it."""
import math

import numpy as np
import pytest

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.params import FcmParams, rod_reference_positions


def _oracle(M=3, nb=1, N=32, L=32.0, W=20, **kw):
    ref = [0, 0, 0] if nb == 1 else rod_reference_positions(nb, 2.2)
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=W, dx=L / N, blob_radius=1.0, viscosity=1.3, kT=0.7,
                           num_bodies=M, blobs_per_body=nb, ncells=4, **kw)
    return Oracle(p, ref), p


@pytest.mark.parametrize("scale,w", [(1.0, 1.0), (2.5, 3.0)])
def test_shear_flow_known_answer(scale, w):
    # dx = 0.3 a resolves the envelope (sigma/dx = 1.88, as the reference's DX);
    # 28 points reach 7.4 sigma on each side
    o, p = _oracle(N=64, L=19.2, W=28)
    o.produce_shear_velocity_field(scale, w)
    N, L = p.nx, p.nx * p.dx
    k = 2 * math.pi * w / L
    amp = scale * p.kT / (p.blob_radius * p.viscosity * k * k)
    y = np.arange(N) * p.dx
    # the profile with no blob forces is the imposed flow itself
    prof = o.fluid_x_velocity_in_y(np.zeros(3 * o.Nb))
    assert np.abs(prof - amp * np.sin(k * y)).max() < 1e-12 * amp
    Y = np.array([[10.3, 4.1, 7.7], [12.0, 13.9, 1.2], [3.3, 18.5, 19.1]])
    o.set_up_gaussians(Y.ravel())
    Vs = o.calculate_shear_blob_velocities().reshape(-1, 3)
    sigma = p.blob_radius / math.sqrt(math.pi)
    expect = amp * math.exp(-0.5 * (k * sigma) ** 2) * np.sin(k * Y[:, 1])
    assert np.abs(Vs[:, 0] - expect).max() < 1e-9 * amp
    assert np.abs(Vs[:, 1:]).max() < 1e-12 * amp


def test_shear_enters_rhs_and_leaves_V():
    o, p = _oracle()
    Y = np.array([10.3, 4.1, 7.7, 20.0, 13.9, 1.2, 3.3, 29.5, 30.1])
    o.set_up_gaussians(Y)
    F = np.linspace(-1.0, 1.0, 9)
    V = o.apply_mobility(F)
    o.set_blob_forces(np.zeros(9))
    o.assemble_RHS()
    rhs0 = o.get_RHS()
    o.produce_shear_velocity_field(1.0, 1.0)
    Vs = o.calculate_shear_blob_velocities()
    assert np.array_equal(o.get_V(), V)  # the interpolation of u_shear keeps fcm.V
    o.assemble_RHS()
    rhs1 = o.get_RHS()
    assert np.array_equal(rhs1[:9], -V - Vs)
    assert np.array_equal(rhs1[9:], rhs0[9:])


def test_gdc_rod_follows_shear_flow():
    """A GDC step without noise or forces moves an isolated rod lying along x
    with the imposed flow: every blob sees the same Vshear, so lambda = 0 and the
    rod translates at exactly that velocity without turning.  The EM step never
    interpolates u_shear (main.cpp:270 is in the GDC branch), so its Vshear stays
    zero and the rod stays at rest."""
    for alg in (1, 2):
        o, p = _oracle(M=1, nb=3, N=64, L=19.2, W=28, algorithm=alg, noise=0, gmres_tol=1e-12,
                       gmres_max_iter=100, dt=0.05)
        o.produce_reference_matrices()
        o.produce_shear_velocity_field(1.0, 1.0)
        x0 = np.array([9.7, 3.1, 10.2])
        q0 = np.array([1.0, 0.0, 0.0, 0.0])
        o.set_bodies(x0, q0)
        st, info = o.step(1, 0)
        assert st == 0
        x, q = o.get_bodies()
        if alg == 2:
            assert np.array_equal(x, x0) and np.array_equal(q, q0)
            continue
        o.fill_all_blob_pos(1)
        o.set_up_gaussians()
        Vs = o.calculate_shear_blob_velocities().reshape(-1, 3)
        assert np.ptp(Vs[:, 0]) < 1e-10 * abs(Vs[0, 0]) and abs(Vs[0, 0]) > 1e-3
        dx = (x - x0) / p.dt
        assert abs(dx[0] - Vs[0, 0]) < 1e-9 * abs(Vs[0, 0])
        assert abs(dx[1]) < 1e-12 and abs(dx[2]) < 1e-12
        assert np.abs(q - q0).max() < 1e-12
