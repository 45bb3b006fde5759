"""Force dipoles in the oracle (no reference code; the FCM dipole terms of
Lomholt & Maxey 2003).  Pinned by known answers: the dipole envelope
sigma_D = a/(6 sqrt(pi))^(1/3) makes the rotational self-mobility of an isolated
blob exactly 1/(8 pi eta a^3); in a periodic cube of side L the mean-rotation
correction lowers it to (1 - (4 pi/3) a^3/L^3) / (8 pi eta a^3).  A single blob
has no translation-rotation coupling, and the mobility is symmetric (Lorentz
reciprocity): F.V(T) = T.Omega(F) and S1:E(S2) = S2:E(S1)."""
import math

import numpy as np
import pytest

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.params import FcmParams


def _oracle(n, N=96, L=32.0, W=24):
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=W, dx=L / N, blob_radius=1.0, viscosity=1.0, num_bodies=n,
                           blobs_per_body=1, ncells=3)
    return Oracle(p, [0, 0, 0]), p


def _solve(o, F=None, T=None, S=None):
    o.set_up_dipole_distribution(F, T, S)
    o.produce_deterministic_velocity_field()
    V = o.calculate_deterministic_blob_velocities()
    Om, E = o.calculate_deterministic_blob_rotations()
    return V, Om, E


@pytest.mark.parametrize("L,N", [(32.0, 96), (42.0, 126)])
def test_rotational_self_mobility(L, N):
    if N % 2:
        N += 1
    o, p = _oracle(1, N=N, L=L)
    Y = np.array([L / 2 + 0.3, L / 2 - 0.2, L / 2 + 0.1])
    o.set_up_gaussians(Y)
    T = np.array([0.3, -0.5, 1.0])
    V, Om, E = _solve(o, T=T)
    expect = (1.0 - 4.0 * math.pi / 3.0 / L ** 3) / (8.0 * math.pi)
    assert np.allclose(Om, expect * T, rtol=2e-6, atol=1e-12)
    # discretisation leaves couplings of order 1e-9 (|Omega| ~ 0.04)
    assert np.abs(V).max() < 1e-9 and np.abs(E).max() < 1e-8
    F = np.array([1.0, 0.2, -0.4])
    V, Om, E = _solve(o, F=F)
    assert np.abs(Om).max() < 1e-9


def test_reciprocity_two_blobs():
    o, p = _oracle(2)
    Y = np.array([14.1, 16.3, 15.2, 17.0, 15.1, 16.9])
    o.set_up_gaussians(Y)
    rng = np.random.default_rng(4)
    F = rng.standard_normal(6)
    T = rng.standard_normal(6)
    S1 = rng.standard_normal((2, 3, 3))
    S2 = rng.standard_normal((2, 3, 3))
    S1 = 0.5 * (S1 + S1.transpose(0, 2, 1))
    S2 = 0.5 * (S2 + S2.transpose(0, 2, 1))
    VT, _, _ = _solve(o, T=T)
    _, OmF, _ = _solve(o, F=F)
    assert abs(F @ VT - T @ OmF) < 1e-10 * (abs(F @ VT) + 1e-3)
    _, _, E2 = _solve(o, S=S2.ravel())
    _, _, E1 = _solve(o, S=S1.ravel())
    a, b = S1.ravel() @ E2, S2.ravel() @ E1
    assert abs(a - b) < 1e-9 * (abs(a) + 1e-3)
