"""Force dipoles on the GPU (fcm_set_up_dipole_distribution,
fcm_calculate_deterministic_blob_rotations; no reference counterpart) against
the oracle's restatement on the same inputs: blob velocities, rotation rates
and strain rates within 1e-10 relative (norm-wise), with forces, torques and
stresslets together, on ragged tile lists (a dense cluster and blobs on the
periodic boundary)."""
import math

import numpy as np
import pytest

from tests.conftest import rel_err
from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _params(n, N=96, L=32.0, W=24):
    return FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=W, dx=L / N, blob_radius=1.0, viscosity=1.0, num_bodies=n,
                              blobs_per_body=1, ncells=3)


def _inputs(n, L, seed):
    rng = np.random.default_rng(seed)
    Y = rng.uniform(0.0, L, (n, 3))
    Y[:40] = rng.uniform(10.0, 12.5, (40, 3))  # many blobs in one tile
    Y[40] = (0.0, 0.0, 0.0)
    Y[41] = (L - 1e-9, 1e-9, L / 2)
    F = rng.standard_normal(3 * n)
    T = rng.standard_normal(3 * n)
    S = rng.standard_normal((n, 3, 3))
    S = 0.5 * (S + S.transpose(0, 2, 1))
    return Y.ravel(), F, T, S.ravel()


@pytest.mark.parametrize("parts", [("F", "T", "S"), ("T",), ("S",)])
def test_dipoles_match_oracle(gpu, parts):
    n, L = 300, 32.0
    Y, F, T, S = _inputs(n, L, 5)
    kw = {k: v for k, v in (("F", F), ("T", T), ("S", S)) if k in parts}
    res = []
    for s in (Suspension(_params(n), [0, 0, 0]), Oracle(_params(n), [0, 0, 0])):
        s.set_up_gaussians(Y)
        s.set_up_dipole_distribution(**kw)
        s.produce_deterministic_velocity_field()
        V = s.calculate_deterministic_blob_velocities()
        Om, E = s.calculate_deterministic_blob_rotations()
        res.append((V, Om, E))
    for a, b in zip(res[0], res[1]):
        assert rel_err(a, b) < TOL


def test_rotational_self_mobility_gpu(gpu):
    L = 32.0
    s = Suspension(_params(1), [0, 0, 0])
    s.set_up_gaussians(np.array([L / 2 + 0.3, L / 2 - 0.2, L / 2 + 0.1]))
    T = np.array([0.3, -0.5, 1.0])
    s.set_up_dipole_distribution(T=T)
    s.produce_deterministic_velocity_field()
    Om, E = s.calculate_deterministic_blob_rotations()
    expect = (1.0 - 4.0 * math.pi / 3.0 / L ** 3) / (8.0 * math.pi)
    assert np.allclose(Om, expect * T, rtol=2e-6, atol=1e-12)
