"""Fluctuation-dissipation of the oracle's real-space noise path (the
reference's fcm_fluid_solver.cpp:167-361 with polar-method normals)."""
import numpy as np

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200.params import FcmParams


def test_oracle_fluctuation_dissipation():
    N, dx = 16, 0.5
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=12, dx=dx, num_bodies=2, blobs_per_body=1, ncells=3,
                           kT=1.0, dt=0.01)
    Y = np.array([[2.1, 3.2, 4.3], [5.6, 1.1, 6.9]]).ravel()
    o = Oracle(p, [0, 0, 0])
    o.set_up_gaussians(Y)
    n = 6
    Mm = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        Mm[:, j] = o.apply_mobility(e)
    T = (2.0 * p.kT / p.dt) * 0.5 * (Mm + Mm.T)
    S = 600
    Vs = np.zeros((S, n))
    for i in range(S):
        o.produce_random_velocity_field(4321, i)
        Vs[i] = o.calculate_random_blob_velocities()
    C = Vs.T @ Vs / S
    expected = np.sqrt(np.sum(np.outer(np.diag(T), np.diag(T)) + T ** 2) / S)
    assert np.linalg.norm(C - T) < 3.0 * expected
