"""Fluctuation-dissipation of the Philox noise path, mixed precision accuracy
and error statuses, on the GPU."""
import numpy as np
import pytest

from tests.conftest import rel_err
from timstochrigidbodiessim_b200 import configs
from timstochrigidbodiessim_b200.fcm import Suspension
from timstochrigidbodiessim_b200.params import FcmParams, rod_reference_positions

pytestmark = pytest.mark.gpu


def fdt_setup(precision=0):
    # three free blobs, well-resolved Gaussians (sigma/dx = 1.41)
    N, dx = 32, 0.4
    p = FcmParams.defaults(nx=N, ny=N, nz=N, ngauss=16, dx=dx, num_bodies=3, blobs_per_body=1, ncells=3,
                           kT=1.0, dt=0.01, precision=precision)
    Y = np.array([[3.1, 4.2, 5.3], [6.6, 7.1, 8.9], [9.7, 2.2, 11.1]]).ravel()
    return p, Y


def mobility_matrix(s, n):
    Mm = np.zeros((n, n))
    for j in range(n):
        e = np.zeros(n)
        e[j] = 1.0
        Mm[:, j] = s.apply_mobility(e)
    return 0.5 * (Mm + Mm.T)


@pytest.mark.parametrize("precision", [0, 1])
def test_fluctuation_dissipation(gpu, precision):
    """<V V^T> of the random blob velocities equals (2 kT/dt) M within the
    sampling error of S samples (E|C - T|_F^2 = sum_ij (T_ii T_jj + T_ij^2)/S)."""
    p, Y = fdt_setup(precision)
    s = Suspension(p, [0, 0, 0])
    s.set_up_gaussians(Y)
    n = 9
    T = (2.0 * p.kT / p.dt) * mobility_matrix(s, n)
    S = 6000
    Vs = np.zeros((S, n))
    for i in range(S):
        s.produce_random_velocity_field(1234, i)
        Vs[i] = s.calculate_random_blob_velocities()
    C = Vs.T @ Vs / S
    mean = Vs.mean(0)
    se_mean = np.sqrt(np.diag(T) / S)
    assert np.all(np.abs(mean) < 5 * se_mean)
    expected = np.sqrt(np.sum(np.outer(np.diag(T), np.diag(T)) + T ** 2) / S)
    err = np.linalg.norm(C - T)
    assert err < 3.0 * expected, (err / np.linalg.norm(T), expected / np.linalg.norm(T))
    # samples with different counters are independent, same counter reproduces
    s.produce_random_velocity_field(1234, 7)
    assert np.array_equal(s.calculate_random_blob_velocities(), Vs[7])


def test_noise_is_hermitian_consistent(gpu):
    """The Fourier-space draw yields a real field whose mean is zero: check the
    field itself via the padded velocity grids."""
    p, Y = fdt_setup()
    s = Suspension(p, [0, 0, 0])
    s.produce_random_velocity_field(99, 3)
    ux, uy, uz = s.get_velocity_field(1)
    pad = p.pad
    for u in (ux, uy, uz):
        u = u.reshape(p.nx, p.ny, pad)[:, :, : p.nz]
        assert abs(u.mean()) < 1e-12 * np.abs(u).max()
        assert np.abs(u).max() > 0


def test_mixed_precision_mobility_error(gpu):
    p, ref, x, q, fe = configs.workload("rods32_L64_g64")
    p64 = p.copy(precision=0)
    p32 = p.copy(precision=1)
    a, b = Suspension(p64, ref), Suspension(p32, ref)
    for s in (a, b):
        s.set_bodies(x, q)
        s.fill_all_blob_pos()
        s.set_up_gaussians()
    F = np.random.default_rng(2).standard_normal(3 * p.num_blobs)
    err = rel_err(b.apply_mobility(F), a.apply_mobility(F))
    assert err < 2e-6, err


def test_mixed_precision_solve_matches_fp64(gpu):
    """FP32 grid work inside FP64 iterative refinement reaches the FP64
    solution to <= 1e-6 relative blob/body velocity error."""
    p, ref, x, q, fe = configs.workload("rods32_L64_g64", gmres_tol=1e-10)
    sols = []
    for prec in (0, 1):
        s = Suspension(p.copy(precision=prec), ref)
        s.set_bodies(x, q)
        s.set_external_forces(fe)
        s.produce_reference_matrices()
        s.fill_all_blob_pos()
        s.set_up_gaussians()
        s.calculate_forces()
        s.assemble_RHS()
        st, soln, it, rel = s.invert_saddle_point_system()
        assert st == 0, (prec, it, rel)
        sols.append(soln)
    Nb = p.num_blobs
    assert rel_err(sols[1][3 * Nb:], sols[0][3 * Nb:]) < 1e-6
    assert rel_err(sols[1][:3 * Nb], sols[0][:3 * Nb]) < 1e-6


def test_error_statuses(gpu):
    from timstochrigidbodiessim_b200 import capi
    p, ref, x, q, fe = configs.workload("rods32_L64_g64")
    s = Suspension(p, ref)
    # interpolation before set_up_gaussians -> FCM_ERR_STATE
    with pytest.raises(capi.FcmError) as e:
        s.calculate_deterministic_blob_velocities()
    assert e.value.status == 4
    s.set_bodies(x, q)
    s.fill_all_blob_pos()
    s.set_up_gaussians()
    # non-finite right-hand side -> FCM_ERR_NONFINITE, context still usable
    bad = np.zeros(p.system_size)
    bad[5] = np.nan
    s.set_RHS(bad)
    with pytest.raises(capi.FcmError) as e:
        s.invert_saddle_point_system()
    assert e.value.status == 6
    # max_iter 1 at a tiny tolerance -> FCM_ERR_NOT_CONVERGED with the iterate returned
    s2 = Suspension(p.copy(gmres_max_iter=1, gmres_tol=1e-15), ref)
    s2.set_bodies(x, q)
    s2.set_external_forces(fe)
    s2.fill_all_blob_pos()
    s2.set_up_gaussians()
    s2.calculate_forces()
    s2.assemble_RHS()
    st, soln, it, rel = s2.invert_saddle_point_system()
    assert st == 5 and it == 1 and np.all(np.isfinite(soln)) and np.abs(soln).max() > 0
    # the first context still works after the failure
    F = np.ones(3 * p.num_blobs)
    assert np.all(np.isfinite(s.apply_mobility(F)))


def test_overlap_rejects_step(gpu):
    """SKIP_ON_OVERLAP: a step that ends with overlapping bodies is rejected and
    the bodies are restored (main.cpp:316-328).  The two rods start 1.5a apart
    and the step is far too short to separate them."""
    nb = 2
    ref = np.array(rod_reference_positions(nb, 2.2))
    p = FcmParams.defaults(nx=32, ny=32, nz=32, ngauss=8, dx=0.5, num_bodies=2, blobs_per_body=nb, ncells=3,
                           potential=3, noise=0, skip_on_overlap=1, dt=1e-6, gmres_tol=1e-8)
    s = Suspension(p, ref)
    x = np.array([8.0, 8.0, 8.0, 8.0, 8.0, 9.5])
    qq = np.array([1.0, 0, 0, 0, 1.0, 0, 0, 0])
    s.set_bodies(x, qq)
    s.produce_reference_matrices()
    st, info = s.step(0, 0)
    assert st == 7 and info.overlap == 1
    x2, q2 = s.get_bodies()
    assert np.array_equal(x2, x) and np.array_equal(q2, qq)
    # without the check the same step is accepted
    s2 = Suspension(p.copy(skip_on_overlap=0), ref)
    s2.set_bodies(x, qq)
    s2.produce_reference_matrices()
    st2, info2 = s2.step(0, 0)
    assert st2 == 0 and info2.overlap == 0
