"""The GPU path against numbers computed by the reference itself.

tests/golden/ref_<config>.npz hold what the reference's own classes computed
(compiled unchanged from its sources with the project-written stand-ins of
oracle/ref_shim; tests/golden/make_ref_golden.py).  Here the library, given the
same parameters and bodies, must give: blob positions, cell ids and Gaussian
stencil indices bit for bit; steric forces 1e-12; M F, K, K^T, P^-1 and the
saddle-point product 1e-10; its own probed reference matrices 1e-9 -- on the
tetrahedra in a periodic box (Euler-Maruyama build) and on the reference's
22-blob rods in its default slip channel.  Time steps are tied to the reference
through the oracle (tests/test_oracle_vs_reference.py and the GPU-oracle step
tests), since the library draws its noise in Fourier space.
"""
import os

import numpy as np
import pytest

from tests.conftest import rel_err
from tests.test_oracle_vs_reference import _load, _params
from timstochrigidbodiessim_b200.fcm import Suspension

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.mark.parametrize("config", ["em_tetra", "gdc_rods_slip"])
def test_gpu_against_reference_numbers(gpu, config):
    g = _load(config)
    c = g["cfg"]
    M, nb = int(c[0]), int(c[1])
    s = Suspension(_params(c, M, nb), g["blob_ref_pos"])
    s.produce_reference_matrices()  # body 0 at the centre, as the reference produced them
    Minv, N, KTKinv = s.get_reference_matrices()
    n3 = 3 * nb
    assert rel_err(np.asarray(Minv).reshape(n3, n3), g["ref_Minv"]) < 1e-9
    assert rel_err(np.asarray(N).reshape(6, 6), g["ref_N"]) < 1e-9
    s.set_reference_matrices(g["ref_Minv"], g["ref_N"])
    s.set_bodies(g["x"], g["q"])
    s.fill_all_blob_pos()
    assert np.array_equal(s.get_all_blob_pos(), g["Y"])
    s.list_populate()
    assert np.array_equal(s.list_get_cells(), g["cells"])
    s.set_up_gaussians()
    ind, _ = s.get_gaussians()
    assert np.array_equal(ind, g["gauss_ind"])
    s.calculate_forces()
    assert rel_err(s.get_blob_forces(), g["forces"]) < 1e-12
    assert rel_err(s.apply_mobility(g["F"]), g["V"]) < TOL
    assert rel_err(s.multiply_by_K_at_midstep(g["U"]), g["KU"]) < TOL
    assert rel_err(s.multiply_by_KT_at_midstep(g["lam"]), g["KTlam"]) < TOL
    assert rel_err(s.multiply_by_Pinv(g["v"]), g["Pinv_v"]) < TOL
    assert rel_err(s.multiply_by_saddle_point_matrix(g["v"]), g["A_v"]) < TOL
    s.close()
