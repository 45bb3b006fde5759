"""ctypes wrapper of the reference build (oracle/_ref/libref_<config>.so): the
reference's own classes compiled unchanged from its sources with the stand-in
headers of oracle/ref_shim and the compile-time parameters of
oracle/ref_shim/cfg_<config>/config.hpp (recipe: `make -C oracle ref`).  Test
side only: it generates the fixtures that pin the oracle
(tests/golden/make_ref_golden.py) and, where the build exists, checks the
oracle against it directly.
"""
import ctypes
import os

import numpy as np

from timstochrigidbodiessim_b200.params import FcmParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
CONFIGS = ("em_tetra", "gdc_rods_slip")

D = ctypes.POINTER(ctypes.c_double)
I32 = ctypes.POINTER(ctypes.c_int32)


def available(config):
    return os.path.exists(os.path.join(REF_DIR, "libref_%s.so" % config))


def _dp(a):
    return a.ctypes.data_as(D)


class Reference:
    """One reference build: a collection, an FCM solver and a GMRES solver of the
    reference's classes, driven through oracle/ref_harness.cpp."""

    def __init__(self, config):
        L = ctypes.CDLL(os.path.join(REF_DIR, "libref_%s.so" % config))
        sig = {
            "rh_init": (ctypes.c_int, []),
            "rh_config": (None, [D]),
            "rh_blob_ref_pos": (None, [D]),
            "rh_set_bodies": (None, [D, D]),
            "rh_get_bodies": (None, [D, D]),
            "rh_produce_reference_matrices": (None, []),
            "rh_get_reference_matrices": (None, [D, D, D]),
            "rh_set_reference_matrices": (None, [D, D]),
            "rh_sprng_reset": (None, [ctypes.c_uint64, ctypes.c_uint64]),
            "rh_blob_positions": (None, [D]),
            "rh_gaussians": (None, [I32, D]),
            "rh_mobility": (None, [D, D]),
            "rh_random_velocities": (None, [D]),
            "rh_forces": (None, [ctypes.c_double, D]),
            "rh_potential": (ctypes.c_double, []),
            "rh_cells": (None, [I32]),
            "rh_multiply_K": (None, [D, D]),
            "rh_multiply_KT": (None, [D, D]),
            "rh_multiply_by_Pinv": (None, [D, D]),
            "rh_multiply_by_saddle_point_matrix": (None, [D, D]),
            "rh_step": (ctypes.c_int, [ctypes.c_double, D, D]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        self.L = L
        self.config = config
        self.nb = L.rh_init()
        c = np.zeros(19)
        L.rh_config(_dp(c))
        self.cfg = c
        self.M = int(c[0])
        self.Nb = self.M * self.nb
        self.n = 3 * self.Nb + 6 * self.M
        self.W = int(c[12])
        self.ref = np.zeros(3 * self.nb)
        L.rh_blob_ref_pos(_dp(self.ref))

    def params(self):
        """The oracle's FcmParams for this build's compile-time parameters."""
        c = self.cfg
        return FcmParams.defaults(nx=int(c[2]), ny=int(c[3]), nz=int(c[4]), dx=float(c[5]), blob_radius=float(c[6]),
                                  viscosity=float(c[7]), kT=float(c[8]), dt=float(c[9]), gmres_tol=float(c[10]),
                                  gmres_max_iter=int(c[11]), ngauss=int(c[12]), ncells=int(c[13]),
                                  slip_channel=int(c[14]), algorithm=int(c[15]), potential=int(c[16]),
                                  fd_delta=float(c[17]), skip_on_overlap=int(c[18]), num_bodies=self.M,
                                  blobs_per_body=self.nb, precision=0, noise=1)

    def set_bodies(self, x, q):
        x = np.ascontiguousarray(x, dtype=np.float64)
        q = np.ascontiguousarray(q, dtype=np.float64)
        self.L.rh_set_bodies(_dp(x), _dp(q))

    def get_bodies(self):
        x, q = np.zeros(3 * self.M), np.zeros(4 * self.M)
        self.L.rh_get_bodies(_dp(x), _dp(q))
        return x, q

    def produce_reference_matrices(self):
        self.L.rh_produce_reference_matrices()

    def get_reference_matrices(self):
        """(ref_Minv, ref_N, ref_KTKinv) as matrices, as the oracle returns them."""
        n3 = 3 * self.nb
        Minv, N, K = np.zeros(n3 * n3), np.zeros(36), np.zeros(36)
        self.L.rh_get_reference_matrices(_dp(Minv), _dp(N), _dp(K))
        return Minv.reshape(n3, n3, order="F"), N.reshape(6, 6, order="F"), K.reshape(6, 6, order="F")

    def set_reference_matrices(self, Minv, N):
        Minv = np.ascontiguousarray(np.asarray(Minv).ravel(order="F"), dtype=np.float64)
        N = np.ascontiguousarray(np.asarray(N).ravel(order="F"), dtype=np.float64)
        self.L.rh_set_reference_matrices(_dp(Minv), _dp(N))

    def sprng_reset(self, seed, stream=0):
        self.L.rh_sprng_reset(seed, stream)

    def _vec(self, name, n, *args):
        out = np.zeros(n)
        conv = [_dp(np.ascontiguousarray(a, dtype=np.float64)) if isinstance(a, np.ndarray) else a for a in args]
        getattr(self.L, name)(*conv, _dp(out))
        return out

    def blob_positions(self):
        return self._vec("rh_blob_positions", 3 * self.Nb)

    def gaussians(self):
        ind = np.zeros(3 * self.Nb * self.W, dtype=np.int32)
        w = np.zeros(3 * self.Nb * self.W)
        self.L.rh_gaussians(ind.ctypes.data_as(I32), _dp(w))
        return ind.reshape(self.Nb, 3, self.W), w.reshape(self.Nb, 3, self.W)

    def mobility(self, F):
        return self._vec("rh_mobility", 3 * self.Nb, np.asarray(F, dtype=np.float64))

    def random_velocities(self):
        return self._vec("rh_random_velocities", 3 * self.Nb)

    def forces(self, t=0.0):
        return self._vec("rh_forces", 3 * self.Nb, ctypes.c_double(t))

    def potential(self):
        return float(self.L.rh_potential())

    def cells(self):
        c = np.zeros(self.Nb, dtype=np.int32)
        self.L.rh_cells(c.ctypes.data_as(I32))
        return c

    def multiply_K(self, U):
        return self._vec("rh_multiply_K", 3 * self.Nb, np.asarray(U, dtype=np.float64))

    def multiply_KT(self, lam):
        return self._vec("rh_multiply_KT", 6 * self.M, np.asarray(lam, dtype=np.float64))

    def multiply_by_Pinv(self, v):
        return self._vec("rh_multiply_by_Pinv", self.n, np.asarray(v, dtype=np.float64))

    def multiply_by_saddle_point_matrix(self, v):
        return self._vec("rh_multiply_by_saddle_point_matrix", self.n, np.asarray(v, dtype=np.float64))

    def step(self, t):
        """One step in main.cpp's order; (status, saddle-point solution, nu)."""
        soln = np.zeros(self.n)
        nu = np.zeros(1)
        st = self.L.rh_step(ctypes.c_double(t), _dp(soln), _dp(nu))
        return int(st), soln, float(nu[0])
