"""Fixtures from the reference itself: tests/golden/ref_<config>.npz.

Each fixture is computed by the reference's own classes, compiled unchanged from
its sources with the project-written stand-ins of oracle/ref_shim (one-rank
MPI, an Armadillo subset, FFTW 2.x real transforms, SPRNG) and the compile-time
parameters of oracle/ref_shim/cfg_<config>/config.hpp:

    make -C oracle ref          # needs the reference's sources (REF_SRC)
    python tests/golden/make_ref_golden.py

tests/test_oracle_vs_reference.py checks the oracle against these fixtures.
Bodies are placed by this script; the reference matrices are produced first,
with body 0 at the box (or channel) centre, as main.cpp:91-94 does before the
bodies are seeded; the noise is the SPRNG stand-in's stream (seed 77 / 5,
stream 0), which the oracle's sequential-noise mode reproduces.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from tests.ref_lib import Reference  # noqa: E402
from timstochrigidbodiessim_b200 import configs  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden")


def placement(config, R, rng):
    """Start bodies of a configuration: tetrahedra on a 3x2 lattice in the
    z = L/2 plane with random orientations; rods in the channel's mid-plane,
    parallel to the walls, a third of the box apart in z."""
    p = R.params()
    L = p.nx * p.dx
    if config.startswith("gdc_rods"):
        x = np.array([[14.5, 7.28, 5.0], [14.0, 7.28, 15.0], [15.0, 7.28, 24.5]]).ravel()
        th = rng.uniform(-0.2, 0.2, 3)
        q = np.stack([np.cos(th / 2), np.zeros(3), np.sin(th / 2), np.zeros(3)], 1).ravel()
        return x, q
    ijk = np.array([[i, j, 0] for i in range(3) for j in range(2)])
    x = ((ijk + 0.5) * np.array([L / 3, L / 2, 1.0]) + np.array([0, 0, L / 2])).ravel()
    q = configs.random_unit_quaternions(rng, R.M).ravel()
    if config.startswith("mcmc"):  # bodies brought close, so every pair term matters
        x = (x.reshape(-1, 3) * np.array([0.55, 0.6, 1.0])).ravel()
    return x, q


def make(config, steps):
    R = Reference(config)
    rng = np.random.default_rng(2024)
    out = {"cfg": R.cfg, "blob_ref_pos": R.ref}
    dynamic = not config.startswith("mcmc")
    if dynamic:
        R.produce_reference_matrices()  # body 0 at the centre, identity orientation
        Minv, N, K = R.get_reference_matrices()
        out.update(ref_Minv=Minv, ref_N=N, ref_KTKinv=K)
    x, q = placement(config, R, rng)
    R.set_bodies(x, q)
    out.update(x=x, q=q, Y=R.blob_positions(), cells=R.cells())
    ind, w = R.gaussians()
    out.update(gauss_ind=ind, gauss_w=w)
    if not dynamic:
        out["potential"] = np.array([R.potential()])
        np.savez_compressed(os.path.join(OUT, "ref_%s.npz" % config), **out)
        return
    F = rng.standard_normal(3 * R.Nb)
    U = rng.standard_normal(6 * R.M)
    lam = rng.standard_normal(3 * R.Nb)
    v = rng.standard_normal(R.n)
    out.update(F=F, V=R.mobility(F), U=U, KU=R.multiply_K(U), lam=lam, KTlam=R.multiply_KT(lam), v=v,
               Pinv_v=R.multiply_by_Pinv(v), A_v=R.multiply_by_saddle_point_matrix(v), forces=R.forces(0.0))
    R.sprng_reset(77, 0)
    out["V_random"] = R.random_velocities()
    R.set_bodies(x, q)
    R.sprng_reset(5, 0)
    xs, qs, sol, nus, sts = [], [], [], [], []
    for k in range(steps):
        st, soln, nu = R.step(k * float(R.cfg[9]))
        xb, qb = R.get_bodies()
        xs.append(xb)
        qs.append(qb)
        sol.append(soln)
        nus.append(nu)
        sts.append(st)
    out.update(step_x=np.array(xs), step_q=np.array(qs), step_soln=np.array(sol), step_nu=np.array(nus),
               step_status=np.array(sts))
    np.savez_compressed(os.path.join(OUT, "ref_%s.npz" % config), **out)


if __name__ == "__main__":
    wanted = sys.argv[1:] or ["em_tetra", "gdc_rods_slip", "mcmc_tetra_soft", "mcmc_tetra_philic"]
    for c in wanted:
        make(c, steps=3 if c == "em_tetra" else 2)
        print("wrote", c, flush=True)
