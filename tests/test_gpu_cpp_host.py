"""The reference-named C++ classes (csrc/host) through the rigid_bodies_sim
driver, which runs main.cpp's loop on them, against the CPU oracle."""
import os
import subprocess

import numpy as np
import pytest

from tests.oracle_lib import Oracle
from timstochrigidbodiessim_b200 import build, configs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("algorithm", [2, 1])
def test_driver_matches_oracle(gpu, tmp_path, algorithm):
    p, ref, x, q, fe = configs.rod_suspension(M=8, grid=32, L=24.0, nb=6, seed=5, gmres_tol=1e-12, noise=0,
                                              ngauss=12, algorithm=algorithm)
    shape = tmp_path / "shape.txt"
    shape.write_text("\n".join("%.17g %.17g %.17g" % tuple(ref[3 * m:3 * m + 3]) for m in range(p.blobs_per_body)))
    ic = tmp_path / "ic.dat"
    ic.write_text("0 " + " ".join("%.17g %.17g %.17g %.17g %.17g %.17g %.17g" % (tuple(x[3 * n:3 * n + 3]) +
                                                                                tuple(q[4 * n:4 * n + 4]))
                                  for n in range(p.num_bodies)) + "\n")
    args = [build.DRIVER, "shape=%s" % shape, "ic=%s" % ic, "steps=3", "name=%s" % (tmp_path / "run"),
            "digits=17", "body_force_z=-1"]
    for k in ("nx", "ny", "nz", "ngauss", "dx", "dt", "ncells", "potential", "steric_fs", "steric_rc",
              "gmres_max_iter", "gmres_tol", "algorithm", "noise"):
        args.append("%s=%r" % (k, getattr(p, k)))
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "run.dat").read_text().strip().splitlines()
    assert len(lines) == 3
    last = np.array([float(v) for v in lines[-1].split()])
    xg = last[1:].reshape(-1, 7)[:, :3].ravel()
    qg = last[1:].reshape(-1, 7)[:, 3:].ravel()
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    o.set_external_forces(fe)
    o.produce_reference_matrices()
    for i in range(3):
        st, info = o.step(0, i)
        assert st == 0
    xo, qo = o.get_bodies()
    assert np.abs(xg - xo).max() < 1e-8
    assert np.abs(qg - qo).max() < 1e-8
    assert "skipped_steps 0" in r.stdout


def test_driver_mcmc_matches_oracle(gpu, tmp_path):
    """The driver's MARKOV_CHAIN_MONTE_CARLO mode (main.cpp:113-210): samples
    every 200 steps once past mcmc_save_after, the last one equal to the
    oracle's run of the same length and seed; also writes the blob forces file
    in time-stepping mode."""
    p, ref, x, q, fe = configs.rod_suspension(M=32, grid=32, L=24.0, seed=3)
    p = p.copy(potential=0, ncells=3)
    shape = tmp_path / "shape.txt"
    shape.write_text("\n".join("%.17g %.17g %.17g" % tuple(ref[3 * m:3 * m + 3]) for m in range(p.blobs_per_body)))
    ic = tmp_path / "ic.dat"
    ic.write_text("0 " + " ".join("%.17g %.17g %.17g %.17g %.17g %.17g %.17g" % (tuple(x[3 * n:3 * n + 3]) +
                                                                                tuple(q[4 * n:4 * n + 4]))
                                  for n in range(p.num_bodies)) + "\n")
    args = [build.DRIVER, "shape=%s" % shape, "ic=%s" % ic, "mcmc=400", "mcmc_save_after=0", "seed=9",
            "name=%s" % (tmp_path / "mc"), "digits=17"]
    for k in ("nx", "ny", "nz", "ngauss", "dx", "dt", "ncells", "potential", "kT"):
        args.append("%s=%r" % (k, getattr(p, k)))
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = (tmp_path / "mc.dat").read_text().strip().splitlines()
    assert len(lines) == 2 and lines[-1].split()[0].startswith("4")
    last = np.array([float(v) for v in lines[-1].split()])
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    st, state = o.mcmc_run(9, 400)
    xo, qo = o.get_bodies()
    assert np.abs(last[1:].reshape(-1, 7)[:, :3].ravel() - xo).max() < 1e-12
    assert np.abs(last[1:].reshape(-1, 7)[:, 3:].ravel() - qo).max() < 1e-12
    assert "Saved sample 400" in r.stdout


def test_driver_shear_matches_oracle(gpu, tmp_path):
    """The driver with SHEARING_FORCES (shear=1): GDC steps on the oracle's
    trajectory with the imposed flow on, and one x-velocity profile per save
    (main.cpp:371-433), whose mean over y is zero (the k = 0 mode is removed)
    and which follows the imposed sin profile."""
    p, ref, x, q, fe = configs.rod_suspension(M=8, grid=32, L=24.0, nb=6, seed=5, gmres_tol=1e-12, noise=0,
                                              ngauss=12, algorithm=1)
    shape = tmp_path / "shape.txt"
    shape.write_text("\n".join("%.17g %.17g %.17g" % tuple(ref[3 * m:3 * m + 3]) for m in range(p.blobs_per_body)))
    ic = tmp_path / "ic.dat"
    ic.write_text("0 " + " ".join("%.17g %.17g %.17g %.17g %.17g %.17g %.17g" % (tuple(x[3 * n:3 * n + 3]) +
                                                                                tuple(q[4 * n:4 * n + 4]))
                                  for n in range(p.num_bodies)) + "\n")
    args = [build.DRIVER, "shape=%s" % shape, "ic=%s" % ic, "steps=3", "name=%s" % (tmp_path / "sh"),
            "digits=17", "body_force_z=-1", "shear=1", "shear_scale=2.0", "shear_wavenumber=1.0"]
    for k in ("nx", "ny", "nz", "ngauss", "dx", "dt", "ncells", "potential", "steric_fs", "steric_rc",
              "gmres_max_iter", "gmres_tol", "algorithm", "noise"):
        args.append("%s=%r" % (k, getattr(p, k)))
    r = subprocess.run(args, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    last = np.array([float(v) for v in (tmp_path / "sh.dat").read_text().strip().splitlines()[-1].split()])
    o = Oracle(p, ref)
    o.set_bodies(x, q)
    o.set_external_forces(fe)
    o.produce_reference_matrices()
    o.produce_shear_velocity_field(2.0, 1.0)
    for i in range(3):
        assert o.step(0, i)[0] == 0
    xo, qo = o.get_bodies()
    assert np.abs(last[1:].reshape(-1, 7)[:, :3].ravel() - xo).max() < 1e-8
    assert np.abs(last[1:].reshape(-1, 7)[:, 3:].ravel() - qo).max() < 1e-8
    prof = (tmp_path / "sh_fluid_x_velocity_in_y.dat").read_text().strip().splitlines()
    assert len(prof) == 3
    u = np.array([float(v) for v in prof[-1].split()[1:]])
    assert u.size == p.ny
    L = p.ny * p.dx
    k = 2 * np.pi / L
    amp = 2.0 * p.kT / (p.blob_radius * p.viscosity * k * k)
    assert abs(u.mean()) < 1e-5 * amp  # the saved values carry 6 digits
    assert np.corrcoef(u, np.sin(k * np.arange(p.ny) * p.dx))[0, 1] > 0.99
