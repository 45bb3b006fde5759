"""Synthetic suspensions with the shapes and sizes of the benchmark workloads.

Bodies are rigid straight rods of ``nb`` touching blobs (spacing 2.2a) with
centres uniform in the periodic box, orientations uniform unit quaternions (a
normalised 4-D Gaussian, as quaternion.cpp:10-17 draws them) and no inter-body
blob pair closer than 2a.  Each body carries the constant force (0, 0, -1).
Steric repulsion is the polynomial potential 3 with F_s = 40 kT/a
(= U0/b of the reference's soft sphere) and r_c = 2.2a; the cell list uses the
largest cell count whose cells are at least r_c wide.
"""
import math

import numpy as np

from .params import FcmParams, rod_reference_positions

A = 1.0


def box_for_volume_fraction(num_blobs, phi, a=A):
    return (num_blobs * 4.0 / 3.0 * math.pi * a ** 3 / phi) ** (1.0 / 3.0)


def random_unit_quaternions(rng, n):
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q


def rotation_matrices(q):
    """Rotation matrices of quaternion.cpp:61-103 for an (n,4) array."""
    s, v0, v1, v2 = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    R = np.zeros((len(q), 3, 3))
    R[:, 0, 0] = 1 - 2 * v1 * v1 - 2 * v2 * v2
    R[:, 1, 1] = 1 - 2 * v0 * v0 - 2 * v2 * v2
    R[:, 2, 2] = 1 - 2 * v0 * v0 - 2 * v1 * v1
    R[:, 0, 1] = 2 * v0 * v1 - 2 * s * v2
    R[:, 1, 0] = 2 * v0 * v1 + 2 * s * v2
    R[:, 0, 2] = 2 * v0 * v2 + 2 * s * v1
    R[:, 2, 0] = 2 * v0 * v2 - 2 * s * v1
    R[:, 1, 2] = 2 * v1 * v2 - 2 * s * v0
    R[:, 2, 1] = 2 * v1 * v2 + 2 * s * v0
    return R


def seed_bodies(rng, M, ref, L, min_dist=2.0 * A, max_trials=200000):
    """Random non-overlapping placement by rejection (cell-hashed blob checks)."""
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, 3)
    nb = len(ref)
    cell = max(min_dist, 1e-9)
    ncell = max(1, int(L // cell))
    h = L / ncell
    grid = {}
    xs = np.zeros((M, 3))
    qs = np.zeros((M, 4))
    placed = 0
    trials = 0
    md2 = min_dist * min_dist
    while placed < M:
        trials += 1
        if trials > max_trials:
            raise RuntimeError("could not place %d bodies (placed %d)" % (M, placed))
        x = rng.uniform(0.0, L, 3)
        q = random_unit_quaternions(rng, 1)[0]
        R = rotation_matrices(q[None])[0]
        pos = (x[None, :] + ref @ R.T) % L
        ok = True
        for p in pos:
            ci = (p // h).astype(int) % ncell
            for dx in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dz in (-1, 0, 1):
                        key = ((ci[0] + dx) % ncell, (ci[1] + dy) % ncell, (ci[2] + dz) % ncell)
                        for o in grid.get(key, ()):
                            d = p - o
                            d -= L * np.round(d / L)
                            if d @ d < md2:
                                ok = False
                                break
                        if not ok:
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        for p in pos:
            ci = tuple((p // h).astype(int) % ncell)
            grid.setdefault(ci, []).append(p)
        xs[placed] = x
        qs[placed] = q
        placed += 1
    return xs.ravel(), qs.ravel()


def rod_suspension(M, grid, L=None, phi=None, nb=6, seed=1234, gmres_tol=1e-10, gmres_max_iter=100,
                   dt=0.01, kT=1.0, noise=1, algorithm=2, precision=0, ngauss=20):
    """Params, blob_ref_pos, x, q and external forces of a rod suspension."""
    Nb = M * nb
    if L is None:
        L = box_for_volume_fraction(Nb, phi)
    rc = 2.2 * A
    ncells = max(3, int(L // rc))
    p = FcmParams.defaults(nx=grid, ny=grid, nz=grid, ngauss=ngauss, dx=L / grid, blob_radius=A,
                           viscosity=1.0, kT=kT, dt=dt, num_bodies=M, blobs_per_body=nb, ncells=ncells,
                           potential=3, steric_fs=40.0 * kT / A, steric_rc=rc, gmres_max_iter=gmres_max_iter,
                           gmres_tol=gmres_tol, fd_delta=1e-5, algorithm=algorithm, precision=precision,
                           noise=noise, skip_on_overlap=0)
    ref = np.array(rod_reference_positions(nb, 2.2, A))
    rng = np.random.default_rng(seed)
    x, q = seed_bodies(rng, M, ref, L)
    fe = np.zeros(6 * M)
    fe[2::6] = -1.0
    return p, ref, x, q, fe


# The benchmark workloads (sizes as stated; synthetic, seeded).
WORKLOADS = {
    # 32 rods, L = 64a, 64^3 grid: the CPU-runnable case
    "rods32_L64_g64": dict(M=32, grid=64, L=64.0),
    # 2048 rods (12,288 blobs), volume fraction 0.10, 256^3 grid
    "rods2048_phi0.10_g256": dict(M=2048, grid=256, phi=0.10),
    # 8192 rods (49,152 blobs), volume fraction 0.15, 384^3 grid
    "rods8192_phi0.15_g384": dict(M=8192, grid=384, phi=0.15),
}


def workload(name, **overrides):
    kw = dict(WORKLOADS[name])
    kw.update(overrides)
    return rod_suspension(**kw)
