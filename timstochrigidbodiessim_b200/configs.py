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


def relax_overlaps(x, q, ref, L, min_dist=2.0 * A, max_iter=5000):
    """Push overlapping bodies apart until no inter-body blob pair is closer than
    min_dist: the drag relaxation of collection_of_rigid_bodies.cpp:491-615
    (blob repulsion summed to body force and torque, applied with a drag
    mobility), with a linear repulsion and a periodic KD-tree for the pairs."""
    from scipy.spatial import cKDTree
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, 3)
    nb = len(ref)
    x = x.reshape(-1, 3).copy()
    q = q.reshape(-1, 4).copy()
    M = len(x)
    body = np.repeat(np.arange(M), nb)
    target = 1.02 * min_dist
    for _ in range(max_iter):
        R = rotation_matrices(q)
        r = np.einsum("nij,mj->nmi", R, ref).reshape(-1, 3)
        Y = (np.repeat(x, nb, axis=0) + r) % L
        pairs = cKDTree(Y % L, boxsize=L).query_pairs(target, output_type="ndarray")
        if len(pairs):
            pairs = pairs[body[pairs[:, 0]] != body[pairs[:, 1]]]
        if not len(pairs):
            break
        d = Y[pairs[:, 0]] - Y[pairs[:, 1]]
        d -= L * np.round(d / L)
        dist = np.linalg.norm(d, axis=1, keepdims=True)
        if dist.min() >= min_dist:  # pushed towards `target`, done once clear of min_dist
            break
        f = (target - dist) * d / np.maximum(dist, 1e-12)
        Fb = np.zeros_like(Y)
        np.add.at(Fb, pairs[:, 0], f)
        np.add.at(Fb, pairs[:, 1], -f)
        Fbody = np.zeros((M, 3))
        Tbody = np.zeros((M, 3))
        np.add.at(Fbody, body, Fb)
        np.add.at(Tbody, body, np.cross(r, Fb))
        x = (x + 0.5 * Fbody / nb) % L
        w = 0.5 * Tbody / (nb * max(1.0, float(np.mean(np.sum(ref ** 2, axis=1)))))
        th = np.linalg.norm(w, axis=1)
        ok = th > 1e-12
        e = np.zeros((M, 4))
        e[:, 0] = 1.0
        e[ok, 0] = np.cos(0.5 * th[ok])
        e[ok, 1:] = np.sin(0.5 * th[ok])[:, None] * w[ok] / th[ok, None]
        s0, v0 = e[:, 0], e[:, 1:]
        s1, v1 = q[:, 0], q[:, 1:]
        q = np.concatenate([(s0 * s1 - np.sum(v0 * v1, axis=1))[:, None],
                            s0[:, None] * v1 + s1[:, None] * v0 + np.cross(v0, v1)], axis=1)
        q /= np.linalg.norm(q, axis=1, keepdims=True)
    else:
        raise RuntimeError("overlap relaxation did not converge")
    return x.ravel(), q.ravel()


def seed_bodies(rng, M, ref, L, min_dist=2.0 * A, max_trials=200000, max_fail=3000):
    """Random non-overlapping placement by rejection sampling.  When the box is too
    crowded for that (rods jam near volume fraction 0.2), place the bodies by
    rejection in a box of 0.85x the target density and compress it to L in 1%
    steps of the side, relaxing overlaps after each step."""
    try:
        return _rsa(rng, M, ref, L, min_dist, max_trials, max_fail)
    except RuntimeError:
        pass
    L0 = L * (1.0 / 0.85) ** (1.0 / 3.0)
    x, q = _rsa(rng, M, ref, L0, min_dist, max_trials, max_fail)
    Lc = L0
    while Lc > L:
        Ln = max(L, Lc * 0.99)
        x = (x * (Ln / Lc)) % Ln
        x, q = relax_overlaps(x, q, ref, Ln, min_dist)
        Lc = Ln
    return x, q


def _rsa(rng, M, ref, L, min_dist, max_trials=None, max_fail=None, batch=2048, max_empty=24):
    """Random sequential addition, vectorised: batches of candidate bodies are
    checked against the placed blobs with a periodic KD-tree, and accepted one by
    one against the blobs accepted since the tree was built.  Raises when
    max_empty consecutive batches add nothing (jammed)."""
    from scipy.spatial import cKDTree
    ref = np.asarray(ref, dtype=np.float64).reshape(-1, 3)
    nb = len(ref)
    xs, qs = [], []
    placed_Y = np.zeros((0, 3))
    md2 = min_dist * min_dist
    empty = 0
    while len(xs) < M:
        tree = cKDTree(placed_Y % L, boxsize=L) if len(placed_Y) else None
        cx = rng.uniform(0.0, L, (batch, 3))
        cq = random_unit_quaternions(rng, batch)
        cY = ((cx[:, None, :] + np.einsum("nij,mj->nmi", rotation_matrices(cq), ref)) % L)
        if tree is not None:
            hit = tree.query_ball_point(cY.reshape(-1, 3), r=min_dist * (1.0 - 1e-12), return_length=True, workers=-1)
            ok = ~(hit.reshape(batch, nb) > 0).any(axis=1)
        else:
            ok = np.ones(batch, dtype=bool)
        recent = np.zeros((0, 3))
        added = 0
        for c in np.nonzero(ok)[0]:
            if len(recent):
                d = cY[c][:, None, :] - recent[None, :, :]
                d -= L * np.round(d / L)
                if (np.einsum("ijk,ijk->ij", d, d) < md2).any():
                    continue
            xs.append(cx[c])
            qs.append(cq[c])
            recent = np.concatenate([recent, cY[c]])
            added += 1
            if len(xs) == M or added >= 32:
                break
        placed_Y = np.concatenate([placed_Y, recent])
        empty = 0 if added else empty + 1
        if empty >= max_empty:
            raise RuntimeError("could not place %d bodies (placed %d)" % (M, len(xs)))
    return np.array(xs).ravel(), np.array(qs).ravel()


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


def rod_channel(M, grid, L, nb=6, seed=1234, margin=2.2 * A, gmres_tol=1e-10, gmres_max_iter=100, dt=0.01,
                kT=1.0, noise=1, algorithm=2, precision=0, ngauss=20, max_trials=200000):
    """A rod suspension in a slip channel (slip_channel = 1): an L^3 periodic box
    whose bodies live in 0 < y < L/2, every blob at least `margin` from the walls
    (outside the walls' spring range 2.2a by default), placed by rejection.
    Returns params, blob_ref_pos, x, q and external forces (-1 along z, parallel
    to the walls)."""
    p, ref, _, _, fe = rod_suspension(M=1, grid=grid, L=L, nb=nb, seed=seed, gmres_tol=gmres_tol,
                                      gmres_max_iter=gmres_max_iter, dt=dt, kT=kT, noise=noise,
                                      algorithm=algorithm, precision=precision, ngauss=ngauss)
    p.num_bodies = M
    p.slip_channel = 1
    rng = np.random.default_rng(seed)
    H = 0.5 * L
    Y = np.zeros((0, 3))
    xs, qs = [], []
    for _ in range(max_trials):
        if len(xs) == M:
            break
        c = rng.uniform(0.0, 1.0, 3) * np.array([L, H, L])
        qq = random_unit_quaternions(rng, 1)
        b = c + (rotation_matrices(qq)[0] @ np.asarray(ref).reshape(-1, 3).T).T
        if b[:, 1].min() < margin or b[:, 1].max() > H - margin:
            continue
        b[:, 0] %= L
        b[:, 2] %= L
        if len(Y):
            d = np.abs(Y[None, :, :] - b[:, None, :])
            d[..., 0] = np.minimum(d[..., 0], L - d[..., 0])
            d[..., 2] = np.minimum(d[..., 2], L - d[..., 2])
            if (np.einsum("ijk,ijk->ij", d, d) < (2.0 * A) ** 2).any():
                continue
        Y = np.vstack([Y, b])
        xs.append([c[0] % L, c[1], c[2] % L])
        qs.append(qq[0])
    if len(xs) < M:
        raise RuntimeError("rod_channel: could not place %d rods" % M)
    fe = np.zeros(6 * M)
    fe[2::6] = -1.0
    return p, ref, np.array(xs).ravel(), np.array(qs).ravel(), fe


def random_walk_cluster(rng, nb=12, bond=2.2 * A, min_dist=2.0 * A, draws=32, max_tries=100000):
    """A rigid cluster shape grown from a seed blob: each new blob is bonded at
    distance `bond` to a randomly chosen earlier blob, at least min_dist from all
    of them; of `draws` such clusters the most compact (smallest largest distance
    from the centroid) is kept, re-centred on its centroid.  Returns (nb, 3)."""
    best, best_r = None, np.inf
    tries = 0
    for _ in range(draws):
        pts = [np.zeros(3)]
        while len(pts) < nb:
            tries += 1
            if tries > max_tries:
                raise RuntimeError("cluster could not grow")
            v = rng.standard_normal(3)
            c = pts[rng.integers(len(pts))] + bond * v / np.linalg.norm(v)
            if min(np.linalg.norm(c - p) for p in pts) >= min_dist * (1.0 - 1e-12):
                pts.append(c)
        P = np.array(pts)
        P -= P.mean(axis=0)
        r = np.linalg.norm(P, axis=1).max()
        if r < best_r:
            best, best_r = P, r
    return best


def random_walk_clusters(rng, M, nb=12, bond=2.2 * A, min_dist=2.0 * A, draws=4, max_rounds=100000):
    """M independent random cluster shapes, grown all at once: each starts from a
    seed blob, and every new blob is bonded at distance `bond` to a randomly
    chosen earlier blob of its cluster, at least min_dist from all of them (a
    rejected draw is drawn again); of `draws` clusters grown per shape the most
    compact (smallest largest distance from the centroid) is kept, re-centred on
    its centroid.  Returns (M, nb, 3)."""
    n = M * draws
    pts = np.zeros((n, nb, 3))
    rounds = 0
    for k in range(1, nb):
        todo = np.arange(n)
        while len(todo):
            rounds += 1
            if rounds > max_rounds:
                raise RuntimeError("clusters could not grow")
            j = rng.integers(0, k, len(todo))
            v = rng.standard_normal((len(todo), 3))
            c = pts[todo, j] + bond * v / np.linalg.norm(v, axis=1, keepdims=True)
            d = np.linalg.norm(pts[todo, :k] - c[:, None, :], axis=2).min(axis=1)
            ok = d >= min_dist * (1.0 - 1e-12)
            pts[todo[ok], k] = c[ok]
            todo = todo[~ok]
    pts -= pts.mean(axis=1, keepdims=True)
    r = np.linalg.norm(pts, axis=2).max(axis=1).reshape(M, draws)
    best = r.argmin(axis=1)
    return pts.reshape(M, draws, nb, 3)[np.arange(M), best]


def lattice_start(rng, M, ref, L, min_dist=2.0 * A, tries=16, rounds=12, jitter=0.0):
    """Bodies of shape ref (nb, 3) -- or each of its own shape, ref (M, nb, 3) --
    near the sites of a cubic lattice of side
    M^(1/3) in the box L (each centre within +-jitter spacings of its site),
    each placed and turned to keep its blobs at least min_dist from the blobs of
    the bodies placed before it.  Sites are filled in 27 classes
    (i, j, k mod 3), so bodies of one class (three spacings apart) are placed
    together against a periodic KD-tree of the placed blobs; a site with no clear
    orientation after `rounds` batches of `tries` draws keeps the draw with the
    largest clearance.  Returns x (M, 3), q (M, 4)."""
    from scipy.spatial import cKDTree
    ref = np.asarray(ref, dtype=np.float64)
    if ref.ndim == 3:  # (M, nb, 3): one shape per body
        shapes = ref
    else:
        shapes = np.broadcast_to(ref.reshape(1, -1, 3), (M, ref.size // 3, 3))
    nb = shapes.shape[1]
    side = int(round(M ** (1.0 / 3.0)))
    if side ** 3 != M:
        raise ValueError("M must be a cube for the lattice start")
    idx = np.arange(M)
    ijk = np.stack([idx // (side * side), (idx // side) % side, idx % side], axis=1)
    sp = L / side
    x = (ijk + 0.5) * sp
    q = np.zeros((M, 4))
    placed_Y = np.zeros((0, 3))
    cls = (ijk % 3) @ np.array([9, 3, 1])
    for c in range(27):
        mem = np.nonzero(cls == c)[0]
        tree = cKDTree(placed_Y % L, boxsize=L) if len(placed_Y) else None
        best_q = random_unit_quaternions(rng, len(mem))
        best_x = x[mem].copy()
        best_d = np.full(len(mem), -1.0)
        todo = np.ones(len(mem), dtype=bool)
        for _ in range(rounds):
            if tree is None or not todo.any():
                break
            sel = np.nonzero(todo)[0]
            qs = random_unit_quaternions(rng, len(sel) * tries)
            xs = np.repeat(x[mem[sel]], tries, axis=0) + rng.uniform(-jitter, jitter, (len(sel) * tries, 3)) * sp
            sh = np.repeat(shapes[mem[sel]], tries, axis=0)                                    # (s*t, nb, 3)
            cb = (xs[:, None, :] + np.einsum("tij,tnj->tni", rotation_matrices(qs), sh)) % L   # (s*t, nb, 3)
            dist, _ = tree.query(cb.reshape(-1, 3), k=1, workers=-1)
            dist = dist.reshape(len(sel), tries, nb).min(axis=2)
            k = dist.argmax(axis=1)
            dk = dist[np.arange(len(sel)), k]
            better = dk > best_d[sel]
            best_d[sel[better]] = dk[better]
            best_q[sel[better]] = qs.reshape(len(sel), tries, 4)[better, k[better]]
            best_x[sel[better]] = xs.reshape(len(sel), tries, 3)[better, k[better]]
            todo[sel] = best_d[sel] < min_dist
        q[mem] = best_q
        x[mem] = best_x % L
        Yc = (x[mem][:, None, :] + np.einsum("mij,mnj->mni", rotation_matrices(best_q), shapes[mem])).reshape(-1, 3)
        placed_Y = np.concatenate([placed_Y, Yc])
    return x, q


def cluster_suspension(M, grid, phi, nb=12, seed=1234, gmres_tol=1e-10, gmres_max_iter=100, dt=0.01, kT=1.0,
                       noise=1, algorithm=2, precision=0, ngauss=20, per_body=True):
    """M rigid random clusters of nb blobs at volume fraction phi.  With per_body
    (the default) every body has its own shape (random_walk_clusters), and the
    returned blob_ref_pos holds 3*nb values per body (set on a context with
    set_body_shapes, see make_suspension); otherwise one shape
    (random_walk_cluster, the most compact of 32 draws) is shared by all bodies, as
    the reference's collection has one blob_ref_pos.  Centres on a cubic lattice
    (side M^(1/3)), orientations drawn to clear the neighbours (lattice_start);
    what overlap remains is left to the Metropolis equilibration.  Params,
    blob_ref_pos, x, q and external forces."""
    rng = np.random.default_rng(seed)
    if per_body:
        shapes = random_walk_clusters(rng, M, nb)
    else:
        shapes = random_walk_cluster(rng, nb)
    Nb = M * nb
    L = box_for_volume_fraction(Nb, phi)
    rc = 2.2 * A
    ncells = max(3, int(L // rc))
    p = FcmParams.defaults(nx=grid, ny=grid, nz=grid, ngauss=ngauss, dx=L / grid, blob_radius=A,
                           viscosity=1.0, kT=kT, dt=dt, num_bodies=M, blobs_per_body=nb, ncells=ncells,
                           potential=3, steric_fs=40.0 * kT / A, steric_rc=rc, gmres_max_iter=gmres_max_iter,
                           gmres_tol=gmres_tol, fd_delta=1e-5, algorithm=algorithm, precision=precision,
                           noise=noise, skip_on_overlap=0)
    x, q = lattice_start(rng, M, shapes, L)
    fe = np.zeros(6 * M)
    fe[2::6] = -1.0
    return p, shapes.ravel(), x.ravel(), q.ravel(), fe


def has_body_shapes(p, ref):
    """Whether blob_ref_pos `ref` holds one shape per body (3*nb*M values) rather
    than the single shared shape (3*nb)."""
    n = np.asarray(ref).size
    return p.num_bodies > 1 and n == 3 * p.blobs_per_body * p.num_bodies


def make_suspension(p, ref, stream=None, cls=None):
    """A context (Suspension, or `cls`, e.g. the oracle) for params p and
    blob_ref_pos ref: the shared shape, or per-body shapes set with
    set_body_shapes (the oracle then also forms its per-body preconditioner)."""
    if cls is None:
        from .fcm import Suspension
        s = Suspension(p, np.asarray(ref).ravel()[:3 * p.blobs_per_body], stream=stream)
    else:
        s = cls(p, np.asarray(ref).ravel()[:3 * p.blobs_per_body])
    if has_body_shapes(p, ref):
        s.set_body_shapes(np.asarray(ref).ravel())
        if hasattr(s, "produce_body_preconditioners"):
            s.produce_body_preconditioners()
    return s


# The benchmark workloads (sizes as stated; synthetic, seeded).
WORKLOADS = {
    # 32 rods, L = 64a, 64^3 grid: the CPU-runnable case
    "rods32_L64_g64": dict(M=32, grid=64, L=64.0),
    # 2048 rods (12,288 blobs), volume fraction 0.10, 256^3 grid
    "rods2048_phi0.10_g256": dict(M=2048, grid=256, phi=0.10),
    # 8192 rods (49,152 blobs), volume fraction 0.15, 384^3 grid
    "rods8192_phi0.15_g384": dict(M=8192, grid=384, phi=0.15),
    # 32,768 rigid 12-blob random clusters (393,216 blobs), volume fraction
    # 0.20, 512^3 grid; started on a lattice, equilibrated by Metropolis steps
    "clusters32768_phi0.20_g512": dict(kind="clusters", M=32768, grid=512, phi=0.20, mcmc_steps=10000),
    # the same grid spacing (0.394a), volume fraction and cluster size in one
    # eighth of the volume: 4096 clusters (49,152 blobs) on a 256^3 grid, the
    # profiling stand-in for the 512^3 suspension
    "clusters4096_phi0.20_g256": dict(kind="clusters", M=4096, grid=256, phi=0.20, mcmc_steps=2000),
}


def workload(name, **overrides):
    """(params, blob_ref_pos, x, q, forces) of a named workload.  For cluster
    workloads the Metropolis equilibration (WORKLOADS[name]["mcmc_steps"]) is
    run separately (equilibrate), since it needs the GPU library."""
    kw = dict(WORKLOADS[name])
    kw.update(overrides)
    kind = kw.pop("kind", "rods")
    kw.pop("mcmc_steps", None)
    if kind == "clusters":
        return cluster_suspension(**kw)
    return rod_suspension(**kw)


def equilibrate(p, ref, x, q, steps, seed=1234, stream=None):
    """Metropolis equilibration on the GPU (fcm_mcmc_run, main.cpp:113-210) of
    bodies x, q; returns the new (x, q) and the final fcm_mcmc_state."""
    s = make_suspension(p, ref, stream=stream)
    try:
        s.set_bodies(x, q)
        st = s.mcmc_run(seed, steps)
        x2, q2 = s.get_bodies()
    finally:
        s.close()
    return x2, q2, st


def nearest_fft_size(n, lo=64, hi=128):
    """Nearest 2^k or 3*2^k to n, clamped to [lo, hi]."""
    cands = sorted({2 ** k for k in range(4, 12)} | {3 * 2 ** k for k in range(3, 11)})
    best = min(cands, key=lambda c: (abs(c - n), c))
    return int(min(max(best, lo), hi))


def ensemble_member(i, seed0=0, nb=6, gmres_tol=1e-10, dt=0.01, precision=0, **kw):
    """Instance i of the batched ensemble (seed seed0 + i): U[50, 500] rods of nb
    blobs at volume fraction U[0.05, 0.20]; its grid is the 2^k or 3*2^k nearest
    to L/(a/1.86), clamped to 64..128 points per side."""
    rng = np.random.default_rng(seed0 + i)
    M = int(rng.integers(50, 501))
    phi = float(rng.uniform(0.05, 0.20))
    L = box_for_volume_fraction(M * nb, phi)
    grid = nearest_fft_size(1.86 * L / A)
    p, ref, x, q, fe = rod_suspension(M=M, grid=grid, L=L, nb=nb, seed=seed0 + i, gmres_tol=gmres_tol, dt=dt,
                                      precision=precision, **kw)
    return p.as_dict(), ref, x, q, fe


def ensemble_body_counts(n_instances=64, seed0=0):
    """Body count of every ensemble instance (the first draw of ensemble_member),
    without building the instances."""
    return [int(np.random.default_rng(seed0 + i).integers(50, 501)) for i in range(n_instances)]


def ensemble(n_instances=64, seed0=0, workers=1, **kw):
    """The batched ensemble (see ensemble_member), built in `workers` spawned
    processes when workers > 1."""
    import functools
    f = functools.partial(ensemble_member, seed0=seed0, **kw)
    if workers > 1:
        import concurrent.futures as cf
        import multiprocessing as mp
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
            raw = list(ex.map(f, range(n_instances)))
    else:
        raw = [f(i) for i in range(n_instances)]
    return [(FcmParams.defaults(**pd), ref, x, q, fe) for pd, ref, x, q, fe in raw]
