"""Generate the golden fixtures in tests/golden/ (run: python tests/golden/make_golden.py).

The reference (timwestwood/TimStochRigidBodiesSim) ships no tests or golden
data and cannot be built here (MPI, Armadillo, FFTW 2.x, SPRNG are absent).
These fixtures come from a second, independent restatement of the reference's
formulas written with numpy only (no code shared with oracle/), using numpy's
pocketfft, whose rfftn/irfftn have the same sign, scaling and non-Hermitian
C2R behaviour as FFTW 2.x's rfftwnd.  The oracle is pinned by matching them.

Cases (all seeded, tiny):
  fft_*        : fft_solver transform / inverse_transform in the padded,
                 transposed layout (fft_solver.cpp:17-42)
  mobility_*   : M F of fcm_fluid_solver.cpp:131-165, :552-600, :636-701, :363-424
  random_*     : the fluctuating field of :236-361 from injected stress arrays
  cells_*      : cell ids, inter-body pair set and steric forces of linked_list.cpp
  bodies_*     : blob positions, K, K^T, body update (collection_of_rigid_bodies.cpp,
                 particle.cpp, quaternion.cpp)
"""
import math
import os

import numpy as np

PI = 3.14159265358979323846264338327950288
HERE = os.path.dirname(os.path.abspath(__file__))


# ------------------------------------------------------------------ FFT layout
def padded(real):
    nx, ny, nz = real.shape
    pad = 2 * (nz // 2 + 1)
    a = np.zeros((nx, ny, pad))
    a[:, :, :nz] = real
    return a


def fft_transform(real):
    """fft_solver::transform: padded real -> complex in [y][x][kz] order."""
    nx, ny, nz = real.shape
    c = np.fft.rfftn(real).transpose(1, 0, 2)
    out = np.zeros((ny, nx, 2 * (nz // 2 + 1)))
    out[..., 0::2] = c.real
    out[..., 1::2] = c.imag
    return out


def fft_inverse(spec_t, shape):
    """fft_solver::inverse_transform of a complex [y][x][kz] array."""
    nx, ny, nz = shape
    H = spec_t[..., 0::2] + 1j * spec_t[..., 1::2]
    r = np.fft.irfftn(H.transpose(1, 0, 2), s=(nx, ny, nz), axes=(0, 1, 2)) * (nx * ny * nz)
    return padded(r)


# ------------------------------------------------------------------ FCM pieces
def gaussians(Y, N, dx, a, W):
    anorm = 1.0 / (math.sqrt(2.0) * a)
    anorm2 = 2.0 * a * a / PI
    Nb = len(Y)
    ind = np.zeros((Nb, 3, W), dtype=np.int64)
    w = np.zeros((Nb, 3, W))
    for n in range(Nb):
        for d in range(3):
            xc = int(Y[n, d] / dx)
            for i in range(W):
                xg = xc - W // 2 + (i + 1)
                ind[n, d, i] = xg % N[d]
                xx = xg * dx - Y[n, d]
                w[n, d, i] = anorm * math.exp(-xx * xx / anorm2)
    return ind, w


def spread(F, ind, w, N):
    g = np.zeros((3,) + tuple(N))
    for n in range(len(ind)):
        ker = np.einsum("i,j,k->ijk", w[n, 0], w[n, 1], w[n, 2])
        ix = np.ix_(ind[n, 0], ind[n, 1], ind[n, 2])
        for c in range(3):
            np.add.at(g[c], ix, F[3 * n + c] * ker)
    return g


def wavenumbers(N, L):
    q = np.array([(i if i <= N // 2 else i - N) * (2.0 * PI / L) for i in range(N)])
    return q


def project(fh, N, dx, eta):
    nx, ny, nz = N
    qx = wavenumbers(nx, dx * nx)[:, None, None]
    qy = wavenumbers(ny, dx * ny)[None, :, None]
    qz = (np.arange(nz // 2 + 1) * (2.0 * PI / (dx * nz)))[None, None, :]
    G = float(nx * ny * nz)
    norm = 1.0 / (qy * qy + qx * qx + 1e-16 + qz * qz)
    kdotf = (qx * fh[0] + qy * fh[1] + qz * fh[2]) * norm
    u = np.stack([norm * (fh[0] - qx * kdotf) / (eta * G), norm * (fh[1] - qy * kdotf) / (eta * G),
                  norm * (fh[2] - qz * kdotf) / (eta * G)])
    u[:, 0, 0, 0] = 0.0
    return u


def inverse(uh, N):
    G = N[0] * N[1] * N[2]
    return np.fft.irfftn(uh, s=tuple(N), axes=(1, 2, 3)) * G


def interp(u, ind, w, dx):
    V = np.zeros(3 * len(ind))
    for n in range(len(ind)):
        ker = np.einsum("i,j,k->ijk", w[n, 0], w[n, 1], w[n, 2]) * dx ** 3
        ix = np.ix_(ind[n, 0], ind[n, 1], ind[n, 2])
        for c in range(3):
            V[3 * n + c] = np.sum(u[c][ix] * ker)
    return V


def mobility(Y, F, N, dx, a, eta, W):
    ind, w = gaussians(Y, N, dx, a, W)
    f = spread(F, ind, w, N)
    fh = np.fft.rfftn(f, axes=(1, 2, 3))
    fh[:, 0, 0, 0] = 0.0
    u = inverse(project(fh, N, dx, eta), N)
    return interp(u, ind, w, dx), ind, w


def random_velocity(Y, s6, N, dx, a, eta, W):
    """s6: real arrays sxx, syy, szz, sxy, sxz, syz of shape N."""
    nx, ny, nz = N
    sh = [np.fft.rfftn(s) for s in s6]
    sxx, syy, szz, sxy, sxz, syz = sh
    qx = wavenumbers(nx, dx * nx).copy()
    qy = wavenumbers(ny, dx * ny).copy()
    qz = np.arange(nz // 2 + 1) * (2.0 * PI / (dx * nz))
    qx[nx // 2] = 0.0
    qy[ny // 2] = 0.0
    qz[nz // 2] = 0.0
    q1 = qx[:, None, None]; q2 = qy[None, :, None]; q3 = qz[None, None, :]
    fx = 1j * (q1 * sxx + q2 * sxy + q3 * sxz)
    fy = 1j * (q1 * sxy + q2 * syy + q3 * syz)
    fz = 1j * (q1 * sxz + q2 * syz + q3 * szz)
    fh = np.stack([fx, fy, fz])
    fh[:, 0, 0, 0] = 0.0
    u = inverse(project(fh, N, dx, eta), N)
    ind, w = gaussians(Y, N, dx, a, W)
    return interp(u, ind, w, dx)


# ------------------------------------------------------------------ bodies
def quat_matrix(q):
    s, v = q[0], q[1:]
    R = np.eye(3)
    R[1, 1] -= 2 * v[0] * v[0]; R[2, 2] -= 2 * v[0] * v[0]
    R[0, 0] -= 2 * v[1] * v[1]; R[2, 2] -= 2 * v[1] * v[1]
    R[0, 0] -= 2 * v[2] * v[2]; R[1, 1] -= 2 * v[2] * v[2]
    R[1, 0] += 2 * v[0] * v[1]; R[0, 1] += 2 * v[0] * v[1]
    R[2, 0] += 2 * v[0] * v[2]; R[0, 2] += 2 * v[0] * v[2]
    R[1, 2] += 2 * v[1] * v[2]; R[2, 1] += 2 * v[1] * v[2]
    R[1, 0] += 2 * s * v[2]; R[0, 1] -= 2 * s * v[2]
    R[2, 0] -= 2 * s * v[1]; R[0, 2] += 2 * s * v[1]
    R[2, 1] += 2 * s * v[0]; R[1, 2] -= 2 * s * v[0]
    return R


def blob_positions(x, q, ref, L):
    M = len(x) // 3
    nb = len(ref) // 3
    Y = np.zeros((M * nb, 3))
    for n in range(M):
        R = quat_matrix(q[4 * n:4 * n + 4])
        for m in range(nb):
            p = x[3 * n:3 * n + 3] + R @ ref[3 * m:3 * m + 3]
            Y[n * nb + m] = p - L * np.floor(p / L)
    return Y


def mult_K(q, ref, U):
    M = len(q) // 4
    nb = len(ref) // 3
    out = np.zeros(3 * M * nb)
    for n in range(M):
        R = quat_matrix(q[4 * n:4 * n + 4])
        for m in range(nb):
            r = R @ ref[3 * m:3 * m + 3]
            out[3 * (n * nb + m):3 * (n * nb + m) + 3] = U[6 * n:6 * n + 3] + np.cross(U[6 * n + 3:6 * n + 6], r)
    return out


def mult_KT(q, ref, lam):
    M = len(q) // 4
    nb = len(ref) // 3
    out = np.zeros(6 * M)
    for n in range(M):
        R = quat_matrix(q[4 * n:4 * n + 4])
        for m in range(nb):
            r = R @ ref[3 * m:3 * m + 3]
            l = lam[3 * (n * nb + m):3 * (n * nb + m) + 3]
            out[6 * n:6 * n + 3] += l
            out[6 * n + 3:6 * n + 6] += np.cross(r, l)
    return out


def lie_exp(u):
    th = np.linalg.norm(u)
    if th < 1e-10:
        return np.array([1.0, 0, 0, 0])
    return np.concatenate([[math.cos(0.5 * th)], math.sin(0.5 * th) * u / th])


def qmul(a, b):
    return np.concatenate([[a[0] * b[0] - a[1:] @ b[1:]], a[0] * b[1:] + b[0] * a[1:] + np.cross(a[1:], b[1:])])


def body_update(x, q, U, scale, L):
    x = x.copy(); q = q.copy()
    M = len(x) // 3
    for n in range(M):
        u = scale * U[6 * n:6 * n + 6]
        x[3 * n:3 * n + 3] += u[:3]
        q[4 * n:4 * n + 4] = qmul(lie_exp(u[3:]), q[4 * n:4 * n + 4])
        x[3 * n:3 * n + 3] -= L * np.floor(x[3 * n:3 * n + 3] / L)
    return x, q


# ------------------------------------------------------------------ cells
def cell_ids(Y, L, Nc):
    c = np.floor(Nc * (Y / L)).astype(np.int64)
    return c[:, 0] + c[:, 1] * Nc + c[:, 2] * Nc * Nc, c


def pair_set(Y, L, Nc, nb):
    _, c = cell_ids(Y, L, Nc)
    pairs = []
    for i in range(len(Y)):
        for j in range(i + 1, len(Y)):
            if i // nb == j // nb:
                continue
            d = (c[i] - c[j]) % Nc
            if np.all((d == 0) | (d == 1) | (d == Nc - 1)):
                pairs.append((i, j))
    return np.array(pairs, dtype=np.int32).reshape(-1, 2)


def soft_sphere_force(r, a, kT):  # linked_list.cpp:415-419 (force branch)
    U0 = 20.0 * kT
    b = 0.5 * a
    return U0 / b if r < 2 * a else U0 * math.exp((2 * a - r) / b) / b


def steric(Y, pairs, L, a, kT):
    F = np.zeros(3 * len(Y))
    for i, j in pairs:
        d = Y[i] - Y[j]
        d = d - L * np.trunc(2.0 * d / L)
        r = math.sqrt(d @ d)
        m = soft_sphere_force(r, a, kT)
        F[3 * i:3 * i + 3] += m * d / r
        F[3 * j:3 * j + 3] -= m * d / r
    return F


def main():
    rng = np.random.default_rng(20241203)
    out = {}
    # FFT cases
    for tag, shape in (("a", (6, 8, 10)), ("b", (8, 6, 9))):
        r = rng.standard_normal(shape)
        out["fft_%s_in" % tag] = padded(r).ravel()
        out["fft_%s_fwd" % tag] = fft_transform(r).ravel()
        nzh = shape[2] // 2 + 1
        spec = np.zeros((shape[1], shape[0], 2 * nzh))
        spec[...] = rng.standard_normal(spec.shape)  # non-Hermitian input
        out["fft_%s_spec" % tag] = spec.ravel()
        out["fft_%s_inv" % tag] = fft_inverse(spec, shape).ravel()
    # mobility: 3 blobs, 16^3 grid, L = 16 (dx = 1), W = 8
    N = (16, 16, 16)
    dx, a, eta, W = 1.0, 1.0, 1.0, 8
    Y = rng.uniform(0.0, 16.0, (3, 3))
    F = rng.standard_normal(9)
    V, ind, w = mobility(Y, F, N, dx, a, eta, W)
    out.update(mobility_N=np.array(N), mobility_params=np.array([dx, a, eta, W]), mobility_Y=Y.ravel(),
               mobility_F=F, mobility_V=V, mobility_ind=ind.ravel(), mobility_w=w.ravel())
    # mobility on a non-cubic grid with an odd dimension
    N2 = (12, 16, 10)
    Y2 = rng.uniform(0.0, 1.0, (4, 3)) * np.array(N2) * 0.8
    F2 = rng.standard_normal(12)
    V2, _, _ = mobility(Y2, F2, N2, 0.8, a, 1.3, 6)
    out.update(mobility2_N=np.array(N2), mobility2_params=np.array([0.8, a, 1.3, 6]), mobility2_Y=Y2.ravel(),
               mobility2_F=F2, mobility2_V=V2)
    # random field from injected stress: 2 blobs on 12^3, dx = 1
    Nr = (12, 12, 12)
    Yr = rng.uniform(0.0, 12.0, (2, 3))
    s6 = [rng.standard_normal(Nr) for _ in range(6)]
    Vr = random_velocity(Yr, s6, Nr, 1.0, 1.0, 1.0, 8)
    out.update(random_N=np.array(Nr), random_Y=Yr.ravel(), random_V=Vr,
               random_s6=np.stack([padded(s).ravel() for s in s6]).ravel())
    # bodies: 5 rods of 3 blobs in L = 20
    Lb = 20.0
    ref = np.array([-2.2, 0, 0, 0, 0, 0, 2.2, 0.3, -0.1])
    xb = rng.uniform(0, Lb, 15)
    qb = rng.standard_normal((5, 4))
    qb = (qb / np.linalg.norm(qb, axis=1, keepdims=True)).ravel()
    Ub = rng.standard_normal(30)
    lam = rng.standard_normal(45)
    x2, q2 = body_update(xb, qb, Ub, 0.37, Lb)
    out.update(bodies_L=np.array([Lb]), bodies_ref=ref, bodies_x=xb, bodies_q=qb, bodies_U=Ub, bodies_lam=lam,
               bodies_Y=blob_positions(xb, qb, ref, Lb).ravel(), bodies_KU=mult_K(qb, ref, Ub),
               bodies_KTl=mult_KT(qb, ref, lam), bodies_x2=x2, bodies_q2=q2)
    # cells: 40 bodies of 2 blobs in L = 12 with 4 cells per dimension
    Lc, Nc, nbc = 12.0, 4, 2
    Yc = rng.uniform(0.0, Lc, (80, 3))
    cid, _ = cell_ids(Yc, Lc, Nc)
    pairs = pair_set(Yc, Lc, Nc, nbc)
    out.update(cells_L=np.array([Lc]), cells_Nc=np.array([Nc]), cells_nb=np.array([nbc]), cells_Y=Yc.ravel(),
               cells_ids=cid.astype(np.int32), cells_pairs=pairs, cells_F=steric(Yc, pairs, Lc, 1.0, 1.0))
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), sum(v.nbytes for v in out.values()), "bytes")


if __name__ == "__main__":
    main()
