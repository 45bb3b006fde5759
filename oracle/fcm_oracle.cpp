// fcm_oracle.cpp -- TEST INFRASTRUCTURE ONLY (the checker and the timed CPU
// baseline).  CPU FP64 restatement of the reference's FCM mobility path.
//
// Every function below cites the reference file:line it restates.  The MPI
// decomposition is collapsed to one rank: local_nx = nx, local_x_start = 0,
// local_ny_after_transpose = ny, local_y_start_after_transpose = 0 and every
// MPI_Allreduce is a copy.  Substitutions for libraries that are not available:
//   * FFTW 2.x rfftwnd_mpi  -> fft3_forward / fft3_inverse below (Stockham
//     mixed-radix FFT written for this file; same sign, scaling, in-place padded
//     layout and FFTW_TRANSPOSED_ORDER output as fft_solver.cpp:17-42).
//   * Armadillo / LAPACK    -> small dense helpers (Cholesky inverse for
//     inv_sympd, Gauss-Jordan with partial pivoting for inv).
//   * SPRNG                 -> Philox4x32-10 counter stream (Salmon et al.,
//     SC'11) feeding the reference's Marsaglia polar method
//     (parallel_random_numbers.cpp:8-19).
//   * compile-time macros   -> fcm_params fields.
// Parity status: "parity unpinned" against the reference's own outputs (the
// reference cannot be built here and ships no golden data); pinned by the
// known-answer tests in tests/test_oracle_*.py.
//
// Build: oracle/Makefile (g++ -O3 -fopenmp -ffp-contract=off).

#include "fcm_oracle.h"
#include "philox.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double PI = 3.14159265358979323846264338327950288;  // config.hpp:86
int g_threads = 1;

using orcrng::Philox;
using orcrng::UniformStream;

// ============================================================ 1-D complex FFT
// Stockham autosort, radices 4, 2, 3, 5 and generic odd primes, applied to `vb`
// interleaved lines at once: element j of lane b is at [j*vb + b] of separate
// re/im arrays.  Stage with radix p and Ns already-combined points:
//   v_r = x[j + r*n/p] * W_n^{r*(j mod Ns)*n/(Ns*p)},  V = DFT_p(v),
//   y[(j/Ns)*Ns*p + (j mod Ns) + s*Ns] = V_s.
struct Fft1 {
  int n = 0;
  std::vector<int> rad;
  std::vector<double> c, s;  // cos/sin(2*pi*j/n)
  void init(int n_) {
    n = n_;
    rad.clear();
    int m = n;
    while (m % 4 == 0) { rad.push_back(4); m /= 4; }
    while (m % 2 == 0) { rad.push_back(2); m /= 2; }
    for (int p = 3; m > 1; p += 2) {
      while (m % p == 0) { rad.push_back(p); m /= p; }
    }
    c.resize(n);
    s.resize(n);
    for (int j = 0; j < n; ++j) {
      c[j] = std::cos(2.0 * PI * (double)j / (double)n);
      s[j] = std::sin(2.0 * PI * (double)j / (double)n);
    }
  }
};

void fft1_run(const Fft1& P, double* re, double* im, double* tre, double* tim, int vb, int sign) {
  const int n = P.n;
  double *ir = re, *ii = im, *orr = tre, *oi = tim;
  int Ns = 1;
  std::vector<double> ar, ai, wr, wi;
  for (int p : P.rad) {
    const int m = n / p;
    const int tstep = n / (Ns * p);
    ar.assign(p, 0.0); ai.assign(p, 0.0); wr.assign(p, 0.0); wi.assign(p, 0.0);
    for (int j = 0; j < m; ++j) {
      const int k = j % Ns;
      const int base = (j / Ns) * Ns * p + k;
      for (int r = 0; r < p; ++r) {
        const int e = r * k * tstep;
        wr[r] = P.c[e];
        wi[r] = sign * P.s[e];
      }
      for (int b = 0; b < vb; ++b) {
        for (int r = 0; r < p; ++r) {
          const double xr = ir[(size_t)(j + r * m) * vb + b], xi = ii[(size_t)(j + r * m) * vb + b];
          ar[r] = xr * wr[r] - xi * wi[r];
          ai[r] = xr * wi[r] + xi * wr[r];
        }
        if (p == 2) {
          orr[(size_t)base * vb + b] = ar[0] + ar[1];
          oi[(size_t)base * vb + b] = ai[0] + ai[1];
          orr[(size_t)(base + Ns) * vb + b] = ar[0] - ar[1];
          oi[(size_t)(base + Ns) * vb + b] = ai[0] - ai[1];
        } else if (p == 4) {
          const double t0r = ar[0] + ar[2], t0i = ai[0] + ai[2];
          const double t1r = ar[0] - ar[2], t1i = ai[0] - ai[2];
          const double t2r = ar[1] + ar[3], t2i = ai[1] + ai[3];
          const double dr = ar[1] - ar[3], di = ai[1] - ai[3];
          // t3 = (a1 - a3) * (sign * i)
          const double t3r = -sign * di, t3i = sign * dr;
          orr[(size_t)base * vb + b] = t0r + t2r;
          oi[(size_t)base * vb + b] = t0i + t2i;
          orr[(size_t)(base + Ns) * vb + b] = t1r + t3r;
          oi[(size_t)(base + Ns) * vb + b] = t1i + t3i;
          orr[(size_t)(base + 2 * Ns) * vb + b] = t0r - t2r;
          oi[(size_t)(base + 2 * Ns) * vb + b] = t0i - t2i;
          orr[(size_t)(base + 3 * Ns) * vb + b] = t1r - t3r;
          oi[(size_t)(base + 3 * Ns) * vb + b] = t1i - t3i;
        } else {
          const int unit = n / p;
          for (int sidx = 0; sidx < p; ++sidx) {
            double sr = 0.0, si = 0.0;
            for (int r = 0; r < p; ++r) {
              const int e = ((r * sidx) % p) * unit;
              const double cr = P.c[e], ci = sign * P.s[e];
              sr += ar[r] * cr - ai[r] * ci;
              si += ar[r] * ci + ai[r] * cr;
            }
            orr[(size_t)(base + sidx * Ns) * vb + b] = sr;
            oi[(size_t)(base + sidx * Ns) * vb + b] = si;
          }
        }
      }
    }
    std::swap(ir, orr);
    std::swap(ii, oi);
    Ns *= p;
  }
  if (ir != re) {
    std::memcpy(re, ir, sizeof(double) * (size_t)n * vb);
    std::memcpy(im, ii, sizeof(double) * (size_t)n * vb);
  }
}

// ============================================================ 3-D real FFT
// fft_solver.cpp:17-42 with FFTW 2.x rfftwnd_mpi on one rank.  In place on a
// padded real array [x][y][pad], pad = 2*(nz/2+1); forward output is complex in
// FFTW_TRANSPOSED_ORDER [y][x][kz].  The inverse does complex inverse transforms
// along x and y, then a half-complex-to-real transform along z which, as FFTW's
// half-complex format stores no imaginary part for kz = 0 and kz = nz/2, ignores
// those imaginary parts.
struct Fft3 {
  int nx = 0, ny = 0, nz = 0, nzh = 0, pad = 0;
  Fft1 fx, fy, fz;
  std::vector<double> tmp;
  void init(int nx_, int ny_, int nz_) {
    nx = nx_; ny = ny_; nz = nz_;
    nzh = nz / 2 + 1;
    pad = 2 * nzh;  // fft_solver.cpp:26
    fx.init(nx); fy.init(ny); fz.init(nz);
    tmp.assign((size_t)nx * ny * pad, 0.0);
  }
  size_t total() const { return (size_t)nx * ny * pad; }
};

const int VB = 8;

// Complex transform along one axis of an interleaved complex array: line (o, i),
// element j at complex offset o*OS + j*S + i, i in [0, I).
void cpass(double* data, const Fft1& P, int O, size_t OS, size_t S, int I, int sign) {
  const int n = P.n;
  const int nchunks = (I + VB - 1) / VB;
  const long total = (long)O * nchunks;
#pragma omp parallel num_threads(g_threads)
  {
    std::vector<double> re((size_t)n * VB), im((size_t)n * VB), tre((size_t)n * VB), tim((size_t)n * VB);
#pragma omp for schedule(static)
    for (long t = 0; t < total; ++t) {
      const int o = (int)(t / nchunks), ch = (int)(t % nchunks);
      const int i0 = ch * VB, cnt = std::min(VB, I - i0);
      for (int j = 0; j < n; ++j) {
        const double* src = data + 2 * (o * OS + j * S + i0);
        for (int b = 0; b < VB; ++b) {
          if (b < cnt) {
            re[(size_t)j * VB + b] = src[2 * b];
            im[(size_t)j * VB + b] = src[2 * b + 1];
          } else {
            re[(size_t)j * VB + b] = 0.0;
            im[(size_t)j * VB + b] = 0.0;
          }
        }
      }
      fft1_run(P, re.data(), im.data(), tre.data(), tim.data(), VB, sign);
      for (int j = 0; j < n; ++j) {
        double* dst = data + 2 * (o * OS + j * S + i0);
        for (int b = 0; b < cnt; ++b) {
          dst[2 * b] = re[(size_t)j * VB + b];
          dst[2 * b + 1] = im[(size_t)j * VB + b];
        }
      }
    }
  }
}

// z-axis real-to-half-complex on every line of the padded real array; two real
// lines are packed into one complex transform.
void zpass_r2c(Fft3& F, double* a) {
  const int n = F.nz, nzh = F.nzh, pad = F.pad;
  const long nlines = (long)F.nx * F.ny;
  const long npairs = (nlines + 1) / 2;
  const long nchunks = (npairs + VB - 1) / VB;
#pragma omp parallel num_threads(g_threads)
  {
    std::vector<double> re((size_t)n * VB), im((size_t)n * VB), tre((size_t)n * VB), tim((size_t)n * VB);
#pragma omp for schedule(static)
    for (long ch = 0; ch < nchunks; ++ch) {
      for (int b = 0; b < VB; ++b) {
        const long p = ch * VB + b;
        const long l0 = 2 * p, l1 = 2 * p + 1;
        for (int j = 0; j < n; ++j) {
          re[(size_t)j * VB + b] = (l0 < nlines) ? a[l0 * pad + j] : 0.0;
          im[(size_t)j * VB + b] = (l1 < nlines) ? a[l1 * pad + j] : 0.0;
        }
      }
      fft1_run(F.fz, re.data(), im.data(), tre.data(), tim.data(), VB, -1);
      for (int b = 0; b < VB; ++b) {
        const long p = ch * VB + b;
        const long l0 = 2 * p, l1 = 2 * p + 1;
        for (int k = 0; k < nzh; ++k) {
          const int km = (n - k) % n;
          const double zr = re[(size_t)k * VB + b], zi = im[(size_t)k * VB + b];
          const double cr = re[(size_t)km * VB + b], ci = -im[(size_t)km * VB + b];  // conj Z(n-k)
          // A = (Z + conj Zm)/2 ; B = (Z - conj Zm)/(2i)
          const double Ar = 0.5 * (zr + cr), Ai = 0.5 * (zi + ci);
          const double dr = zr - cr, di = zi - ci;
          const double Br = 0.5 * di, Bi = -0.5 * dr;
          if (l0 < nlines) { tre[(size_t)k * VB + b] = Ar; tim[(size_t)k * VB + b] = Ai; }
          if (l1 < nlines) { a[l1 * pad + 2 * k] = Br; }
          // B's imaginary part is written after the loop (in-place hazard on l1
          // is impossible: l1's real input was already consumed above).
          if (l1 < nlines) { a[l1 * pad + 2 * k + 1] = Bi; }
        }
        if (l0 < nlines)
          for (int k = 0; k < nzh; ++k) {
            a[l0 * pad + 2 * k] = tre[(size_t)k * VB + b];
            a[l0 * pad + 2 * k + 1] = tim[(size_t)k * VB + b];
          }
      }
    }
  }
}

// z-axis half-complex-to-real on every line (imaginary parts of kz = 0 and, for
// even nz, kz = nz/2 are ignored, as in FFTW's half-complex format).
void zpass_c2r(Fft3& F, double* a) {
  const int n = F.nz, nzh = F.nzh, pad = F.pad;
  const long nlines = (long)F.nx * F.ny;
  const long npairs = (nlines + 1) / 2;
  const long nchunks = (npairs + VB - 1) / VB;
#pragma omp parallel num_threads(g_threads)
  {
    std::vector<double> re((size_t)n * VB), im((size_t)n * VB), tre((size_t)n * VB), tim((size_t)n * VB);
#pragma omp for schedule(static)
    for (long ch = 0; ch < nchunks; ++ch) {
      for (int b = 0; b < VB; ++b) {
        const long p = ch * VB + b;
        const long l0 = 2 * p, l1 = 2 * p + 1;
        for (int k = 0; k < n; ++k) {
          // Afull(k), Bfull(k) from the stored half spectra.
          double Ar = 0, Ai = 0, Br = 0, Bi = 0;
          int ks = k;
          double cj = 1.0;
          if (k >= nzh) { ks = n - k; cj = -1.0; }
          const bool real_only = (ks == 0) || (n % 2 == 0 && ks == n / 2);
          if (l0 < nlines) { Ar = a[l0 * pad + 2 * ks]; Ai = real_only ? 0.0 : cj * a[l0 * pad + 2 * ks + 1]; }
          if (l1 < nlines) { Br = a[l1 * pad + 2 * ks]; Bi = real_only ? 0.0 : cj * a[l1 * pad + 2 * ks + 1]; }
          // Z = A + i B
          re[(size_t)k * VB + b] = Ar - Bi;
          im[(size_t)k * VB + b] = Ai + Br;
        }
      }
      fft1_run(F.fz, re.data(), im.data(), tre.data(), tim.data(), VB, +1);
      for (int b = 0; b < VB; ++b) {
        const long p = ch * VB + b;
        const long l0 = 2 * p, l1 = 2 * p + 1;
        if (l0 < nlines) {
          for (int j = 0; j < n; ++j) a[l0 * pad + j] = re[(size_t)j * VB + b];
          for (int j = n; j < pad; ++j) a[l0 * pad + j] = 0.0;
        }
        if (l1 < nlines) {
          for (int j = 0; j < n; ++j) a[l1 * pad + j] = im[(size_t)j * VB + b];
          for (int j = n; j < pad; ++j) a[l1 * pad + j] = 0.0;
        }
      }
    }
  }
}

// [x][y][kz] <-> [y][x][kz] complex transposes.
void transpose_xy(Fft3& F, double* a, bool to_yx) {
  const int nx = F.nx, ny = F.ny, nzh = F.nzh;
  double* t = F.tmp.data();
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y) {
      const size_t xy = ((size_t)x * ny + y) * nzh * 2, yx = ((size_t)y * nx + x) * nzh * 2;
      if (to_yx) std::memcpy(t + yx, a + xy, sizeof(double) * 2 * nzh);
      else std::memcpy(t + xy, a + yx, sizeof(double) * 2 * nzh);
    }
  std::memcpy(a, t, sizeof(double) * F.total());
}

// fft_solver.cpp:32-36
void fft3_forward(Fft3& F, double* a) {
  zpass_r2c(F, a);
  cpass(a, F.fy, F.nx, (size_t)F.ny * F.nzh, F.nzh, F.nzh, -1);              // along y
  cpass(a, F.fx, 1, 0, (size_t)F.ny * F.nzh, F.ny * F.nzh, -1);              // along x
  transpose_xy(F, a, true);
}

// fft_solver.cpp:38-42
void fft3_inverse(Fft3& F, double* a) {
  transpose_xy(F, a, false);
  cpass(a, F.fx, 1, 0, (size_t)F.ny * F.nzh, F.ny * F.nzh, +1);
  cpass(a, F.fy, F.nx, (size_t)F.ny * F.nzh, F.nzh, F.nzh, +1);
  zpass_c2r(F, a);
}

// ============================================================ small dense algebra
// Column-major n x n helpers standing in for Armadillo / LAPACK.
typedef std::vector<double> Mat;  // col-major
inline double& at(Mat& A, int n, int i, int j) { return A[(size_t)j * n + i]; }
inline double atc(const Mat& A, int n, int i, int j) { return A[(size_t)j * n + i]; }

// inv(): Gauss-Jordan with partial pivoting.
bool dense_inv(const Mat& A, int n, Mat& out) {
  Mat a = A;
  out.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) at(out, n, i, i) = 1.0;
  for (int c = 0; c < n; ++c) {
    int piv = c;
    for (int r = c + 1; r < n; ++r)
      if (std::fabs(atc(a, n, r, c)) > std::fabs(atc(a, n, piv, c))) piv = r;
    if (atc(a, n, piv, c) == 0.0) return false;
    if (piv != c)
      for (int j = 0; j < n; ++j) { std::swap(at(a, n, c, j), at(a, n, piv, j)); std::swap(at(out, n, c, j), at(out, n, piv, j)); }
    const double d = atc(a, n, c, c);
    for (int j = 0; j < n; ++j) { at(a, n, c, j) /= d; at(out, n, c, j) /= d; }
    for (int r = 0; r < n; ++r) {
      if (r == c) continue;
      const double f = atc(a, n, r, c);
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) { at(a, n, r, j) -= f * atc(a, n, c, j); at(out, n, r, j) -= f * atc(out, n, c, j); }
    }
  }
  return true;
}

// inv_sympd(): Cholesky of the lower triangle, A^{-1} = L^{-T} L^{-1}, symmetric.
bool dense_inv_sympd(const Mat& A, int n, Mat& out) {
  Mat L((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double d = atc(A, n, j, j);
    for (int k = 0; k < j; ++k) d -= atc(L, n, j, k) * atc(L, n, j, k);
    if (!(d > 0.0)) return false;
    const double ljj = std::sqrt(d);
    at(L, n, j, j) = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = atc(A, n, i, j);
      for (int k = 0; k < j; ++k) s -= atc(L, n, i, k) * atc(L, n, j, k);
      at(L, n, i, j) = s / ljj;
    }
  }
  // Linv (lower triangular)
  Mat Li((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    at(Li, n, j, j) = 1.0 / atc(L, n, j, j);
    for (int i = j + 1; i < n; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s -= atc(L, n, i, k) * atc(Li, n, k, j);
      at(Li, n, i, j) = s / atc(L, n, i, i);
    }
  }
  out.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int k = i; k < n; ++k) s += atc(Li, n, k, i) * atc(Li, n, k, j);
      at(out, n, i, j) = s;
      at(out, n, j, i) = s;
    }
  return true;
}

// Cyclic Jacobi eigen-decomposition of a symmetric matrix (col-major).
void jacobi_eigen(Mat A, int n, std::vector<double>& evals, Mat& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) at(V, n, i, i) = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += atc(A, n, i, j) * atc(A, n, i, j);
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = atc(A, n, p, q);
        if (apq == 0.0) continue;
        const double theta = (atc(A, n, q, q) - atc(A, n, p, p)) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {
          const double akp = atc(A, n, k, p), akq = atc(A, n, k, q);
          at(A, n, k, p) = cs * akp - sn * akq;
          at(A, n, k, q) = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = atc(A, n, p, k), aqk = atc(A, n, q, k);
          at(A, n, p, k) = cs * apk - sn * aqk;
          at(A, n, q, k) = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = atc(V, n, k, p), vkq = atc(V, n, k, q);
          at(V, n, k, p) = cs * vkp - sn * vkq;
          at(V, n, k, q) = sn * vkp + cs * vkq;
        }
      }
  }
  evals.resize(n);
  for (int i = 0; i < n; ++i) evals[i] = atc(A, n, i, i);
}

// Armadillo's inv() for a well-conditioned symmetric matrix.  For the singular
// K^T K / K^T M^{-1} K of a body with collinear blobs (no reference body has
// them) the Moore-Penrose pseudo-inverse, dropping eigenvalues below 1e-10 of
// the largest.
bool sym_inv_or_pinv(const Mat& A, int n, Mat& out) {
  std::vector<double> ev;
  Mat V;
  jacobi_eigen(A, n, ev, V);
  double mx = 0.0;
  for (double e : ev) mx = std::max(mx, std::fabs(e));
  bool singular = !(mx > 0.0);
  for (double e : ev)
    if (std::fabs(e) <= 1e-10 * mx) singular = true;
  if (!singular) return dense_inv(A, n, out);
  out.assign((size_t)n * n, 0.0);
  for (int k = 0; k < n; ++k) {
    if (!(std::fabs(ev[k]) > 1e-10 * mx)) continue;
    const double inv = 1.0 / ev[k];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) at(out, n, i, j) += atc(V, n, i, k) * inv * atc(V, n, j, k);
  }
  return true;
}

// y = A x (col-major m x n)
void gemv(const Mat& A, int m, int n, const double* x, double* y) {
  for (int i = 0; i < m; ++i) y[i] = 0.0;
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < m; ++i) y[i] += A[(size_t)j * m + i] * x[j];
}
// y = A^T x (A col-major m x n, y has n entries)
void gemvT(const Mat& A, int m, int n, const double* x, double* y) {
  for (int j = 0; j < n; ++j) {
    double s = 0.0;
    for (int i = 0; i < m; ++i) s += A[(size_t)j * m + i] * x[i];
    y[j] = s;
  }
}

// ============================================================ quaternion / particle
struct Quat {
  double s, v[3];
};

// quaternion.cpp:61-103
void quat_matrix(const Quat& q, double R[3][3]) {
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) R[i][j] = (i == j) ? 1.0 : 0.0;
  double t = 2.0 * q.v[0] * q.v[0];
  R[1][1] -= t; R[2][2] -= t;
  t = 2.0 * q.v[1] * q.v[1];
  R[0][0] -= t; R[2][2] -= t;
  t = 2.0 * q.v[2] * q.v[2];
  R[0][0] -= t; R[1][1] -= t;
  t = 2.0 * q.v[0] * q.v[1];
  R[1][0] += t; R[0][1] += t;
  t = 2.0 * q.v[0] * q.v[2];
  R[2][0] += t; R[0][2] += t;
  t = 2.0 * q.v[1] * q.v[2];
  R[1][2] += t; R[2][1] += t;
  t = 2.0 * q.s * q.v[2];
  R[1][0] += t; R[0][1] -= t;
  t = 2.0 * q.s * q.v[1];
  R[2][0] -= t; R[0][2] += t;
  t = 2.0 * q.s * q.v[0];
  R[2][1] += t; R[1][2] -= t;
}

// quaternion.hpp:55-62 (q*p)
Quat quat_mul(const Quat& q, const Quat& p) {
  Quat o;
  o.s = q.s * p.s - (q.v[0] * p.v[0] + q.v[1] * p.v[1] + q.v[2] * p.v[2]);
  const double cx = q.v[1] * p.v[2] - q.v[2] * p.v[1];
  const double cy = q.v[2] * p.v[0] - q.v[0] * p.v[2];
  const double cz = q.v[0] * p.v[1] - q.v[1] * p.v[0];
  o.v[0] = q.s * p.v[0] + p.s * q.v[0] + cx;
  o.v[1] = q.s * p.v[1] + p.s * q.v[1] + cy;
  o.v[2] = q.s * p.v[2] + p.s * q.v[2] + cz;
  return o;
}

// quaternion.cpp:128-145
Quat lie_exp(const double u[3]) {
  const double theta = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
  Quat q;
  if (theta < 1e-10) {
    q.s = 1.0; q.v[0] = q.v[1] = q.v[2] = 0.0;
    return q;
  }
  const double cs = std::cos(0.5 * theta), sn = std::sin(0.5 * theta);
  q.s = cs;
  q.v[0] = sn * u[0] / theta;
  q.v[1] = sn * u[1] / theta;
  q.v[2] = sn * u[2] / theta;
  return q;
}

struct Body {
  double x[3];
  Quat q;
};

// particle.cpp:49-58 (update(grand_update))
void body_update(Body& b, const double u[6], const double L[3]) {
  b.x[0] += u[0]; b.x[1] += u[1]; b.x[2] += u[2];
  b.q = quat_mul(lie_exp(u + 3), b.q);
  for (int d = 0; d < 3; ++d) b.x[d] -= L[d] * std::floor(b.x[d] / L[d]);
}

inline void cross3(const double a[3], const double b[3], double c[3]) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
inline void matvec3(const double R[3][3], const double v[3], double o[3]) {
  for (int i = 0; i < 3; ++i) o[i] = R[i][0] * v[0] + R[i][1] * v[1] + R[i][2] * v[2];
}
inline void matTvec3(const double R[3][3], const double v[3], double o[3]) {
  for (int i = 0; i < 3; ++i) o[i] = R[0][i] * v[0] + R[1][i] * v[1] + R[2][i] * v[2];
}
// rcross.cpp:5-9 : rcross(x) = {{0,x2,-x1},{-x2,0,x0},{x1,-x0,0}}
inline void rcross(const double x[3], double C[3][3]) {
  C[0][0] = 0; C[0][1] = x[2]; C[0][2] = -x[1];
  C[1][0] = -x[2]; C[1][1] = 0; C[1][2] = x[0];
  C[2][0] = x[1]; C[2][1] = -x[0]; C[2][2] = 0;
}

}  // namespace

// ============================================================ the oracle object
struct orc {
  fcm_params p;
  int M, nb, Nb, Nx, Ny, Nz, W, pad;
  double DX, LX, LY, LZ, a, eta, kT, DT;
  size_t P;  // total_local_size
  Fft3 fft;
  // fcm_fluid_solver fields (fcm_fluid_solver.hpp:20-56)
  std::vector<double> ux, uy, uz, fx, fy, fz, sxx, syy, szz, sxy, sxz, syz;
  std::vector<double> V, Vtemp, ux_rand, uy_rand, uz_rand;
  // SHEARING_FORCES fields (fcm_fluid_solver.cpp:53-61): the imposed flow and its
  // blob velocities; shear is set once the flow has been produced
  std::vector<double> ux_shear, uy_shear, uz_shear, Vshear;
  bool shear = false;
  std::vector<double> qx, qxsq, qy, qysq, qpad, qpadsq;
  std::vector<double> gaussx, gaussy, gaussz;  // [np*W + i]
  std::vector<int> indx, indy, indz;
  int ngauss_rows = 0;
  std::vector<double> gauss_Y;  // the positions of the current Gaussian tables
  Mat ref_Minv, ref_N;
  // collection_of_rigid_bodies fields (collection_of_rigid_bodies.hpp:25-37)
  std::vector<double> blob_ref_pos;  // 3*nb
  std::vector<double> all_blob_pos;  // Nb*3
  Mat ref_KTKinv;
  // per-body shapes (no counterpart in the reference, whose bodies share
  // blob_ref_pos): 3*nb per body, and per body ref_KTKinv (36), ref_Minv
  // ((3nb)^2) and ref_N (36)
  bool per_body = false;
  std::vector<double> shapes, body_KTKinv, body_Minv, body_N;
  // noise from one sequential stream (orc_set_sequential_noise)
  bool seq_noise = false;
  UniformStream seq_rng{0, 0};
  std::vector<Body> bodies, midstep_bodies, temp_bodies;
  std::vector<double> blob_forces, ext_forces, U0;
  double body_radius = 0;
  // linked_list fields (linked_list.hpp:19-23)
  std::vector<int> head, list, map;
  int Nc;
  // gmres_solver fields (gmres_solver.hpp:22-29)
  int system_size;
  std::vector<double> RHS, Q, beta, H, SN, CS;
};

namespace {

// linked_list.cpp:13-21
int get_cell_id(const orc* o, int i, int j, int k) {
  const int N = o->Nc;
  const int imod = int(std::fmod(i + N, N));
  const int jmod = int(std::fmod(j + N, N));
  const int kmod = int(std::fmod(k + N, N));
  return imod + jmod * N + kmod * N * N;
}

// linked_list.cpp:74-78
int find_containing_cell(const orc* o, const double* Y) {
  const int N = o->Nc;
  double c = std::floor(N * (Y[0] / o->LX)) + std::floor(N * (Y[1] / o->LY)) * N +
             std::floor(N * (Y[2] / o->LZ)) * N * N;
  return (int)c;
}

// linked_list.cpp:362-497 (force magnitudes, non-MCMC branches) plus potential 3.
double interaction_magnitude(const orc* o, double r) {
  const double a = o->a, kT = o->kT;
  double magnitude = 0.0;
  if (o->p.potential == 3) {
    const double rc = o->p.steric_rc;
    if (r < rc) {
      const double t = (rc * rc - r * r) / (rc * rc - 4.0 * a * a);
      const double t2 = t * t;
      magnitude = o->p.steric_fs * t2 * t2;
    }
    return magnitude;
  }
  const double U0 = 20.0 * kT;
  const double b = 0.5 * a;
  magnitude = (r < 2.0 * a) ? U0 / b : U0 * std::exp((2.0 * a - r) / b) / b;
  if (o->p.potential == 1 || o->p.potential == 2) {
    const double A = 5.0 * kT, lambda = 0.5 * a;
    if (r < 2.0 * a) {
      double temp = a / lambda;
      temp = A * std::exp(-temp * temp);
      magnitude += 2.0 * a * temp / (lambda * lambda);
      if (o->p.potential == 2) {
        temp = 1.5 * a / lambda;
        temp = A * std::exp(-temp * temp);
        magnitude -= 3.0 * a * temp / (lambda * lambda);
      }
    } else {
      double temp = (r - 3.0 * a) / lambda;
      magnitude += -2.0 * A * temp * std::exp(-temp * temp) / lambda;
      if (o->p.potential == 2) {
        temp = (r - 3.5 * a) / lambda;
        magnitude += 2.0 * A * temp * std::exp(-temp * temp) / lambda;
      }
    }
  }
  return magnitude;
}

void list_initialise(orc* o) {  // linked_list.cpp:23-72 (one rank: my_start=0, my_end=N^3)
  const int N = o->Nc;
  const int total = N * N * N;
  o->head.assign(total, -1);
  o->list.assign(o->Nb, -1);
  o->map.assign(13 * total, 0);
  for (int i = 0; i < N; i++)
    for (int j = 0; j < N; j++)
      for (int k = 0; k < N; k++) {
        const int my_cell = get_cell_id(o, i, j, k);
        const int mp = 13 * my_cell;
        o->map[mp] = get_cell_id(o, i + 1, j, k);
        o->map[mp + 1] = get_cell_id(o, i + 1, j + 1, k);
        o->map[mp + 2] = get_cell_id(o, i, j + 1, k);
        o->map[mp + 3] = get_cell_id(o, i - 1, j + 1, k);
        o->map[mp + 4] = get_cell_id(o, i + 1, j, k - 1);
        o->map[mp + 5] = get_cell_id(o, i + 1, j + 1, k - 1);
        o->map[mp + 6] = get_cell_id(o, i, j + 1, k - 1);
        o->map[mp + 7] = get_cell_id(o, i - 1, j + 1, k - 1);
        o->map[mp + 8] = get_cell_id(o, i + 1, j, k + 1);
        o->map[mp + 9] = get_cell_id(o, i + 1, j + 1, k + 1);
        o->map[mp + 10] = get_cell_id(o, i, j + 1, k + 1);
        o->map[mp + 11] = get_cell_id(o, i - 1, j + 1, k + 1);
        o->map[mp + 12] = get_cell_id(o, i, j, k + 1);
      }
}

// Visit every inter-body pair exactly as linked_list.cpp:192-281 does: same cell
// (later in the list, raw difference), then the 13 half-shell cells
// (minimum image d - L*trunc(2d/L)).  fn(blob1, blob2, dx, dy, dz).
template <class Fn>
void list_visit(const orc* o, const std::vector<double>& Y, Fn fn) {
  const int N = o->Nc, total = N * N * N;
  const int bpb = o->nb;
  for (int i = 0; i < total; i++) {
    int blob1 = o->head[i];
    while (blob1 != -1) {
      const double x1 = Y[3 * blob1], y1 = Y[3 * blob1 + 1], z1 = Y[3 * blob1 + 2];
      const int body1 = blob1 / bpb;
      int blob2 = o->list[blob1];
      while (blob2 != -1) {
        const int body2 = blob2 / bpb;
        if (body1 != body2) fn(blob1, blob2, x1 - Y[3 * blob2], y1 - Y[3 * blob2 + 1], z1 - Y[3 * blob2 + 2]);
        blob2 = o->list[blob2];
      }
      for (int j = 0; j < 13; j++) {
        blob2 = o->head[o->map[13 * i + j]];
        while (blob2 != -1) {
          const int body2 = blob2 / bpb;
          if (body1 != body2) {
            const double x2 = Y[3 * blob2], y2 = Y[3 * blob2 + 1], z2 = Y[3 * blob2 + 2];
            const double xd = x1 - x2 - o->LX * std::trunc(2.0 * (x1 - x2) / o->LX);
            const double yd = y1 - y2 - o->LY * std::trunc(2.0 * (y1 - y2) / o->LY);
            const double zd = z1 - z2 - o->LZ * std::trunc(2.0 * (z1 - z2) / o->LZ);
            fn(blob1, blob2, xd, yd, zd);
          }
          blob2 = o->list[blob2];
        }
      }
      blob1 = o->list[blob1];
    }
  }
}

// Reference position of blob m of body n: the shared blob_ref_pos, or body n's own
// shape.
const double* ref_of(const orc* o, int n, int m) {
  return o->per_body ? &o->shapes[3 * ((size_t)n * o->nb + m)] : &o->blob_ref_pos[3 * m];
}

void blob_pos_of(const orc* o, const Body& b, int n, int m, double out[3]) {
  double R[3][3];
  quat_matrix(b.q, R);
  double r[3];
  matvec3(R, ref_of(o, n, m), r);
  const double Lv[3] = {o->LX, o->LY, o->LZ};
  for (int d = 0; d < 3; ++d) {
    const double pd = b.x[d] + r[d];
    out[d] = pd - Lv[d] * std::floor(pd / Lv[d]);
  }
}

void fill_pos(orc* o, const std::vector<Body>& bs) {  // collection_of_rigid_bodies.cpp:155-193
  for (int n = 0; n < o->M; n++)
    for (int m = 0; m < o->nb; m++) blob_pos_of(o, bs[n], n, m, &o->all_blob_pos[3 * (n * o->nb + m)]);
}

// fcm_fluid_solver.cpp:131-165
void set_up_gaussians(orc* o, const double* Y, int nrows) {
  const int W = o->W;
  const int ngdh = W / 2;
  const double anorm = 1.0 / (std::sqrt(2.0) * o->a);
  const double anorm2 = 2.0 * o->a * o->a / PI;
  const double DX = o->DX;
  o->ngauss_rows = nrows;
  o->gauss_Y.assign(Y, Y + 3 * (size_t)nrows);
  o->gaussx.assign((size_t)nrows * W, 0.0); o->gaussy.assign((size_t)nrows * W, 0.0); o->gaussz.assign((size_t)nrows * W, 0.0);
  o->indx.assign((size_t)nrows * W, 0); o->indy.assign((size_t)nrows * W, 0); o->indz.assign((size_t)nrows * W, 0);
  for (int np = 0; np < nrows; np++) {
    const int xc = int(Y[3 * np] / DX);
    const int yc = int(Y[3 * np + 1] / DX);
    const int zc = int(Y[3 * np + 2] / DX);
    for (int i = 0; i < W; i++) {
      int xg = xc - ngdh + (i + 1);
      o->indx[np * W + i] = xg - o->Nx * int(std::floor(double(xg) / double(o->Nx)));
      double xx = xg * DX - Y[3 * np];
      o->gaussx[np * W + i] = anorm * std::exp(-xx * xx / anorm2);
      int yg = yc - ngdh + (i + 1);
      o->indy[np * W + i] = yg - o->Ny * int(std::floor(double(yg) / double(o->Ny)));
      xx = yg * DX - Y[3 * np + 1];
      o->gaussy[np * W + i] = anorm * std::exp(-xx * xx / anorm2);
      int zg = zc - ngdh + (i + 1);
      o->indz[np * W + i] = zg - o->Nz * int(std::floor(double(zg) / double(o->Nz)));
      xx = zg * DX - Y[3 * np + 2];
      o->gaussz[np * W + i] = anorm * std::exp(-xx * xx / anorm2);
    }
  }
}

// Slip channel (fcm_fluid_solver.cpp:602-632, and :735-760 for the shear forcing):
// fy = 0 on the wall rows 0 and Ny/2; rows above Ny/2 become mirror images.
void slip_image(orc* o) {
  const int Nx = o->Nx, Ny = o->Ny, pad = o->pad, half_y = Ny / 2;
  for (int i = 0; i < Nx; i++) {
    const size_t x_index = (size_t)i * Ny * pad;
    for (int k = 0; k < pad; k++) {
      const size_t z_index = k;
      o->fy[x_index + z_index] = 0.0;
      o->fy[x_index + z_index + (size_t)half_y * pad] = 0.0;
      for (int j = 1 + half_y; j < Ny; j++) {
        const size_t index = x_index + z_index + (size_t)j * pad;
        const size_t image_index = x_index + z_index + (size_t)(Ny - j) * pad;
        o->fx[index] = o->fx[image_index];
        o->fy[index] = -o->fy[image_index];
        o->fz[index] = o->fz[image_index];
      }
    }
  }
}

// fcm_fluid_solver.cpp:552-632.  The x-slab loop mirrors the reference's per-rank
// slab filter (:568-570); with t threads each owns a slab, so every grid point sums
// its blobs in blob order.
void spread(orc* o, const double* F) {
  const size_t P = o->P;
  std::fill(o->fx.begin(), o->fx.end(), 0.0);
  std::fill(o->fy.begin(), o->fy.end(), 0.0);
  std::fill(o->fz.begin(), o->fz.end(), 0.0);
  const int W = o->W, Nx = o->Nx, Ny = o->Ny, pad = o->pad, nrows = o->ngauss_rows;
  (void)P;
#pragma omp parallel num_threads(g_threads)
  {
    int nt = 1, tid = 0;
#ifdef _OPENMP
    nt = omp_get_num_threads();
    tid = omp_get_thread_num();
#endif
    const int x0 = (int)((long)Nx * tid / nt), x1 = (int)((long)Nx * (tid + 1) / nt);
    for (int np = 0; np < nrows; np++) {
      for (int i = 0; i < W; i++) {
        const int ii = o->indx[np * W + i];
        if (ii < x0 || ii >= x1) continue;
        const size_t x_index = (size_t)ii * Ny * pad;
        for (int j = 0; j < W; j++) {
          const int jj = o->indy[np * W + j];
          const size_t y_index = (size_t)jj * pad;
          for (int k = 0; k < W; k++) {
            const int kk = o->indz[np * W + k];
            const size_t index = x_index + y_index + kk;
            const double temp = o->gaussx[np * W + i] * o->gaussy[np * W + j] * o->gaussz[np * W + k];
            const int id = 3 * np;
            o->fx[index] += F[id] * temp;
            o->fy[index] += F[id + 1] * temp;
            o->fz[index] += F[id + 2] * temp;
          }
        }
      }
    }
  }
  if (o->p.slip_channel) slip_image(o);
}

// fcm_fluid_solver.cpp:363-424 / :426-487 (interpolation of ux/uy/uz or u*_rand).
void interp(orc* o, const double* u1, const double* u2, const double* u3) {
  const int W = o->W, Ny = o->Ny, pad = o->pad, nrows = o->ngauss_rows;
  const double norm = o->DX * o->DX * o->DX;
  o->Vtemp.assign(3 * (size_t)nrows, 0.0);
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
  for (int np = 0; np < nrows; np++) {
    double v0 = 0, v1 = 0, v2 = 0;
    for (int i = 0; i < W; i++) {
      const int ii = o->indx[np * W + i];
      const size_t x_index = (size_t)ii * Ny * pad;
      for (int j = 0; j < W; j++) {
        const int jj = o->indy[np * W + j];
        if (o->p.slip_channel && jj >= Ny / 2) continue;  // truncated Gaussians (fcm_fluid_solver.cpp:387-389)
        const size_t y_index = (size_t)jj * pad;
        for (int k = 0; k < W; k++) {
          const int kk = o->indz[np * W + k];
          const size_t index = x_index + y_index + kk;
          const double temp = o->gaussx[np * W + i] * o->gaussy[np * W + j] * o->gaussz[np * W + k] * norm;
          v0 += u1[index] * temp;
          v1 += u2[index] * temp;
          v2 += u3[index] * temp;
        }
      }
    }
    o->Vtemp[3 * np] = v0;
    o->Vtemp[3 * np + 1] = v1;
    o->Vtemp[3 * np + 2] = v2;
  }
  o->V = o->Vtemp;  // MPI_Allreduce on one rank
}

// The k-space projection shared by fcm_fluid_solver.cpp:307-336 and :655-684,
// reading (fx,fy,fz) and writing (ux,uy,uz) in transposed order.
void project(orc* o) {
  const int Nx = o->Nx, Ny = o->Ny, pad = o->pad;
  const double totalpts = double(o->Nx) * double(o->Ny) * double(o->Nz);
  const double eta = o->eta;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int j = 0; j < Ny; j++) {
    const double q2 = o->qy[j];
    const size_t y_index = (size_t)j * Nx * pad;
    for (int i = 0; i < Nx; i++) {
      const double q1 = o->qx[i];
      const double qq = o->qysq[j] + o->qxsq[i] + 1e-16;
      const size_t x_index = (size_t)i * pad;
      for (int k = 0; k < pad; k++) {
        const size_t index = x_index + y_index + k;
        const double q3 = o->qpad[k];
        const double f1 = o->fx[index], f2 = o->fy[index], f3 = o->fz[index];
        const double norm = 1.0 / (qq + o->qpadsq[k]);
        const double kdotf = (q1 * f1 + q2 * f2 + q3 * f3) * norm;
        o->ux[index] = norm * (f1 - q1 * (kdotf)) / (eta * totalpts);
        o->uy[index] = norm * (f2 - q2 * (kdotf)) / (eta * totalpts);
        o->uz[index] = norm * (f3 - q3 * (kdotf)) / (eta * totalpts);
      }
    }
  }
  // fcm_fluid_solver.cpp:338-347 / :686-695
  o->ux[0] = o->ux[1] = 0.0;
  o->uy[0] = o->uy[1] = 0.0;
  o->uz[0] = o->uz[1] = 0.0;
}

// fcm_fluid_solver.cpp:636-701
void produce_deterministic_velocity_field(orc* o) {
  fft3_forward(o->fft, o->fx.data());
  fft3_forward(o->fft, o->fy.data());
  fft3_forward(o->fft, o->fz.data());
  o->fx[0] = o->fx[1] = 0.0;
  o->fy[0] = o->fy[1] = 0.0;
  o->fz[0] = o->fz[1] = 0.0;
  project(o);
  fft3_inverse(o->fft, o->ux.data());
  fft3_inverse(o->fft, o->uy.data());
  fft3_inverse(o->fft, o->uz.data());
}

// fcm_fluid_solver.cpp:236-361 on the stress arrays already filled.
void random_field_from_stress(orc* o) {
  fft3_forward(o->fft, o->sxx.data());
  fft3_forward(o->fft, o->sxy.data());
  fft3_forward(o->fft, o->sxz.data());
  fft3_forward(o->fft, o->syy.data());
  fft3_forward(o->fft, o->szz.data());
  fft3_forward(o->fft, o->syz.data());
  const int Nx = o->Nx, Ny = o->Ny, pad = o->pad;
#pragma omp parallel for num_threads(g_threads) schedule(static)
  for (int j = 0; j < Ny; j++) {
    double q2 = o->qy[j];
    if (j == Ny / 2) q2 = 0.0;
    const size_t y_index = (size_t)j * Nx * pad;
    for (int i = 0; i < Nx; i++) {
      double q1 = o->qx[i];
      if (i == Nx / 2) q1 = 0.0;
      const size_t x_index = (size_t)i * pad;
      for (int k = 0; k < pad; k = k + 2) {
        const size_t index = x_index + y_index + k;
        const size_t index_plus_one = index + 1;
        double q3 = o->qpad[k];
        if (k == pad - 2) q3 = 0.0;
        const std::vector<double>&sxx = o->sxx, &sxy = o->sxy, &sxz = o->sxz, &syy = o->syy, &szz = o->szz, &syz = o->syz;
        o->fx[index] = -q1 * sxx[index_plus_one] - q2 * sxy[index_plus_one] - q3 * sxz[index_plus_one];
        o->fy[index] = -q1 * sxy[index_plus_one] - q2 * syy[index_plus_one] - q3 * syz[index_plus_one];
        o->fz[index] = -q1 * sxz[index_plus_one] - q2 * syz[index_plus_one] - q3 * szz[index_plus_one];
        o->fx[index_plus_one] = q1 * sxx[index] + q2 * sxy[index] + q3 * sxz[index];
        o->fy[index_plus_one] = q1 * sxy[index] + q2 * syy[index] + q3 * syz[index];
        o->fz[index_plus_one] = q1 * sxz[index] + q2 * syz[index] + q3 * szz[index];
      }
    }
  }
  o->fx[0] = o->fx[1] = 0.0;
  o->fy[0] = o->fy[1] = 0.0;
  o->fz[0] = o->fz[1] = 0.0;
  project(o);
  fft3_inverse(o->fft, o->ux.data());
  fft3_inverse(o->fft, o->uy.data());
  fft3_inverse(o->fft, o->uz.data());
  o->ux_rand = o->ux;
  o->uy_rand = o->uy;
  o->uz_rand = o->uz;
}

// collection_of_rigid_bodies.cpp:707-731
void mult_K(const orc* o, const double* in, double* out) {
  for (int i = 0; i < 3 * o->Nb; ++i) out[i] = 0.0;
  for (int i = 0; i < o->M; i++) {
    const int ipos = 6 * i;
    double R[3][3];
    quat_matrix(o->midstep_bodies[i].q, R);
    for (int j = 0; j < o->nb; j++) {
      const int jpos = 3 * (o->nb * i + j);
      double r[3], c[3];
      matvec3(R, ref_of(o, i, j), r);
      cross3(in + ipos + 3, r, c);
      for (int d = 0; d < 3; ++d) out[jpos + d] += in[ipos + d] + c[d];
    }
  }
}

// collection_of_rigid_bodies.cpp:733-757
void mult_KT(const orc* o, const double* in, double* out) {
  for (int i = 0; i < 6 * o->M; ++i) out[i] = 0.0;
  for (int i = 0; i < o->M; i++) {
    const int ipos = 6 * i;
    double R[3][3];
    quat_matrix(o->midstep_bodies[i].q, R);
    for (int j = 0; j < o->nb; j++) {
      const int jpos = 3 * (o->nb * i + j);
      double r[3], c[3];
      matvec3(R, ref_of(o, i, j), r);
      cross3(r, in + jpos, c);
      for (int d = 0; d < 3; ++d) {
        out[ipos + d] += in[jpos + d];
        out[ipos + 3 + d] += c[d];
      }
    }
  }
}

// Rigid projection of blob velocities V onto body n's motion with ref_KTKinv,
// as collection_of_rigid_bodies.cpp:580-600 and :909-939.
void rigid_projection(const orc* o, const Body& body, int n, const double* V, double U[6]) {
  double b[6] = {0, 0, 0, 0, 0, 0};
  double Q[3][3];
  quat_matrix(body.q, Q);
  for (int i = 0; i < o->nb; i++) {
    const int id = n * o->nb + i;
    const double* vel = V + 3 * id;
    double r[3], c[3];
    matvec3(Q, ref_of(o, n, i), r);
    cross3(r, vel, c);
    for (int d = 0; d < 3; ++d) { b[d] += vel[d]; b[3 + d] += c[d]; }
  }
  double bt[6];
  matTvec3(Q, b, bt);
  matTvec3(Q, b + 3, bt + 3);
  double u[6];
  if (o->per_body) {
    const Mat KTKinv(o->body_KTKinv.begin() + 36 * (size_t)n, o->body_KTKinv.begin() + 36 * (size_t)(n + 1));
    gemv(KTKinv, 6, 6, bt, u);
  } else {
    gemv(o->ref_KTKinv, 6, 6, bt, u);
  }
  matvec3(Q, u, U);
  matvec3(Q, u + 3, U + 3);
}

// gmres_solver.cpp:85-146
void mult_Pinv(const orc* o, const double* in, double* out) {
  const int nb = o->nb, n3 = 3 * nb, Nb = o->Nb;
  Mat K((size_t)n3 * 6, 0.0);
  for (int m = 0; m < nb; m++)
    for (int d = 0; d < 3; ++d) K[(size_t)d * n3 + 3 * m + d] = 1.0;
  for (int n = 0; n < o->M; n++) {
    double Q[3][3];
    quat_matrix(o->midstep_bodies[n].q, Q);
    for (int m = 0; m < nb; m++) {
      double r[3], C[3][3];
      matvec3(Q, ref_of(o, n, m), r);
      rcross(r, C);
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) K[(size_t)(3 + j) * n3 + 3 * m + i] = C[i][j];
    }
    // the body's own blocks with per-body shapes
    const size_t mm = (size_t)n3 * n3;
    const Mat ref_Minv = o->per_body ? Mat(o->body_Minv.begin() + mm * n, o->body_Minv.begin() + mm * (n + 1))
                                     : o->ref_Minv;
    const Mat ref_N = o->per_body ? Mat(o->body_N.begin() + 36 * (size_t)n, o->body_N.begin() + 36 * (size_t)(n + 1))
                                  : o->ref_N;
    Mat Minv = ref_Minv;
    Mat N = ref_N;
    auto rot_block = [&](Mat& A, int lda, int r0, int c0, const Mat& src) {
      // A(r0:r0+2, c0:c0+2) = Q * src(r0.., c0..) * Q^T
      double B[3][3], T[3][3];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) B[i][j] = src[(size_t)(c0 + j) * lda + r0 + i];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[i][j] = Q[i][0] * B[0][j] + Q[i][1] * B[1][j] + Q[i][2] * B[2][j];
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[(size_t)(c0 + j) * lda + r0 + i] = T[i][0] * Q[j][0] + T[i][1] * Q[j][1] + T[i][2] * Q[j][2];
    };
    for (int m = 0; m < nb; m++)
      for (int l = m; l < nb; l++) {
        rot_block(Minv, n3, 3 * m, 3 * l, ref_Minv);
        for (int i = 0; i < 3; ++i)
          for (int j = 0; j < 3; ++j) Minv[(size_t)(3 * m + j) * n3 + 3 * l + i] = Minv[(size_t)(3 * l + i) * n3 + 3 * m + j];
      }
    rot_block(N, 6, 0, 0, ref_N);
    rot_block(N, 6, 0, 3, ref_N);
    rot_block(N, 6, 3, 0, ref_N);
    rot_block(N, 6, 3, 3, ref_N);
    const double* in_l = in + (size_t)n3 * n;
    const double* in_U = in + (size_t)3 * Nb + 6 * n;
    std::vector<double> t(n3), t2(n3);
    double u[6], u2[6];
    gemv(Minv, n3, n3, in_l, t.data());
    gemvT(K, n3, 6, t.data(), u);
    for (int d = 0; d < 6; ++d) u[d] = -in_U[d] - u[d];
    gemv(N, 6, 6, u, u2);
    double* out_U = out + (size_t)3 * Nb + 6 * n;
    for (int d = 0; d < 6; ++d) out_U[d] = u2[d];
    gemv(K, n3, 6, u2, t.data());
    for (int d = 0; d < n3; ++d) t[d] += in_l[d];
    gemv(Minv, n3, n3, t.data(), t2.data());
    for (int d = 0; d < n3; ++d) out[(size_t)n3 * n + d] = t2[d];
  }
}

// gmres_solver.cpp:72-83
void mult_A(orc* o, const double* in, double* out) {
  const int Nb = o->Nb;
  spread(o, in);
  produce_deterministic_velocity_field(o);
  interp(o, o->ux.data(), o->uy.data(), o->uz.data());
  std::vector<double> kU(3 * Nb), ktl(6 * o->M);
  mult_K(o, in + 3 * Nb, kU.data());
  mult_KT(o, in, ktl.data());
  for (int i = 0; i < 3 * Nb; ++i) out[i] = o->V[i] - kU[i];
  for (int i = 0; i < 6 * o->M; ++i) out[3 * Nb + i] = -ktl[i];
}

// gmres_solver.cpp:148-306
int gmres(orc* o, double* soln_out, int* iters_out, double* rel_out) {
  const int n = o->system_size;
  const int max_iter = std::min(n, o->p.gmres_max_iter);
  const double tol = o->p.gmres_tol;
  o->Q.assign((size_t)n * (max_iter + 1), 0.0);
  o->beta.assign(max_iter + 1, 0.0);
  o->H.assign((size_t)(max_iter + 1) * (max_iter + 1), 0.0);
  o->CS.assign(max_iter, 0.0);
  o->SN.assign(max_iter, 0.0);
  const int hn = max_iter + 1;
  auto Hm = [&](int i, int j) -> double& { return o->H[(size_t)j * hn + i]; };
  auto Qc = [&](int c) { return o->Q.data() + (size_t)c * n; };
  double nrm = 0.0;
  for (int i = 0; i < n; ++i) nrm += o->RHS[i] * o->RHS[i];
  const double norm_of_RHS = std::sqrt(nrm);
  if (!(norm_of_RHS > 0.0)) {
    if (soln_out) std::fill(soln_out, soln_out + n, 0.0);
    if (iters_out) *iters_out = 0;
    if (rel_out) *rel_out = 0.0;
    return norm_of_RHS == 0.0 ? 0 : FCM_ERR_NONFINITE;
  }
  for (int i = 0; i < n; ++i) Qc(0)[i] = o->RHS[i] / norm_of_RHS;
  o->beta[0] = norm_of_RHS;
  std::vector<double> z(n);
  for (int iter = 1; iter <= max_iter; iter++) {
    mult_Pinv(o, Qc(iter - 1), z.data());
    mult_A(o, z.data(), Qc(iter));
    for (int i = 0; i < iter; i++) {
      double d = 0.0;
      for (int t = 0; t < n; ++t) d += Qc(iter)[t] * Qc(i)[t];
      Hm(i, iter - 1) = d;
      for (int t = 0; t < n; ++t) Qc(iter)[t] -= d * Qc(i)[t];
    }
    double qn = 0.0;
    for (int t = 0; t < n; ++t) qn += Qc(iter)[t] * Qc(iter)[t];
    const double q_norm = std::sqrt(qn);
    Hm(iter, iter - 1) = q_norm;
    if (q_norm != 0.0)
      for (int t = 0; t < n; ++t) Qc(iter)[t] /= q_norm;
    for (int i = 1; i < iter; i++) {
      const double temp = o->CS[i - 1] * Hm(i - 1, iter - 1) + o->SN[i - 1] * Hm(i, iter - 1);
      Hm(i, iter - 1) = o->CS[i - 1] * Hm(i, iter - 1) - o->SN[i - 1] * Hm(i - 1, iter - 1);
      Hm(i - 1, iter - 1) = temp;
    }
    if (Hm(iter, iter - 1) == 0.0) {
      o->CS[iter - 1] = 1.0;
      o->SN[iter - 1] = 0.0;
    } else {
      if (std::fabs(Hm(iter, iter - 1)) > std::fabs(Hm(iter - 1, iter - 1))) {
        const double temp = Hm(iter - 1, iter - 1) / Hm(iter, iter - 1);
        o->SN[iter - 1] = (2.0 * double(Hm(iter, iter - 1) > 0) - 1.0) / std::sqrt(1.0 + temp * temp);
        o->CS[iter - 1] = temp * o->SN[iter - 1];
      } else {
        const double temp = Hm(iter, iter - 1) / Hm(iter - 1, iter - 1);
        o->CS[iter - 1] = (2.0 * double(Hm(iter - 1, iter - 1) > 0) - 1.0) / std::sqrt(1.0 + temp * temp);
        o->SN[iter - 1] = temp * o->CS[iter - 1];
      }
    }
    Hm(iter - 1, iter - 1) = o->CS[iter - 1] * Hm(iter - 1, iter - 1) + o->SN[iter - 1] * Hm(iter, iter - 1);
    Hm(iter, iter - 1) = 0.0;
    o->beta[iter] = -o->SN[iter - 1] * o->beta[iter - 1];
    o->beta[iter - 1] = o->CS[iter - 1] * o->beta[iter - 1];
    const double relative_error = std::fabs(o->beta[iter]) / norm_of_RHS;
    if ((relative_error < tol) || (iter == max_iter)) {
      std::vector<double> y(iter, 0.0);
      y[iter - 1] = o->beta[iter - 1] / Hm(iter - 1, iter - 1);
      for (int i = iter - 2; i >= 0; i--) {
        y[i] = o->beta[i];
        for (int j = iter - 1; j > i; j--) y[i] -= Hm(i, j) * y[j];
        y[i] /= Hm(i, i);
      }
      std::vector<double> soln(n, 0.0);
      for (int i = 0; i < iter; i++)
        for (int t = 0; t < n; ++t) soln[t] += y[i] * Qc(i)[t];
      std::vector<double> x(n);
      mult_Pinv(o, soln.data(), x.data());
      if (soln_out) std::copy(x.begin(), x.end(), soln_out);
      if (iters_out) *iters_out = iter;
      if (rel_out) *rel_out = relative_error;
      if (!std::isfinite(relative_error)) return FCM_ERR_NONFINITE;
      return (relative_error < tol) ? 0 : FCM_ERR_NOT_CONVERGED;
    }
  }
  return FCM_ERR_STATE;
}

void calculate_forces(orc* o) {  // collection_of_rigid_bodies.cpp:623-664
  if (o->p.algorithm == 2) o->midstep_bodies = o->bodies;
  orc_list_populate(o);
  std::fill(o->blob_forces.begin(), o->blob_forces.end(), 0.0);
  orc_apply_barrier_forces(o, o->blob_forces.data());
  if (o->p.slip_channel) {  // :640-662
    const double L = 2.2 * o->a;
    const double K = (40.0 * o->kT / o->a) / L;
    for (int i = 0; i < o->Nb; i++) {
      const double y = o->all_blob_pos[3 * i + 1];
      if (y <= L) {
        o->blob_forces[3 * i + 1] += K * (L - y);
      } else if ((0.5 * o->LY - y <= L) && (y <= 0.5 * o->LY)) {
        o->blob_forces[3 * i + 1] -= K * (L - 0.5 * o->LY + y);
      }
    }
  }
}

// collection_of_rigid_bodies.cpp:207-239
int wall_overlap(const orc* o) {
  if (!o->p.slip_channel) return 0;
  for (int n = 0; n < o->Nb; n++) {
    const double y = o->all_blob_pos[3 * n + 1];
    if ((y == 0.0) || (y >= 0.5 * o->LY)) return 1;
  }
  return 0;
}

}  // namespace

// ============================================================ C API
extern "C" {

void orc_set_threads(int n) { g_threads = n > 0 ? n : 1; }
int orc_get_threads(void) { return g_threads; }

int orc_fft_transform(int nx, int ny, int nz, double* in) {
  Fft3 F;
  F.init(nx, ny, nz);
  fft3_forward(F, in);
  return 0;
}
int orc_fft_inverse_transform(int nx, int ny, int nz, double* in) {
  Fft3 F;
  F.init(nx, ny, nz);
  fft3_inverse(F, in);
  return 0;
}

orc* orc_create(const fcm_params* p, const double* ref) {
  if (!p || p->ncells < 3) return nullptr;
  orc* o = new orc();
  o->p = *p;
  o->M = p->num_bodies; o->nb = p->blobs_per_body; o->Nb = o->M * o->nb;
  o->Nx = p->nx; o->Ny = p->ny; o->Nz = p->nz; o->W = p->ngauss;
  o->DX = p->dx; o->LX = p->dx * p->nx; o->LY = p->dx * p->ny; o->LZ = p->dx * p->nz;
  o->a = p->blob_radius; o->eta = p->viscosity; o->kT = p->kT; o->DT = p->dt;
  o->Nc = p->ncells;
  o->fft.init(o->Nx, o->Ny, o->Nz);
  o->pad = o->fft.pad;
  o->P = o->fft.total();
  for (auto* v : {&o->ux, &o->uy, &o->uz, &o->fx, &o->fy, &o->fz, &o->sxx, &o->syy, &o->szz, &o->sxy, &o->sxz, &o->syz, &o->ux_rand, &o->uy_rand, &o->uz_rand})
    v->assign(o->P, 0.0);
  o->V.assign(3 * (size_t)o->Nb, 0.0);
  o->Vshear.assign(3 * (size_t)o->Nb, 0.0);
  // fcm_fluid_solver.cpp:71-127 wavenumber tables
  auto qtab = [](int N, double L, std::vector<double>& q, std::vector<double>& qsq) {
    q.resize(N); qsq.resize(N);
    const int nptsh = N / 2;
    const double fourier_fac = 2.0 * PI / L;
    for (int i = 0; i < N; i++) {
      q[i] = (i <= nptsh) ? i * fourier_fac : (i - N) * fourier_fac;
      qsq[i] = q[i] * q[i];
    }
  };
  qtab(o->Nx, o->LX, o->qx, o->qxsq);
  qtab(o->Ny, o->LY, o->qy, o->qysq);
  o->qpad.resize(o->pad); o->qpadsq.resize(o->pad);
  const double ffz = 2.0 * PI / o->LZ;
  for (int i = 0; i < o->pad; i += 2) {
    o->qpad[i] = 0.5 * i * ffz;
    o->qpad[i + 1] = o->qpad[i];
    o->qpadsq[i] = o->qpad[i] * o->qpad[i];
    o->qpadsq[i + 1] = o->qpadsq[i];
  }
  // collection_of_rigid_bodies.cpp:15-153 (geometry supplied by the caller)
  o->blob_ref_pos.assign(ref, ref + 3 * o->nb);
  o->all_blob_pos.assign(3 * (size_t)o->Nb, 0.0);
  o->blob_forces.assign(3 * (size_t)o->Nb, 0.0);
  o->ext_forces.assign(6 * (size_t)o->M, 0.0);
  o->U0.assign(6 * (size_t)o->M, 0.0);
  Body b0;
  b0.x[0] = b0.x[1] = b0.x[2] = 0.0;
  b0.q.s = 1.0; b0.q.v[0] = b0.q.v[1] = b0.q.v[2] = 0.0;
  o->bodies.assign(o->M, b0);
  o->midstep_bodies = o->bodies;
  o->temp_bodies = o->bodies;
  for (int i = 0; i < o->nb; i++) {
    const double* r = &o->blob_ref_pos[3 * i];
    o->body_radius = std::max(o->body_radius, std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]));
  }
  {
    const int n3 = 3 * o->nb;
    Mat K((size_t)n3 * 6, 0.0);
    for (int m = 0; m < o->nb; m++) {
      double C[3][3];
      rcross(&o->blob_ref_pos[3 * m], C);
      for (int d = 0; d < 3; ++d) K[(size_t)d * n3 + 3 * m + d] = 1.0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) K[(size_t)(3 + j) * n3 + 3 * m + i] = C[i][j];
    }
    Mat KTK(36, 0.0);
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        double s = 0.0;
        for (int t = 0; t < n3; ++t) s += K[(size_t)i * n3 + t] * K[(size_t)j * n3 + t];
        KTK[(size_t)j * 6 + i] = s;
      }
    sym_inv_or_pinv(KTK, 6, o->ref_KTKinv);  // collection_of_rigid_bodies.cpp:128
  }
  list_initialise(o);
  o->system_size = 3 * o->Nb + 6 * o->M;  // gmres_solver.cpp:18
  o->RHS.assign(o->system_size, 0.0);
  o->ref_Minv.assign((size_t)9 * o->nb * o->nb, 0.0);
  for (int i = 0; i < 3 * o->nb; ++i) o->ref_Minv[(size_t)i * 3 * o->nb + i] = 1.0;
  o->ref_N.assign(36, 0.0);
  for (int i = 0; i < 6; ++i) o->ref_N[i * 6 + i] = 1.0;
  return o;
}

void orc_destroy(orc* o) { delete o; }

void orc_set_bodies(orc* o, const double* x, const double* q) {
  for (int n = 0; n < o->M; ++n) {
    for (int d = 0; d < 3; ++d) o->bodies[n].x[d] = x[3 * n + d];
    o->bodies[n].q.s = q[4 * n];
    for (int d = 0; d < 3; ++d) o->bodies[n].q.v[d] = q[4 * n + 1 + d];
  }
  o->midstep_bodies = o->bodies;
}
static void get_b(const std::vector<Body>& bs, int M, double* x, double* q) {
  for (int n = 0; n < M; ++n) {
    for (int d = 0; d < 3; ++d) x[3 * n + d] = bs[n].x[d];
    q[4 * n] = bs[n].q.s;
    for (int d = 0; d < 3; ++d) q[4 * n + 1 + d] = bs[n].q.v[d];
  }
}
void orc_get_bodies(orc* o, double* x, double* q) { get_b(o->bodies, o->M, x, q); }
void orc_get_midstep_bodies(orc* o, double* x, double* q) { get_b(o->midstep_bodies, o->M, x, q); }
void orc_set_external_forces(orc* o, const double* fe) {
  if (fe) o->ext_forces.assign(fe, fe + 6 * o->M);
  else std::fill(o->ext_forces.begin(), o->ext_forces.end(), 0.0);
}
void orc_fill_all_blob_pos(orc* o, int at_midstep) { fill_pos(o, at_midstep ? o->midstep_bodies : o->bodies); }
void orc_set_all_blob_pos(orc* o, const double* Y) { o->all_blob_pos.assign(Y, Y + 3 * o->Nb); }
void orc_get_all_blob_pos(orc* o, double* Y) { std::copy(o->all_blob_pos.begin(), o->all_blob_pos.end(), Y); }
void orc_multiply_by_K_at_midstep(orc* o, const double* in, double* out) { mult_K(o, in, out); }
void orc_multiply_by_KT_at_midstep(orc* o, const double* in, double* out) { mult_KT(o, in, out); }
void orc_calculate_forces(orc* o) { calculate_forces(o); }
void orc_get_blob_forces(orc* o, double* F) { std::copy(o->blob_forces.begin(), o->blob_forces.end(), F); }
void orc_set_blob_forces(orc* o, const double* F) { o->blob_forces.assign(F, F + 3 * o->Nb); }

// collection_of_rigid_bodies.cpp:566-621
int orc_advance_to_midstep(orc* o, const double* V) {
  const double* Vv = V ? V : o->V.data();
  o->midstep_bodies = o->bodies;
  const double Lv[3] = {o->LX, o->LY, o->LZ};
  for (int n = 0; n < o->M; n++) {
    double U[6];
    rigid_projection(o, o->bodies[n], n, Vv, U);
    for (int d = 0; d < 6; ++d) o->U0[6 * n + d] = U[d];
    double du[6];
    for (int d = 0; d < 6; ++d) du[d] = 0.5 * o->DT * U[d];
    body_update(o->midstep_bodies[n], du, Lv);
  }
  orc_fill_all_blob_pos(o, 1);
  orc_list_populate(o);
  return (wall_overlap(o) || (o->p.skip_on_overlap && orc_check_for_overlap(o))) ? 1 : 0;  // :611-617
}

// collection_of_rigid_bodies.cpp:869-953
double orc_calculate_divU(orc* o) {
  double divU = 0.0;
  o->temp_bodies = o->bodies;
  const double Lv[3] = {o->LX, o->LY, o->LZ};
  for (int i = 0; i < 6; i++) {
    double evec[6] = {0, 0, 0, 0, 0, 0};
    evec[i] = (i < 3) ? o->p.fd_delta * o->a : o->p.fd_delta;
    for (int n = 0; n < o->M; n++) body_update(o->bodies[n], evec, Lv);
    fill_pos(o, o->bodies);
    set_up_gaussians(o, o->all_blob_pos.data(), o->Nb);
    interp(o, o->ux_rand.data(), o->uy_rand.data(), o->uz_rand.data());
    const std::vector<double> V = o->V;
    for (int n = 0; n < o->M; n++) {
      double U[6];
      rigid_projection(o, o->bodies[n], n, V.data(), U);
      divU += (U[i] - o->U0[6 * n + i]) / evec[i];
      o->bodies[n] = o->temp_bodies[n];
    }
  }
  return divU;
}

// collection_of_rigid_bodies.cpp:759-790
int orc_end_of_step_update(orc* o, const double* U, double nu) {
  o->temp_bodies = o->bodies;
  const double Lv[3] = {o->LX, o->LY, o->LZ};
  for (int n = 0; n < o->M; n++) {
    double du[6];
    for (int d = 0; d < 6; ++d) du[d] = nu * o->DT * U[6 * n + d];
    body_update(o->bodies[n], du, Lv);
  }
  orc_fill_all_blob_pos(o, 0);
  orc_list_populate(o);
  return (wall_overlap(o) || (o->p.skip_on_overlap && orc_check_for_overlap(o))) ? 1 : 0;  // :780-786
}
void orc_reset_to_start_of_step(orc* o) { o->bodies = o->temp_bodies; }

// linked_list.cpp:104-190 via collection_of_rigid_bodies.cpp:195-205
int orc_check_for_overlap(orc* o) {
  const double lim = 4.0 * o->a * o->a;
  bool hit = false;
  list_visit(o, o->all_blob_pos, [&](int, int, double dx, double dy, double dz) {
    if (dx * dx + dy * dy + dz * dz < lim) hit = true;
  });
  return hit ? 1 : 0;
}

// linked_list.cpp:80-102
void orc_list_populate(orc* o) {
  const int total = o->Nc * o->Nc * o->Nc;
  for (int i = 0; i < total; i++) o->head[i] = -1;
  for (int i = 0; i < o->Nb; i++) {
    const int my_cell = find_containing_cell(o, &o->all_blob_pos[3 * i]);
    o->list[i] = o->head[my_cell];
    o->head[my_cell] = i;
  }
}
void orc_list_get_cells(orc* o, int32_t* cell) {
  for (int i = 0; i < o->Nb; i++) cell[i] = find_containing_cell(o, &o->all_blob_pos[3 * i]);
}
int64_t orc_list_get_pairs(orc* o, int32_t* pairs, int64_t cap) {
  std::vector<std::pair<int, int>> v;
  list_visit(o, o->all_blob_pos, [&](int b1, int b2, double, double, double) {
    v.push_back(std::make_pair(std::min(b1, b2), std::max(b1, b2)));
  });
  std::sort(v.begin(), v.end());
  const int64_t n = (int64_t)v.size();
  if (pairs && n <= cap)
    for (int64_t i = 0; i < n; ++i) { pairs[2 * i] = v[i].first; pairs[2 * i + 1] = v[i].second; }
  return n;
}
// linked_list.cpp:192-281
void orc_apply_barrier_forces(orc* o, double* F) {
  list_visit(o, o->all_blob_pos, [&](int b1, int b2, double dx, double dy, double dz) {
    const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
    const double mag = interaction_magnitude(o, r);
    const double dir[3] = {dx / r, dy / r, dz / r};
    for (int d = 0; d < 3; ++d) {
      F[3 * b1 + d] += mag * dir[d];
      F[3 * b2 + d] -= mag * dir[d];
    }
  });
}

void orc_set_up_gaussians(orc* o, const double* Y) {
  set_up_gaussians(o, Y ? Y : o->all_blob_pos.data(), o->Nb);
}
void orc_get_gaussians(orc* o, int32_t* ind, double* w) {
  const int W = o->W;
  for (int np = 0; np < o->ngauss_rows; ++np)
    for (int i = 0; i < W; ++i) {
      ind[(np * 3 + 0) * W + i] = o->indx[np * W + i];
      ind[(np * 3 + 1) * W + i] = o->indy[np * W + i];
      ind[(np * 3 + 2) * W + i] = o->indz[np * W + i];
      w[(np * 3 + 0) * W + i] = o->gaussx[np * W + i];
      w[(np * 3 + 1) * W + i] = o->gaussy[np * W + i];
      w[(np * 3 + 2) * W + i] = o->gaussz[np * W + i];
    }
}

void orc_inject_random_stress(orc* o, const double* sxx, const double* syy, const double* szz,
                              const double* sxy, const double* sxz, const double* syz) {
  o->sxx.assign(sxx, sxx + o->P);
  o->syy.assign(syy, syy + o->P);
  o->szz.assign(szz, szz + o->P);
  o->sxy.assign(sxy, sxy + o->P);
  o->sxz.assign(sxz, sxz + o->P);
  o->syz.assign(syz, syz + o->P);
  random_field_from_stress(o);
}

// fcm_fluid_solver.cpp:167-234 (SLIP_CHANNEL false): fill order i, k, j; one
// normal per array per index, in the order sxx, syy, szz, sxy, sxz, syz.  Each
// x-plane i draws from its own stream (seed; counter*2^20 + i), as each
// reference MPI rank draws its x-slab from its own SPRNG stream, so the planes
// fill in parallel.
// In sequential mode (orc_set_sequential_noise) every plane draws, in plane
// order, from one stream that continues across calls -- the single SPRNG stream
// of one reference rank -- and (seed, counter) are not used.
void orc_produce_random_velocity_field(orc* o, uint64_t seed, uint64_t counter) {
  const double var1 = std::sqrt(2.0 * o->kT * o->eta / (o->DX * o->DX * o->DX * o->DT));
  const double var2 = std::sqrt(2.0) * var1;
  const int Ny = o->Ny, pad = o->pad;
  const bool seq = o->seq_noise;
#pragma omp parallel for num_threads(seq ? 1 : g_threads) schedule(static)
  for (int i = 0; i < o->Nx; i++) {
    UniformStream plane_rng(seed, (counter << 20) + (uint64_t)i);
    UniformStream& rng = seq ? o->seq_rng : plane_rng;
    const size_t x_index = (size_t)i * Ny * pad;
    const int half_y = Ny / 2;
    for (int k = 0; k < pad; k++)
      for (int j = 0; j < Ny; j++) {
        const size_t index = x_index + k + (size_t)j * pad;
        if (o->p.slip_channel) {  // fcm_fluid_solver.cpp:186-217
          if ((j == 0) || (j == half_y)) {
            o->sxx[index] = std::sqrt(2.0) * var2 * rng.gaussian_random();
            o->syy[index] = std::sqrt(2.0) * var2 * rng.gaussian_random();
            o->szz[index] = std::sqrt(2.0) * var2 * rng.gaussian_random();
            o->sxz[index] = std::sqrt(2.0) * var1 * rng.gaussian_random();
            o->sxy[index] = 0.0;
            o->syz[index] = 0.0;
          } else if (j < half_y) {
            o->sxx[index] = var2 * rng.gaussian_random();
            o->syy[index] = var2 * rng.gaussian_random();
            o->szz[index] = var2 * rng.gaussian_random();
            o->sxz[index] = var1 * rng.gaussian_random();
            o->sxy[index] = var1 * rng.gaussian_random();
            o->syz[index] = var1 * rng.gaussian_random();
          } else {
            const size_t image_index = x_index + k + (size_t)(Ny - j) * pad;
            o->sxx[index] = o->sxx[image_index];
            o->syy[index] = o->syy[image_index];
            o->szz[index] = o->szz[image_index];
            o->sxz[index] = o->sxz[image_index];
            o->sxy[index] = -o->sxy[image_index];
            o->syz[index] = -o->syz[image_index];
          }
          continue;
        }
        o->sxx[index] = var2 * rng.gaussian_random();
        o->syy[index] = var2 * rng.gaussian_random();
        o->szz[index] = var2 * rng.gaussian_random();
        o->sxy[index] = var1 * rng.gaussian_random();
        o->sxz[index] = var1 * rng.gaussian_random();
        o->syz[index] = var1 * rng.gaussian_random();
      }
  }
  random_field_from_stress(o);
}

void orc_set_sequential_noise(orc* o, int on, uint64_t seed, uint64_t stream) {
  o->seq_noise = on != 0;
  o->seq_rng = UniformStream(seed, stream);
}

void orc_calculate_random_blob_velocities(orc* o, double* V) {
  interp(o, o->ux_rand.data(), o->uy_rand.data(), o->uz_rand.data());
  if (V) std::copy(o->V.begin(), o->V.end(), V);
}
void orc_set_up_force_distribution(orc* o, const double* F) { spread(o, F); }
void orc_produce_deterministic_velocity_field(orc* o) { produce_deterministic_velocity_field(o); }
void orc_calculate_deterministic_blob_velocities(orc* o, double* V) {
  interp(o, o->ux.data(), o->uy.data(), o->uz.data());
  if (V) std::copy(o->V.begin(), o->V.end(), V);
}
void orc_get_V(orc* o, double* V) { std::copy(o->V.begin(), o->V.end(), V); }
void orc_get_grid(orc* o, int which, double* out) {
  const std::vector<double>* g[9] = {&o->fx, &o->fy, &o->fz, &o->ux, &o->uy, &o->uz, &o->ux_rand, &o->uy_rand, &o->uz_rand};
  if (which >= 0 && which < 9) std::copy(g[which]->begin(), g[which]->end(), out);
}

// fcm_fluid_solver.cpp:842-881.  Body 0 alone at the box centre with the identity
// orientation (collection_of_rigid_bodies.cpp:132-151); the other bodies carry
// zero force in the reference, so they are left out of the spread.
void orc_produce_reference_matrices(orc* o) {
  const int nb = o->nb, n3 = 3 * nb;
  Body c;
  c.x[0] = 0.5 * o->LX; c.x[1] = (o->p.slip_channel ? 0.25 : 0.5) * o->LY; c.x[2] = 0.5 * o->LZ;  // :139-147
  c.q.s = 1.0; c.q.v[0] = c.q.v[1] = c.q.v[2] = 0.0;
  std::vector<double> Y((size_t)3 * nb);
  for (int m = 0; m < nb; ++m) blob_pos_of(o, c, 0, m, &Y[3 * m]);
  // save the blob-table state of the caller
  const std::vector<double> gx = o->gaussx, gy = o->gaussy, gz = o->gaussz, Vs = o->V;
  const std::vector<int> ix = o->indx, iy = o->indy, iz = o->indz;
  const int rows = o->ngauss_rows;
  set_up_gaussians(o, Y.data(), nb);
  Mat Mb((size_t)n3 * n3, 0.0);
  std::vector<double> evec(n3, 0.0);
  for (int n = 0; n < n3; n++) {
    evec[std::max(0, n - 1)] = 0.0;
    evec[n] = 1.0;
    spread(o, evec.data());
    produce_deterministic_velocity_field(o);
    interp(o, o->ux.data(), o->uy.data(), o->uz.data());
    for (int i = 0; i < n3; ++i) Mb[(size_t)n * n3 + i] = o->V[i];
  }
  dense_inv_sympd(Mb, n3, o->ref_Minv);
  Mat K((size_t)n3 * 6, 0.0);
  for (int m = 0; m < nb; m++) {
    double C[3][3];
    rcross(&o->blob_ref_pos[3 * m], C);
    for (int d = 0; d < 3; ++d) K[(size_t)d * n3 + 3 * m + d] = 1.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) K[(size_t)(3 + j) * n3 + 3 * m + i] = C[i][j];
  }
  Mat KtMK(36, 0.0);
  std::vector<double> col(n3), t(n3);
  for (int j = 0; j < 6; ++j) {
    for (int i = 0; i < n3; ++i) col[i] = K[(size_t)j * n3 + i];
    gemv(o->ref_Minv, n3, n3, col.data(), t.data());
    for (int i = 0; i < 6; ++i) {
      double s = 0.0;
      for (int r = 0; r < n3; ++r) s += K[(size_t)i * n3 + r] * t[r];
      KtMK[(size_t)j * 6 + i] = s;
    }
  }
  sym_inv_or_pinv(KtMK, 6, o->ref_N);  // fcm_fluid_solver.cpp:877
  o->gaussx = gx; o->gaussy = gy; o->gaussz = gz; o->V = Vs;
  o->indx = ix; o->indy = iy; o->indz = iz;
  o->ngauss_rows = rows;
}
void orc_get_reference_matrices(orc* o, double* Minv, double* N, double* KTKinv) {
  if (Minv) std::copy(o->ref_Minv.begin(), o->ref_Minv.end(), Minv);
  if (N) std::copy(o->ref_N.begin(), o->ref_N.end(), N);
  if (KTKinv) std::copy(o->ref_KTKinv.begin(), o->ref_KTKinv.end(), KTKinv);
}
void orc_set_reference_matrices(orc* o, const double* Minv, const double* N) {
  if (Minv) o->ref_Minv.assign(Minv, Minv + (size_t)9 * o->nb * o->nb);
  if (N) o->ref_N.assign(N, N + 36);
}

// ---------------------------------------------------------------- per-body shapes
// No counterpart in the reference (one blob_ref_pos per collection).  Each body
// gets its own shape and ref_KTKinv = inv(K^T K) of that shape
// (collection_of_rigid_bodies.cpp:117-130 applied per body); the preconditioner
// blocks start as identities (as the single-shape ones do before
// produce_reference_matrices).
void orc_set_body_shapes(orc* o, const double* shapes) {
  const int nb = o->nb, n3 = 3 * nb, M = o->M;
  o->shapes.assign(shapes, shapes + (size_t)n3 * M);
  o->body_KTKinv.assign(36 * (size_t)M, 0.0);
  o->body_Minv.assign((size_t)n3 * n3 * M, 0.0);
  o->body_N.assign(36 * (size_t)M, 0.0);
  for (int n = 0; n < M; ++n) {
    Mat K((size_t)n3 * 6, 0.0);
    for (int m = 0; m < nb; m++) {
      double C[3][3];
      rcross(&o->shapes[3 * ((size_t)n * nb + m)], C);
      for (int d = 0; d < 3; ++d) K[(size_t)d * n3 + 3 * m + d] = 1.0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) K[(size_t)(3 + j) * n3 + 3 * m + i] = C[i][j];
    }
    Mat KTK(36, 0.0), KTKinv;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j < 6; ++j) {
        double sum = 0.0;
        for (int t = 0; t < n3; ++t) sum += K[(size_t)i * n3 + t] * K[(size_t)j * n3 + t];
        KTK[(size_t)j * 6 + i] = sum;
      }
    sym_inv_or_pinv(KTK, 6, KTKinv);
    std::copy(KTKinv.begin(), KTKinv.end(), o->body_KTKinv.begin() + 36 * (size_t)n);
    for (int i = 0; i < n3; ++i) o->body_Minv[(size_t)n * n3 * n3 + (size_t)i * n3 + i] = 1.0;
    for (int i = 0; i < 6; ++i) o->body_N[36 * (size_t)n + 7 * i] = 1.0;
  }
  o->per_body = true;
}

void orc_set_body_preconditioners(orc* o, const double* Minv, const double* N) {
  const size_t n3 = 3 * (size_t)o->nb;
  if (Minv) o->body_Minv.assign(Minv, Minv + n3 * n3 * o->M);
  if (N) o->body_N.assign(N, N + 36 * (size_t)o->M);
}

void orc_get_body_preconditioners(orc* o, double* Minv, double* N, double* KTKinv) {
  if (Minv) std::copy(o->body_Minv.begin(), o->body_Minv.end(), Minv);
  if (N) std::copy(o->body_N.begin(), o->body_N.end(), N);
  if (KTKinv) std::copy(o->body_KTKinv.begin(), o->body_KTKinv.end(), KTKinv);
}

// The preconditioner blocks of every body from the free-space FCM blob-blob
// mobility.  Two blobs with Gaussian force envelopes of variance sigma^2 = a^2/pi
// interact through the Stokeslet smoothed by their convolved envelope (variance
// s^2 = 2 sigma^2): with g(r) the mean of |x - Z| over Z ~ N(0, s^2 I), the
// biharmonic part of the Stokes solution is -g/(8 pi) and the flow is
//   M(r) = [(2 erf/r - g'/r) I + (g'/r - g'') rr/r^2] / (8 pi eta),
//   g'  = (1 - s^2/r^2) erf + sqrt(2/pi)(s/r) e,   g'' = 2 s^2/r^3 erf - 2 sqrt(2/pi)(s/r^2) e,
// erf = erf(r/(sqrt2 s)), e = exp(-r^2/(2 s^2)); M(0) = I/(6 pi eta a).  Then
// ref_Minv = inv(M_body) and ref_N = inv(K^T ref_Minv K) in the body frame.
void orc_produce_body_preconditioners(orc* o) {
  const int nb = o->nb, n3 = 3 * nb;
  const double a = o->a, eta = o->p.viscosity;
  const double s = std::sqrt(2.0 / PI) * a, c2 = std::sqrt(2.0 / PI);
  for (int n = 0; n < o->M; ++n) {
    const double* sh = &o->shapes[(size_t)n * n3];
    Mat Mb((size_t)n3 * n3, 0.0);
    for (int i = 0; i < nb; ++i)
      for (int j = 0; j < nb; ++j) {
        double d[3] = {sh[3 * i] - sh[3 * j], sh[3 * i + 1] - sh[3 * j + 1], sh[3 * i + 2] - sh[3 * j + 2]};
        const double r = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double Aii, Brr;
        if (i == j || r < 1e-10 * s) {
          Aii = 1.0 / (6.0 * PI * eta * a);
          Brr = 0.0;
        } else {
          const double er = std::erf(r / (std::sqrt(2.0) * s)), e = std::exp(-r * r / (2.0 * s * s));
          const double g1 = (1.0 - s * s / (r * r)) * er + c2 * (s / r) * e;
          const double g2 = 2.0 * s * s / (r * r * r) * er - 2.0 * c2 * s / (r * r) * e;
          Aii = (2.0 * er / r - g1 / r) / (8.0 * PI * eta);
          Brr = (g1 / r - g2) / (8.0 * PI * eta) / (r * r);
        }
        for (int p = 0; p < 3; ++p)
          for (int q = 0; q < 3; ++q)
            Mb[(size_t)(3 * j + q) * n3 + 3 * i + p] = (p == q ? Aii : 0.0) + Brr * d[p] * d[q];
      }
    Mat Minv, N;
    dense_inv_sympd(Mb, n3, Minv);
    Mat K((size_t)n3 * 6, 0.0);
    for (int m = 0; m < nb; m++) {
      double C[3][3];
      rcross(&sh[3 * m], C);
      for (int dd = 0; dd < 3; ++dd) K[(size_t)dd * n3 + 3 * m + dd] = 1.0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) K[(size_t)(3 + j) * n3 + 3 * m + i] = C[i][j];
    }
    Mat KtMK(36, 0.0);
    std::vector<double> col(n3), t(n3);
    for (int j = 0; j < 6; ++j) {
      for (int i = 0; i < n3; ++i) col[i] = K[(size_t)j * n3 + i];
      gemv(Minv, n3, n3, col.data(), t.data());
      for (int i = 0; i < 6; ++i) {
        double sum = 0.0;
        for (int r = 0; r < n3; ++r) sum += K[(size_t)i * n3 + r] * t[r];
        KtMK[(size_t)j * 6 + i] = sum;
      }
    }
    sym_inv_or_pinv(KtMK, 6, N);
    std::copy(Minv.begin(), Minv.end(), o->body_Minv.begin() + (size_t)n * n3 * n3);
    std::copy(N.begin(), N.end(), o->body_N.begin() + 36 * (size_t)n);
  }
}

// gmres_solver.cpp:58-70
void orc_assemble_RHS(orc* o) {
  const int Nb = o->Nb;
  for (int i = 0; i < 3 * Nb; ++i) o->RHS[i] = -o->V[i];
  if (o->shear)  // gmres_solver.cpp:62-64
    for (int i = 0; i < 3 * Nb; ++i) o->RHS[i] -= o->Vshear[i];
  std::vector<double> kt(6 * o->M);
  mult_KT(o, o->blob_forces.data(), kt.data());
  for (int i = 0; i < 6 * o->M; ++i) o->RHS[3 * Nb + i] = -kt[i] - o->ext_forces[i];
}
void orc_get_RHS(orc* o, double* rhs) { std::copy(o->RHS.begin(), o->RHS.end(), rhs); }
void orc_set_RHS(orc* o, const double* rhs) { o->RHS.assign(rhs, rhs + o->system_size); }
void orc_multiply_by_Pinv(orc* o, const double* in, double* out) { mult_Pinv(o, in, out); }
void orc_multiply_by_saddle_point_matrix(orc* o, const double* in, double* out) { mult_A(o, in, out); }
int orc_invert_saddle_point_system(orc* o, double* soln, int* iters, double* rel) {
  return gmres(o, soln, iters, rel);
}

// main.cpp:222-451 (one pass of the while loop; `continue` becomes a rejected step).
static int step_impl(orc* o, bool injected, const double* s6, uint64_t seed, uint64_t step_index, fcm_step_info* info) {
  fcm_step_info inf;
  std::memset(&inf, 0, sizeof(inf));
  inf.refinement_sweeps = 1;
  const bool noise = o->p.noise != 0;
  orc_fill_all_blob_pos(o, 0);
  if (noise) {
    if (injected) {
      const size_t P = o->P;
      orc_inject_random_stress(o, s6, s6 + P, s6 + 2 * P, s6 + 3 * P, s6 + 4 * P, s6 + 5 * P);
    } else {
      orc_produce_random_velocity_field(o, seed, step_index);
    }
  } else {
    std::fill(o->ux_rand.begin(), o->ux_rand.end(), 0.0);
    std::fill(o->uy_rand.begin(), o->uy_rand.end(), 0.0);
    std::fill(o->uz_rand.begin(), o->uz_rand.end(), 0.0);
  }
  set_up_gaussians(o, o->all_blob_pos.data(), o->Nb);
  interp(o, o->ux_rand.data(), o->uy_rand.data(), o->uz_rand.data());
  double nu = 1.0;
  if (o->p.algorithm == 1) {
    if (orc_advance_to_midstep(o, nullptr)) {
      inf.overlap = 1;
      if (info) *info = inf;
      return FCM_ERR_OVERLAP;
    }
    const double divU = orc_calculate_divU(o);
    inf.divU = divU;
    nu = 1.0 + 0.5 * o->DT * divU;
    orc_fill_all_blob_pos(o, 1);
    set_up_gaussians(o, o->all_blob_pos.data(), o->Nb);
    interp(o, o->ux_rand.data(), o->uy_rand.data(), o->uz_rand.data());
    if (o->shear) orc_calculate_shear_blob_velocities(o, nullptr);  // main.cpp:270-272
  }
  calculate_forces(o);
  orc_assemble_RHS(o);
  std::vector<double> soln(o->system_size);
  int iters = 0;
  double rel = 0.0;
  const int st = gmres(o, soln.data(), &iters, &rel);
  inf.gmres_iters = iters;
  inf.gmres_rel_residual = rel;
  inf.status = st;
  const int ov = orc_end_of_step_update(o, soln.data() + 3 * o->Nb, nu);
  if (ov) {
    orc_reset_to_start_of_step(o);
    inf.overlap = 1;
    if (info) *info = inf;
    return FCM_ERR_OVERLAP;
  }
  if (info) *info = inf;
  return 0;
}

int orc_step(orc* o, uint64_t seed, uint64_t step_index, fcm_step_info* info) {
  return step_impl(o, false, nullptr, seed, step_index, info);
}
int orc_step_injected(orc* o, const double* s6, fcm_step_info* info) {
  return step_impl(o, true, s6, 0, 0, info);
}

}  // extern "C"

// ------------------------------------------------------------------ force dipoles
// No reference code: the FCM force-dipole (stresslet and torque) terms named
// for this project, restated from the published FCM dipole formulation (Lomholt
// & Maxey, J. Comput. Phys. 184 (2003) 381-405) on the reference's grid
// conventions.  Dipole envelope: a Gaussian of width sigma_D = a / (6 sqrt(pi))^(1/3)
// on the same W-point stencil as the force envelope (fcm_fluid_solver.cpp:131-165).
// Blob dipole D_ij = S_ij - 1/2 eps_ijk T_k (S symmetric, row-major 9 per blob);
// force density f_i = F_i Delta + D_ij (x_j - Y_j) / sigma_D^2 Delta_D, whose
// first moment is D (torque T, stresslet S).  Moments of the velocity,
// M_kj = DX^3 sum u_k (x_j - Y_j) / sigma_D^2 Delta_D (= the average of du_k/dx_j):
// Omega_i = 1/2 eps_ijk M_kj, E_ij = (M_ij + M_ji) / 2.
namespace {

// Dipole weights of blob np, dimension d: g = Delta_D factor, h = g (x - Y) / sigma_D^2,
// on the stencil points ind[] of set_up_gaussians.
void dipole_weights(const orc* o, const double* Y, int np, int d, double* g, double* h) {
  const int W = o->W, ngdh = W / 2;
  const double sD = o->a / std::cbrt(6.0 * std::sqrt(PI));
  const double anorm = 1.0 / (std::sqrt(2.0 * PI) * sD);
  const double anorm2 = 2.0 * sD * sD;
  const int c = int(Y[3 * np + d] / o->DX);
  for (int i = 0; i < W; i++) {
    const int xg = c - ngdh + (i + 1);
    const double xx = xg * o->DX - Y[3 * np + d];
    g[i] = anorm * std::exp(-xx * xx / anorm2);
    h[i] = g[i] * xx / (sD * sD);
  }
}

void blob_dipole(const double* T, const double* S, int np, double D[3][3]) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) D[i][j] = S ? S[9 * np + 3 * i + j] : 0.0;
  if (T) {
    const double* t = T + 3 * np;
    // -1/2 eps_ijk T_k
    D[0][1] += -0.5 * t[2];
    D[1][0] += 0.5 * t[2];
    D[0][2] += 0.5 * t[1];
    D[2][0] += -0.5 * t[1];
    D[1][2] += -0.5 * t[0];
    D[2][1] += 0.5 * t[0];
  }
}

}  // namespace

extern "C" {

void orc_set_up_dipole_distribution(orc* o, const double* F, const double* T, const double* S) {
  const int W = o->W, Ny = o->Ny, pad = o->pad, nrows = o->ngauss_rows;
  std::vector<double> zero;
  if (!F) {
    zero.assign(3 * (size_t)nrows, 0.0);
    F = zero.data();
  }
  spread(o, F);
  if (!T && !S) return;
  const double* Y = o->gauss_Y.data();
  std::vector<double> gx(W), hx(W), gy(W), hy(W), gz(W), hz(W);
  for (int np = 0; np < nrows; np++) {
    double D[3][3];
    blob_dipole(T, S, np, D);
    dipole_weights(o, Y, np, 0, gx.data(), hx.data());
    dipole_weights(o, Y, np, 1, gy.data(), hy.data());
    dipole_weights(o, Y, np, 2, gz.data(), hz.data());
    for (int i = 0; i < W; i++) {
      const size_t x_index = (size_t)o->indx[np * W + i] * Ny * pad;
      for (int j = 0; j < W; j++) {
        const size_t y_index = (size_t)o->indy[np * W + j] * pad;
        for (int k = 0; k < W; k++) {
          const size_t index = x_index + y_index + o->indz[np * W + k];
          const double r[3] = {hx[i] * gy[j] * gz[k], gx[i] * hy[j] * gz[k], gx[i] * gy[j] * hz[k]};
          o->fx[index] += D[0][0] * r[0] + D[0][1] * r[1] + D[0][2] * r[2];
          o->fy[index] += D[1][0] * r[0] + D[1][1] * r[1] + D[1][2] * r[2];
          o->fz[index] += D[2][0] * r[0] + D[2][1] * r[1] + D[2][2] * r[2];
        }
      }
    }
  }
}

// Omega (3 per blob) and E (9 per blob, row-major) of the deterministic field.
void orc_calculate_deterministic_blob_rotations(orc* o, double* Om, double* E) {
  const int W = o->W, Ny = o->Ny, pad = o->pad, nrows = o->ngauss_rows;
  const double norm = o->DX * o->DX * o->DX;
  const double* Y = o->gauss_Y.data();
  const double* u[3] = {o->ux.data(), o->uy.data(), o->uz.data()};
#pragma omp parallel for num_threads(g_threads) schedule(dynamic, 16)
  for (int np = 0; np < nrows; np++) {
    std::vector<double> gx(W), hx(W), gy(W), hy(W), gz(W), hz(W);
    dipole_weights(o, Y, np, 0, gx.data(), hx.data());
    dipole_weights(o, Y, np, 1, gy.data(), hy.data());
    dipole_weights(o, Y, np, 2, gz.data(), hz.data());
    double M[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
    for (int i = 0; i < W; i++) {
      const size_t x_index = (size_t)o->indx[np * W + i] * Ny * pad;
      for (int j = 0; j < W; j++) {
        const size_t y_index = (size_t)o->indy[np * W + j] * pad;
        for (int k = 0; k < W; k++) {
          const size_t index = x_index + y_index + o->indz[np * W + k];
          const double r[3] = {hx[i] * gy[j] * gz[k], gx[i] * hy[j] * gz[k], gx[i] * gy[j] * hz[k]};
          for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) M[a][b] += u[a][index] * r[b];
        }
      }
    }
    for (int a = 0; a < 3; a++)
      for (int b = 0; b < 3; b++) M[a][b] *= norm;
    if (Om) {
      Om[3 * np] = 0.5 * (M[2][1] - M[1][2]);
      Om[3 * np + 1] = 0.5 * (M[0][2] - M[2][0]);
      Om[3 * np + 2] = 0.5 * (M[1][0] - M[0][1]);
    }
    if (E)
      for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) E[9 * np + 3 * a + b] = 0.5 * (M[a][b] + M[b][a]);
  }
}

}  // extern "C"

// ------------------------------------------------------------------ Metropolis Monte Carlo
namespace {

// linked_list.cpp:362-497, MARKOV_CHAIN_MONTE_CARLO branches (pair energies);
// potential 3: U(r) = int_r^rc F_s ((rc^2 - s^2)/(rc^2 - 4a^2))^4 ds.
double interaction_energy(const orc* o, double r) {
  const double a = o->a, kT = o->kT;
  if (o->p.potential == 3) {
    // degree-8 polynomial integrand: 5-point Gauss-Legendre is exact, all terms positive
    const double rc = o->p.steric_rc;
    if (r >= rc) return 0.0;
    const double xg[5] = {-0.9061798459386640, -0.5384693101056831, 0.0, 0.5384693101056831, 0.9061798459386640};
    const double wg[5] = {0.2369268850561891, 0.4786286704993665, 0.5688888888888889, 0.4786286704993665,
                          0.2369268850561891};
    const double D = rc * rc - 4.0 * a * a, mid = 0.5 * (rc + r), half = 0.5 * (rc - r);
    double u = 0.0;
    for (int k = 0; k < 5; ++k) {
      const double s = mid + half * xg[k];
      const double t = (rc * rc - s * s) / D;
      const double t2 = t * t;
      u += wg[k] * (t2 * t2);
    }
    return o->p.steric_fs * half * u;
  }
  const double U0 = 20.0 * kT, b = 0.5 * a;
  double e = (r < 2.0 * a) ? U0 + U0 * (2.0 * a - r) / b : U0 * std::exp((2.0 * a - r) / b);
  if (o->p.potential == 1 || o->p.potential == 2) {
    const double A = 5.0 * kT, lambda = 0.5 * a;
    if (r < 2.0 * a) {
      double temp = a / lambda;
      temp = A * std::exp(-temp * temp);
      e -= temp;
      e += 2.0 * a * (2.0 * a - r) * temp / (lambda * lambda);
      if (o->p.potential == 2) {
        temp = 1.5 * a / lambda;
        temp = A * std::exp(-temp * temp);
        e += temp;
        e -= 3.0 * a * (2.0 * a - r) * temp / (lambda * lambda);
      }
    } else {
      double temp = (r - 3.0 * a) / lambda;
      e -= A * std::exp(-temp * temp);
      if (o->p.potential == 2) {
        temp = (r - 3.5 * a) / lambda;
        e += A * std::exp(-temp * temp);
      }
    }
  }
  return e;
}

// linked_list.cpp:283-360 on the current list.
double barrier_potential(const orc* o) {
  double U = 0.0;
  list_visit(o, o->all_blob_pos, [&](int, int, double dx, double dy, double dz) {
    U += interaction_energy(o, std::sqrt(dx * dx + dy * dy + dz * dz));
  });
  return U;
}

// Uniform in [0, 1) with 53 bits from Philox4x32-10, counter (i, 0x4D434D43,
// attempt), key seed: the same numbers as the GPU's Metropolis kernels.
double mcmc_uniform(uint64_t seed, uint64_t attempt, uint32_t i) {
  const uint32_t ctr[4] = {i, 0x4D434D43u, (uint32_t)attempt, (uint32_t)(attempt >> 32)};
  uint32_t out[4];
  Philox::gen(ctr, (uint32_t)seed, (uint32_t)(seed >> 32), out);
  return ((double)(out[0] >> 5) * 67108864.0 + (double)(out[1] >> 6)) * (1.0 / 9007199254740992.0);
}

// collection_of_rigid_bodies.cpp:666-705: the pair potential, then a slip
// channel's wall potential blob by blob (:679-700).
double total_potential(orc* o) {
  double potential = barrier_potential(o);
  if (o->p.slip_channel) {
    const double L = 2.2 * o->a;
    const double K = 40.0 * o->kT / (L * o->a);
    for (int i = 0; i < o->Nb; i++) {
      const double y = o->all_blob_pos[3 * i + 1];
      if (y <= L) {
        potential += 0.5 * K * (L - y) * (L - y);
      } else if ((0.5 * o->LY - y <= L) && (y <= 0.5 * o->LY)) {
        potential += 0.5 * K * (L - 0.5 * o->LY + y) * (L - 0.5 * o->LY + y);
      }
    }
  }
  return potential;
}

}  // namespace

extern "C" {

// collection_of_rigid_bodies.cpp:666-705 for the current bodies.
double orc_calculate_potential(orc* o) {
  orc_fill_all_blob_pos(o, 0);
  orc_list_populate(o);
  return total_potential(o);
}

// main.cpp:113-210 with Philox uniforms (see mcmc_uniform).
int orc_mcmc_run(orc* o, uint64_t seed, int64_t n_steps, fcm_mcmc_state* st) {
  double body_radius = 0.0;  // collection_of_rigid_bodies.cpp:110-114 (over every shape)
  const std::vector<double>& all_refs = o->per_body ? o->shapes : o->blob_ref_pos;
  for (size_t m = 0; m < all_refs.size(); m += 3) {
    const double* r = &all_refs[m];
    body_radius = std::max(body_radius, std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]));
  }
  if (body_radius == 0.0) body_radius = o->a;
  double U_old = orc_calculate_potential(o);
  const double rs = 20.0;
  int64_t n = st->steps, attempt = st->attempts;
  const int64_t target = n + n_steps, cap = attempt + 100 * n_steps + 1000;
  double scale = st->scale, acc = st->acceptance_ratio;
  std::vector<double> move(6 * (size_t)o->M);
  while (n < target && attempt < cap) {
    for (int b = 0; b < o->M; ++b)
      for (int d = 0; d < 6; ++d) {
        double mv = scale * (2.0 * mcmc_uniform(seed, (uint64_t)attempt, (uint32_t)(6 * b + d)) - 1.0);
        if (d >= 3) mv /= body_radius;
        move[6 * b + d] = mv;
      }
    if (orc_end_of_step_update(o, move.data(), 1.0)) {
      orc_reset_to_start_of_step(o);
      ++attempt;
      continue;
    }
    const double U = total_potential(o);
    const double u = mcmc_uniform(seed, (uint64_t)attempt, (uint32_t)(6 * o->M));
    if (u < std::exp((U_old - U) / o->kT)) {
      U_old = U;
      acc = ((rs - 1.0) * acc + 1.0) / rs;
    } else {
      orc_reset_to_start_of_step(o);
      acc *= (rs - 1.0) / rs;
    }
    ++n;
    scale *= acc > 0.5 ? 1.02 : 0.98;
    ++attempt;
  }
  orc_fill_all_blob_pos(o, 0);
  orc_list_populate(o);
  st->scale = scale;
  st->acceptance_ratio = acc;
  st->potential = U_old;
  st->steps = n;
  st->attempts = attempt;
  return n < target ? FCM_ERR_OVERLAP : FCM_OK;
}

}  // extern "C"

// ------------------------------------------------------------------ shear forcing
// fcm_fluid_solver.cpp:703-842 (SHEARING_FORCES, SLIP_CHANNEL false): the Stokes
// flow driven by the body force fx(j) = scale*kT*sin(wavenumber*2*pi*j/Ny)/a,
// fy = fz = 0, on every grid point.  Its k-space steps (:771-833) are those of
// produce_deterministic_velocity_field (:636-701); the result is kept as
// u*_shear and the force and velocity grids are left holding this solve, as in
// the reference.
extern "C" {

void orc_produce_shear_velocity_field(orc* o, double scale, double wavenumber) {
  const int Nx = o->Nx, Ny = o->Ny, Nz = o->Nz, pad = o->pad;
  std::fill(o->fx.begin(), o->fx.end(), 0.0);
  std::fill(o->fy.begin(), o->fy.end(), 0.0);
  std::fill(o->fz.begin(), o->fz.end(), 0.0);
  for (int i = 0; i < Nx; i++) {
    const size_t x_index = (size_t)i * Ny * pad;
    for (int j = 0; j < Ny; j++) {
      const size_t y_index = (size_t)j * pad;
      const double f = scale * o->kT * std::sin(wavenumber * 2.0 * PI * double(j) / double(Ny)) / o->a;
      for (int k = 0; k < Nz; k++) o->fx[x_index + y_index + k] = f;
    }
  }
  if (o->p.slip_channel) slip_image(o);  // :735-760
  produce_deterministic_velocity_field(o);
  o->ux_shear = o->ux;
  o->uy_shear = o->uy;
  o->uz_shear = o->uz;
  o->shear = true;
}

// fcm_fluid_solver.cpp:489-550: Vshear = J u_shear on the current Gaussians
// (V itself is left as it was).
void orc_calculate_shear_blob_velocities(orc* o, double* Vshear) {
  if (!o->shear) return;
  const std::vector<double> keep = o->V;
  interp(o, o->ux_shear.data(), o->uy_shear.data(), o->uz_shear.data());
  o->Vshear = o->V;
  o->V = keep;
  if (Vshear) std::copy(o->Vshear.begin(), o->Vshear.end(), Vshear);
}

// main.cpp:371-433: the deterministic flow of blob forces F (3Nb) on the current
// Gaussians plus the imposed flow, x-velocity averaged over x and z for every y
// (profile: Ny values).  The force and velocity grids keep that solve.
void orc_fluid_x_velocity_in_y(orc* o, const double* F, double* profile) {
  orc_set_up_force_distribution(o, F);
  produce_deterministic_velocity_field(o);
  const int Nx = o->Nx, Ny = o->Ny, Nz = o->Nz, pad = o->pad;
  for (int j = 0; j < Ny; j++) {
    const size_t y_index = (size_t)j * pad;
    double u_local = 0.0;
    for (int i = 0; i < Nx; i++) {
      const size_t x_index = (size_t)i * Ny * pad;
      for (int k = 0; k < Nz; k++) {
        const size_t index = x_index + y_index + k;
        u_local += o->ux[index] + (o->shear ? o->ux_shear[index] : 0.0);
      }
    }
    profile[j] = u_local / (Nx * Nz);
  }
}

}  // extern "C"
