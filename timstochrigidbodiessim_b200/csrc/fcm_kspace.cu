// fcm_kspace.cu -- Fourier-space Stokes projection and fluctuating stress.
//
// Projection restates fcm_fluid_solver.cpp:636-701 (and :294-347):
//   u_c = norm * (f_c - q_c * (q.f) * norm) / (eta * G),
//   norm = 1 / (qy^2 + qx^2 + 1e-16 + qz^2), u(0) = 0, with the unzeroed Nyquist
//   wavenumbers (+N/2 * 2pi/L) of fcm_fluid_solver.cpp:71-127.
// The fluctuating term restates :243-292: f = i (q~ . sigma) with q~ = q whose
// Nyquist components are zeroed.
//
// C2R semantics.  At Nyquist indices the projection is not even in q, so the
// projected spectrum is not Hermitian in the kz = 0 and kz = nz/2 planes.  The
// reference's FFTW 2.x inverse uses only the Hermitian part of those planes
// (complex inverse along x, y, then a half-complex z transform without the
// imaginary parts of kz = 0, nz/2).  These kernels therefore write, in those two
// planes, u_sym(k) = (u(k) + conj(u(-k)))/2, with u(-k) computed from the
// partner mode; cuFFT's C2R of a Hermitian-consistent spectrum then equals the
// reference's transform.  One thread handles each {k, -k} pair.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <type_traits>

#include "fcm_internal.cuh"

namespace fcm {

namespace {

template <typename T>
struct V2 {
  T x, y;
};

template <typename C>
__device__ __forceinline__ V2<double> ld(const C& v) {
  return V2<double>{(double)v.x, (double)v.y};
}

// Wavenumber of index i on an n-point grid (fcm_fluid_solver.cpp:77-91).
__device__ __forceinline__ double wavenumber(int i, int n, double fac) {
  return (i <= n / 2) ? (double)i * fac : (double)(i - n) * fac;
}

// Projection of one complex mode (re and im share the real factors).  The
// reference divides every component by eta*G; here one reciprocal of the
// mode's |q|^2 and a precomputed 1/(eta*G) are used instead (a last-bit change).
template <typename T>
__device__ __forceinline__ void project_mode(double q1, double q2, double q3, const V2<T> f[3], V2<T> u[3],
                                             T inv_etaG) {
  const T t1 = (T)q1, t2 = (T)q2, t3 = (T)q3;
  const T qq = (T)(q2 * q2) + (T)(q1 * q1) + (T)1e-16;
  const T norm = (T)1 / (qq + (T)(q3 * q3));
  const T kr = (t1 * f[0].x + t2 * f[1].x + t3 * f[2].x) * norm;
  const T ki = (t1 * f[0].y + t2 * f[1].y + t3 * f[2].y) * norm;
  const T sc = norm * inv_etaG;
  const T qv[3] = {t1, t2, t3};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    u[c].x = sc * (f[c].x - qv[c] * kr);
    u[c].y = sc * (f[c].y - qv[c] * ki);
  }
}

__device__ __forceinline__ void mode_coords(long long t, const KParams& k, int& x, int& y, int& kz) {
  kz = (int)(t % k.nzh);
  const long long xy = t / k.nzh;
  y = (int)(xy % k.ny);
  x = (int)(xy / k.ny);
}

__device__ __forceinline__ bool is_plane(int kz, const KParams& k) {
  return kz == 0 || ((k.nz % 2) == 0 && kz == k.nz / 2);
}

template <typename C, typename T>
__device__ __forceinline__ void store3(C* spec, long long Gc, long long t, const V2<T> u[3]) {
  if (!FCM_INB(t, Gc, BS_SPECTRUM)) return;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    C v;
    v.x = u[c].x;
    v.y = u[c].y;
    spec[c * Gc + t] = v;
  }
}

template <typename C, typename T>
__device__ __forceinline__ void load3(const C* spec, long long Gc, long long t, V2<T> f[3]) {
  if (!FCM_INB(t, Gc, BS_SPECTRUM)) {
    for (int c = 0; c < 3; ++c) f[c] = V2<T>{(T)0, (T)0};
    return;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const C v = spec[c * Gc + t];
    f[c].x = v.x;
    f[c].y = v.y;
  }
}

// Deterministic projection in place (fcm_fluid_solver.cpp:642-695).
template <typename T, typename C>
__device__ __forceinline__ void project_one(C* __restrict__ spec, const KParams& k, long long t) {
  if (t >= k.Gc) return;
  int x, y, kz;
  mode_coords(t, k, x, y, kz);
  const double q1 = wavenumber(x, k.nx, k.fx), q2 = wavenumber(y, k.ny, k.fy), q3 = (double)kz * k.fz;
  V2<T> f[3], u[3];
  if (!is_plane(kz, k)) {
    load3(spec, k.Gc, t, f);
    project_mode<T>(q1, q2, q3, f, u, (T)k.inv_etaG);
    store3(spec, k.Gc, t, u);
    return;
  }
  const int xp = (k.nx - x) % k.nx, yp = (k.ny - y) % k.ny;
  const long long tp = ((long long)xp * k.ny + yp) * k.nzh + kz;
  if (tp < t) return;  // the partner's thread writes both
  if (t == 0) {        // f(0) = 0 and u(0) = 0 (fcm_fluid_solver.cpp:642-651, :686-695)
    V2<T> z[3] = {{0, 0}, {0, 0}, {0, 0}};
    store3(spec, k.Gc, t, z);
    return;
  }
  load3(spec, k.Gc, t, f);
  project_mode<T>(q1, q2, q3, f, u, (T)k.inv_etaG);
  if (tp == t) {
    for (int c = 0; c < 3; ++c) u[c].y = 0;
    store3(spec, k.Gc, t, u);
    return;
  }
  V2<T> fp[3], up[3];
  load3(spec, k.Gc, tp, fp);
  const double p1 = wavenumber(xp, k.nx, k.fx), p2 = wavenumber(yp, k.ny, k.fy);
  project_mode<T>(p1, p2, q3, fp, up, (T)k.inv_etaG);
  V2<T> us[3], usp[3];
  for (int c = 0; c < 3; ++c) {
    us[c].x = (T)0.5 * (u[c].x + up[c].x);
    us[c].y = (T)0.5 * (u[c].y - up[c].y);
    usp[c].x = us[c].x;
    usp[c].y = -us[c].y;
  }
  store3(spec, k.Gc, t, us);
  store3(spec, k.Gc, tp, usp);
}

template <typename T, typename C>
__global__ void __launch_bounds__(256, 4) k_project(C* __restrict__ spec, KParams k) {
  project_one<T, C>(spec, k, blockIdx.x * (long long)blockDim.x + threadIdx.x);
}

// Batched: kblock_map[blockIdx.x] = (member, block of 256 modes).
template <typename T, typename C, int P>
__global__ void __launch_bounds__(256, 4) k_b_project(const BMember* __restrict__ mem,
                                                      const int2* __restrict__ kblock_map, int mask) {
  const int2 mb = kblock_map[blockIdx.x];
  const BMember& m = mem[mb.x];
  if (bskip(m, mask) || m.xfft[P]) return;  // that precision's fused x-transform projects it
  project_one<T, C>((C*)m.spec[P], m.kp, (long long)mb.y * 256 + threadIdx.x);
}

// f = i (q~ . sigma) for one mode; sigma order xx, yy, zz, xy, xz, yz.
template <typename T>
__device__ __forceinline__ void stress_divergence(double q1, double q2, double q3, const V2<T> s[6], V2<T> f[3]) {
  const T a = (T)q1, b = (T)q2, c = (T)q3;
  // (q.sigma)_x = q1 sxx + q2 sxy + q3 sxz, etc.; i*(r + i m) = -m + i r
  const T rx = a * s[0].x + b * s[3].x + c * s[4].x, mx = a * s[0].y + b * s[3].y + c * s[4].y;
  const T ry = a * s[3].x + b * s[1].x + c * s[5].x, my = a * s[3].y + b * s[1].y + c * s[5].y;
  const T rz = a * s[4].x + b * s[5].x + c * s[2].x, mz = a * s[4].y + b * s[5].y + c * s[2].y;
  f[0].x = -mx; f[0].y = rx;
  f[1].x = -my; f[1].y = ry;
  f[2].x = -mz; f[2].y = rz;
}

// Nyquist-zeroed wavenumbers of the stress divergence (fcm_fluid_solver.cpp:245-278).
__device__ __forceinline__ void divergence_q(int x, int y, int kz, const KParams& k, double& q1, double& q2,
                                             double& q3) {
  q1 = (x == k.nx / 2) ? 0.0 : wavenumber(x, k.nx, k.fx);
  q2 = (y == k.ny / 2) ? 0.0 : wavenumber(y, k.ny, k.fy);
  q3 = (kz == k.nzh - 1) ? 0.0 : (double)kz * k.fz;
}

// Two standard normals from two 32-bit words (Box-Muller, single precision).
__device__ __forceinline__ void box_muller(unsigned int a, unsigned int b, float& n1, float& n2) {
  const float u1 = ((float)a + 0.5f) * 2.3283064365386963e-10f;
  const float u2 = ((float)b + 0.5f) * 2.3283064365386963e-10f;
  const float r = sqrtf(-2.0f * logf(u1));
  float sn, cs;
  sincospif(2.0f * u2, &sn, &cs);
  n1 = r * cs;
  n2 = r * sn;
}

// Twelve normals for mode index m: three Philox blocks with counter
// (m, block, counter_lo, counter_hi), key (seed_lo, seed_hi).
__device__ __forceinline__ void mode_normals(unsigned long long m, uint64_t seed, uint64_t counter, float nrm[12]) {
  const uint2 key = make_uint2((unsigned int)seed, (unsigned int)(seed >> 32));
#pragma unroll
  for (int blk = 0; blk < 3; ++blk) {
    const uint4 r = philox4x32_10(make_uint4((unsigned int)m, (unsigned int)blk, (unsigned int)counter,
                                             (unsigned int)(counter >> 32)), key);
    box_muller(r.x, r.y, nrm[4 * blk], nrm[4 * blk + 1]);
    box_muller(r.z, r.w, nrm[4 * blk + 2], nrm[4 * blk + 3]);
  }
}

// Fluctuating velocity spectrum.  Source 0: six stress spectra (R2C of the
// injected real-space arrays); source 1: stress drawn directly in Fourier space.
// For white real-space noise of variance v^2 per point, the unnormalised DFT has
// E|s(k)|^2 = G v^2, independent real and imaginary parts of variance G v^2/2
// for k != -k, a real value of variance G v^2 for self-conjugate k, and
// s(-k) = conj(s(k)); the Fourier-space draw reproduces exactly that law.
template <typename T, typename C, int SOURCE>
__global__ void k_fluct(C* __restrict__ spec, const cufftDoubleComplex* __restrict__ sig, KParams k, uint64_t seed,
                        uint64_t counter, const uint64_t* __restrict__ dargs, double amp_diag, double amp_off) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= k.Gc) return;
  if (dargs) {  // (seed, counter) from device memory (a captured step reads them there)
    seed = dargs[0];
    counter = dargs[1];
  }
  int x, y, kz;
  mode_coords(t, k, x, y, kz);
  const bool plane = is_plane(kz, k);
  long long tp = t;
  int xp = x, yp = y;
  if (plane) {
    xp = (k.nx - x) % k.nx;
    yp = (k.ny - y) % k.ny;
    tp = ((long long)xp * k.ny + yp) * k.nzh + kz;
    if (tp < t) return;
  }
  if (t == 0) {
    V2<T> z[3] = {{0, 0}, {0, 0}, {0, 0}};
    store3(spec, k.Gc, t, z);
    return;
  }
  V2<T> s[6], sp[6];
  if (SOURCE == 0) {
    for (int c = 0; c < 6; ++c) {
      const cufftDoubleComplex v = sig[c * k.Gc + t];
      s[c].x = (T)v.x;
      s[c].y = (T)v.y;
      if (plane && tp != t) {
        const cufftDoubleComplex w = sig[c * k.Gc + tp];
        sp[c].x = (T)w.x;
        sp[c].y = (T)w.y;
      }
    }
  } else if (k.slip) {
    // Image-symmetric stress of a slip channel (fcm_fluid_solver.cpp:186-217): xx, yy,
    // zz, xz even in y, xy and yz odd, the even ones with twice the variance on the
    // wall rows 0 and ny/2 and the odd ones zero there.  Its DFT along y is real
    // and even (odd: imaginary and odd) with independent rows ky = 0..ny/2, those of
    // the even components of variance ny v^2 (2 ny v^2 on ky = 0, ny/2), those of
    // the odd ones ny v^2 (0 on ky = 0, ny/2).  So row y takes the draw of row
    // yr = min(y, ny - y): even components a white (x, z) spectrum of variance
    // G v^2 (doubled on the wall rows), odd ones -i times one (zero on the wall
    // rows), negated for y > ny/2.  In the kz = 0 and nz/2 planes (x, yr) pairs
    // with (-x, yr) as the 2D spectrum of a real field.
    const int h = k.ny / 2;
    const int yr = y <= h ? y : k.ny - y;
    const bool wall = yr == 0 || yr == h;
    const int xm = (k.nx - x) % k.nx;
    const int xr = (plane && xm < x) ? xm : x;
    const bool cj = xr != x, xself = plane && xm == x;
    float nrm[12];
    mode_normals((unsigned long long)(((long long)xr * k.ny + yr) * k.nzh + kz), seed, counter, nrm);
    for (int c = 0; c < 6; ++c) {
      const double amp = (c < 3) ? amp_diag : amp_off;  // order xx, yy, zz, xy, xz, yz
      double re, im;
      if (xself) {
        re = amp * 1.4142135623730951 * (double)nrm[2 * c];
        im = 0.0;
      } else {
        re = amp * (double)nrm[2 * c];
        im = amp * (double)nrm[2 * c + 1];
      }
      if (cj) im = -im;
      if (c == 3 || c == 5) {  // odd: -i (re + i im), zero on the walls, negated above ny/2
        const double sg = wall ? 0.0 : (y > h ? -1.0 : 1.0);
        const double r2 = sg * im, i2 = -sg * re;
        re = r2;
        im = i2;
      } else if (wall) {
        re *= 1.4142135623730951;
        im *= 1.4142135623730951;
      }
      s[c].x = (T)re;
      s[c].y = (T)im;
      sp[c].x = s[c].x;
      sp[c].y = -s[c].y;
    }
  } else {
    float nrm[12];
    mode_normals((unsigned long long)t, seed, counter, nrm);
    const bool selfconj = plane && (tp == t);
    for (int c = 0; c < 6; ++c) {
      const double amp = (c < 3) ? amp_diag : amp_off;
      if (selfconj) {
        s[c].x = (T)(amp * 1.4142135623730951 * (double)nrm[2 * c]);
        s[c].y = 0;
      } else {
        s[c].x = (T)(amp * (double)nrm[2 * c]);
        s[c].y = (T)(amp * (double)nrm[2 * c + 1]);
      }
      sp[c].x = s[c].x;
      sp[c].y = -s[c].y;
    }
  }
  double q1, q2, q3;
  divergence_q(x, y, kz, k, q1, q2, q3);
  V2<T> f[3], u[3];
  stress_divergence<T>(q1, q2, q3, s, f);
  const double r1 = wavenumber(x, k.nx, k.fx), r2 = wavenumber(y, k.ny, k.fy), r3 = (double)kz * k.fz;
  project_mode<T>(r1, r2, r3, f, u, (T)k.inv_etaG);
  if (!plane) {
    store3(spec, k.Gc, t, u);
    return;
  }
  if (tp == t) {
    for (int c = 0; c < 3; ++c) u[c].y = 0;
    store3(spec, k.Gc, t, u);
    return;
  }
  double p1, p2, p3;
  divergence_q(xp, yp, kz, k, p1, p2, p3);
  V2<T> fp[3], up[3];
  stress_divergence<T>(p1, p2, p3, sp, fp);
  project_mode<T>(wavenumber(xp, k.nx, k.fx), wavenumber(yp, k.ny, k.fy), r3, fp, up, (T)k.inv_etaG);
  V2<T> us[3], usp[3];
  for (int c = 0; c < 3; ++c) {
    us[c].x = (T)0.5 * (u[c].x + up[c].x);
    us[c].y = (T)0.5 * (u[c].y - up[c].y);
    usp[c].x = us[c].x;
    usp[c].y = -us[c].y;
  }
  store3(spec, k.Gc, t, us);
  store3(spec, k.Gc, tp, usp);
}

// ------------------------------------------------------------------ fused x-transform
// The Stokes solve of a force grid as 2D transforms over (y, z) for every x-plane
// (cuFFT, or the library's kernels further below) with the transform along x, the
// projection and the inverse transform along x fused: interior CTAs take the
// x-pencils of TK consecutive kz of one y row (all three components), transform
// them along x, project every mode and transform back; plane CTAs do the same for
// the kz = 0 and kz = nz/2 modes of a row pair {y, -y}, whose modes pair as
// {k, -k}.  A 3D DFT is the x-DFT of the (y, z) DFTs, so this is the transform pair
// of the 3D path with the projection between.  Pencils are transformed in two
// register steps, N = N1 * N2 (both divisors of 96 up to 32).

template <typename T, typename C>
__device__ __forceinline__ V2<T> ldt(const C& v) {
  return V2<T>{(T)v.x, (T)v.y};
}

__constant__ double2 c_w96d[96];  // exp(-2 pi i k / 96)
__constant__ float2 c_w96f[96];

template <typename T>
__device__ __forceinline__ V2<T> w96(int k);
template <>
__device__ __forceinline__ V2<double> w96<double>(int k) {
  const double2 w = c_w96d[k];
  return V2<double>{w.x, w.y};
}
template <>
__device__ __forceinline__ V2<float> w96<float>(int k) {
  const float2 w = c_w96f[k];
  return V2<float>{w.x, w.y};
}

template <typename T>
__device__ __forceinline__ V2<T> cadd(V2<T> a, V2<T> b) { return V2<T>{a.x + b.x, a.y + b.y}; }
template <typename T>
__device__ __forceinline__ V2<T> csub(V2<T> a, V2<T> b) { return V2<T>{a.x - b.x, a.y - b.y}; }
template <typename T>
__device__ __forceinline__ V2<T> cmul(V2<T> a, V2<T> b) { return V2<T>{a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x}; }
template <typename T>
__device__ __forceinline__ V2<T> cmulc(V2<T> a, V2<T> b) { return V2<T>{a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y}; }
// -i z (forward) or +i z (inverse)
template <typename T, bool INV>
__device__ __forceinline__ V2<T> rot(V2<T> z) { return INV ? V2<T>{-z.y, z.x} : V2<T>{z.y, -z.x}; }

// In-register DFT of R points, R a divisor of 96: forward exp(-2 pi i n k / R),
// inverse exp(+2 pi i n k / R), unnormalised.  Decimation in time, R = P * Q.
template <typename T, int R, bool INV>
__device__ __forceinline__ void dft(V2<T> (&a)[R]) {
  if constexpr (R == 1) {
    return;
  } else if constexpr (R == 2) {
    const V2<T> t = a[1];
    a[1] = csub(a[0], t);
    a[0] = cadd(a[0], t);
  } else if constexpr (R == 3) {
    // W_3 = -1/2 -+ i sqrt(3)/2
    const T h = (T)0.86602540378443864676;
    const V2<T> t1 = cadd(a[1], a[2]);
    const V2<T> t2 = V2<T>{a[0].x - (T)0.5 * t1.x, a[0].y - (T)0.5 * t1.y};
    const V2<T> d = rot<T, INV>(csub(a[1], a[2]));
    a[0] = cadd(a[0], t1);
    a[1] = V2<T>{t2.x + h * d.x, t2.y + h * d.y};
    a[2] = V2<T>{t2.x - h * d.x, t2.y - h * d.y};
  } else if constexpr (R == 4) {
    const V2<T> s0 = cadd(a[0], a[2]), s1 = csub(a[0], a[2]);
    const V2<T> s2 = cadd(a[1], a[3]), s3 = rot<T, INV>(csub(a[1], a[3]));
    a[0] = cadd(s0, s2);
    a[2] = csub(s0, s2);
    a[1] = cadd(s1, s3);
    a[3] = csub(s1, s3);
  } else {
    constexpr int P = (R % 4 == 0) ? 4 : ((R % 2 == 0) ? 2 : 3);
    constexpr int Q = R / P;
    static_assert(96 % R == 0, "register DFT sizes divide 96");
    V2<T> b[P][Q];
#pragma unroll
    for (int p = 0; p < P; ++p)
#pragma unroll
      for (int m = 0; m < Q; ++m) b[p][m] = a[P * m + p];
#pragma unroll
    for (int p = 0; p < P; ++p) dft<T, Q, INV>(b[p]);
#pragma unroll
    for (int p = 1; p < P; ++p)
#pragma unroll
      for (int m = 1; m < Q; ++m) {
        const V2<T> w = w96<T>(((p * m) % R) * (96 / R));
        b[p][m] = INV ? cmulc(b[p][m], w) : cmul(b[p][m], w);
      }
#pragma unroll
    for (int m = 0; m < Q; ++m) {
      V2<T> c[P];
#pragma unroll
      for (int p = 0; p < P; ++p) c[p] = b[p][m];
      dft<T, P, INV>(c);
#pragma unroll
      for (int j = 0; j < P; ++j) a[m + Q * j] = c[j];
    }
  }
}

// Step over n1 (or k1) of every column: positions j*N2 + n2, j < N1.  Forward: DFT,
// then the twiddle W_N^(n2 k1); inverse: DFT only (its twiddle came in step b).
template <typename T, int N1, int N2, bool INV>
__device__ __forceinline__ void xpass_a(V2<T>* __restrict__ s, const V2<T>* __restrict__ tw, int ncol, int NC) {
  for (int i = threadIdx.x; i < N2 * ncol; i += blockDim.x) {
    const int col = i % ncol, n2 = i / ncol;
    V2<T> a[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) a[j] = s[(j * N2 + n2) * NC + col];
    dft<T, N1, INV>(a);
    if (!INV) {
#pragma unroll
      for (int j = 1; j < N1; ++j) a[j] = cmul(a[j], tw[n2 * j]);
    }
#pragma unroll
    for (int j = 0; j < N1; ++j) s[(j * N2 + n2) * NC + col] = a[j];
  }
}

// Step over n2 (or k2) of every column: positions k1*N2 + j, j < N2.  Inverse: DFT,
// then the twiddle W_N^(-n2 k1).
template <typename T, int N1, int N2, bool INV>
__device__ __forceinline__ void xpass_b(V2<T>* __restrict__ s, const V2<T>* __restrict__ tw, int ncol, int NC) {
  for (int i = threadIdx.x; i < N1 * ncol; i += blockDim.x) {
    const int col = i % ncol, k1 = i / ncol;
    V2<T> b[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) b[j] = s[(k1 * N2 + j) * NC + col];
    dft<T, N2, INV>(b);
    if (INV) {
#pragma unroll
      for (int j = 1; j < N2; ++j) b[j] = cmulc(b[j], tw[j * k1]);
    }
#pragma unroll
    for (int j = 0; j < N2; ++j) s[(k1 * N2 + j) * NC + col] = b[j];
  }
}

// Plane CTA: the kz = 0 (blockIdx.x = 0) or kz = nz/2 (blockIdx.x = 1) modes of PP
// row pairs {y, -y}, y = blockIdx.y * PP + p <= ny/2.  Mode k of row y pairs with -k
// of row -y (of the same row when y = -y), and one thread projects each {k, -k}
// pair and writes both, symmetrised as in k_project.  Shared memory: pencils
// [N][6 PP] (column (2 p + r) * 3 + c, r = 0 for y, 1 for -y) and the twiddles.
template <typename T, typename C, int N1, int N2, int PP>
__device__ __forceinline__ void xfft_planes_cta(C* __restrict__ spec, const KParams& k, const C* __restrict__ twN) {
  constexpr int N = N1 * N2;
  constexpr int NC = 6 * PP;
  extern __shared__ __align__(16) unsigned char xfft_smem[];
  V2<T>* s = reinterpret_cast<V2<T>*>(xfft_smem);
  V2<T>* tw = s + N * NC;
  const int h = k.ny / 2;
  const int kz = blockIdx.x == 0 ? 0 : k.nz / 2;  // nz is even on this path
  const int y0 = (int)blockIdx.y * PP;
  const long long xs = (long long)k.ny * k.nzh;
  for (int i = threadIdx.x; i < N; i += blockDim.x) tw[i] = ldt<T>(twN[i]);
  for (int i = threadIdx.x; i < N * NC; i += blockDim.x) {
    const int col = i % NC, x = i / NC, c = col % 3, r = (col / 3) & 1, y = y0 + col / 6;
    const int yr = r ? (k.ny - y) % k.ny : y;
    const bool live = y <= h && !(r && yr == y) &&
                      FCM_INB(c * k.Gc + x * xs + (long long)yr * k.nzh + kz, 3 * k.Gc, BS_SPECTRUM);
    s[x * NC + col] = live ? ldt<T>(spec[c * k.Gc + x * xs + (long long)yr * k.nzh + kz]) : V2<T>{(T)0, (T)0};
  }
  __syncthreads();
  xpass_a<T, N1, N2, false>(s, tw, NC, NC);
  __syncthreads();
  xpass_b<T, N1, N2, false>(s, tw, NC, NC);
  __syncthreads();
  const T ie = (T)k.inv_etaG;
  const double q3 = (double)kz * k.fz;
  for (int i = threadIdx.x; i < N * PP; i += blockDim.x) {
    const int pos = i % N, p = i / N, y = y0 + p;
    if (y > h) continue;
    const int yp = (k.ny - y) % k.ny;
    const bool two = yp != y;
    const int kx = pos / N2 + N1 * (pos % N2);
    const int kxp = (k.nx - kx) % k.nx;
    const int posp = (kxp % N1) * N2 + kxp / N1;
    const int cb = 6 * p, pb = two ? 6 * p + 3 : cb;
    if (kz == 0 && kx == 0 && y == 0) {  // f(0) = 0 and u(0) = 0
#pragma unroll
      for (int c = 0; c < 3; ++c) s[pos * NC + cb + c] = V2<T>{(T)0, (T)0};
      continue;
    }
    if (!two && kxp < kx) continue;  // the partner's thread writes the pair
    V2<T> f[3], u[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) f[c] = s[pos * NC + cb + c];
    project_mode<T>(wavenumber(kx, k.nx, k.fx), wavenumber(y, k.ny, k.fy), q3, f, u, ie);
    if (!two && kxp == kx) {  // self-conjugate mode
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u[c].y = (T)0;
        s[pos * NC + cb + c] = u[c];
      }
      continue;
    }
    V2<T> fp[3], up[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) fp[c] = s[posp * NC + pb + c];
    project_mode<T>(wavenumber(kxp, k.nx, k.fx), wavenumber(yp, k.ny, k.fy), q3, fp, up, ie);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      V2<T> us;
      us.x = (T)0.5 * (u[c].x + up[c].x);
      us.y = (T)0.5 * (u[c].y - up[c].y);
      s[pos * NC + cb + c] = us;
      s[posp * NC + pb + c] = V2<T>{us.x, -us.y};
    }
  }
  __syncthreads();
  xpass_b<T, N1, N2, true>(s, tw, NC, NC);
  __syncthreads();
  xpass_a<T, N1, N2, true>(s, tw, NC, NC);
  __syncthreads();
  for (int i = threadIdx.x; i < N * NC; i += blockDim.x) {
    const int col = i % NC, x = i / NC, c = col % 3, r = (col / 3) & 1, y = y0 + col / 6;
    const int yr = r ? (k.ny - y) % k.ny : y;
    if (y > h || (r && yr == y)) continue;
    const V2<T> v = s[x * NC + col];
    C o;
    o.x = v.x;
    o.y = v.y;
    if (FCM_INB(c * k.Gc + x * xs + (long long)yr * k.nzh + kz, 3 * k.Gc, BS_SPECTRUM))
      spec[c * k.Gc + x * xs + (long long)yr * k.nzh + kz] = o;
  }
}

// One spectrum element (8 bytes FP32, 16 bytes FP64) from global to shared memory
// by an asynchronous copy (cp.async; the element addresses are aligned to their
// size, the rows of nz/2 + 1 elements are not 16-byte aligned in FP32).
template <typename C>
__device__ __forceinline__ void elem_async(C* dst, const C* src) {
  const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
  if constexpr (sizeof(C) == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
}

// Interior CTA (every kz of the chunk except the Hermitian planes): the step over
// n1 transforms the CTA's pencils [N][3 TK] into shared memory (twiddled): for
// N >= 384 they are first copied there by asynchronous copies, all of the CTA's
// loads in flight at once (measured 1% faster at 512 points, slower at 256), for
// shorter pencils each is read straight into registers; after one barrier each
// thread takes one (k1, kz) and runs, without barriers, the forward step over n2
// of the three components, the projection of those N2 modes and the inverse step
// over n2 with its twiddles; after a second barrier the inverse step over n1 goes
// from shared memory to registers to the spectrum.  Twiddles W_N^j are read
// through the cache.
// Asynchronous copies of the pencils of block (y, k0) into s[x][column]; columns
// the CTA does not transform (kz = 0, kz >= nz/2) are not copied and not used.
template <typename T, typename C, int N1, int N2, int TK>
__device__ __forceinline__ void xfft_block_copy(const C* __restrict__ spec, const KParams& k, int y, int k0,
                                                V2<T>* s) {
  constexpr int NC = 3 * TK;
  const int kzn = k.nz / 2;
  const long long xs = (long long)k.ny * k.nzh;
  const long long row = (long long)y * k.nzh + k0;
  for (int i = threadIdx.x; i < N1 * N2 * NC; i += blockDim.x) {
    const int col = i % NC, x = i / NC, kzl = col % TK, c = col / TK;
    const int kz = k0 + kzl;
    const long long e = c * k.Gc + row + kzl + (long long)x * xs;
    if (kz != 0 && kz < kzn && FCM_INB(e, 3 * k.Gc, BS_SPECTRUM))
      elem_async<C>(reinterpret_cast<C*>(s + (size_t)x * NC + col), spec + e);
  }
}

// The three steps of one interior block (y, k0) on shared memory s; with
// FROM_SMEM the block's pencils are already in s (xfft_block_copy), else the
// first step reads them from the spectrum.
template <typename T, typename C, int N1, int N2, int TK, bool FROM_SMEM>
__device__ __forceinline__ void xfft_interior_block(C* __restrict__ spec, const KParams& k,
                                                    const C* __restrict__ twN, int y, int k0, V2<T>* s) {
  constexpr int NC = 3 * TK;
  const int kzn = k.nz / 2;
  const long long xs = (long long)k.ny * k.nzh;  // x stride of the spectrum
  const long long row = (long long)y * k.nzh + k0;
  constexpr bool ASYNC = FROM_SMEM;
  // forward step over n1: item (column, n2), column = c*TK + kz_local
  for (int i = threadIdx.x; i < N2 * NC; i += blockDim.x) {
    const int col = i % NC, n2 = i / NC, kzl = col % TK, c = col / TK;
    const int kz = k0 + kzl;
    const bool mine = kz != 0 && kz < kzn;
    V2<T> a[N1];
    if constexpr (ASYNC) {
      if (!mine) continue;
#pragma unroll
      for (int j = 0; j < N1; ++j) a[j] = s[(j * N2 + n2) * NC + col];
    } else {
      const C* src = spec + c * k.Gc + row + kzl;
#pragma unroll
      for (int j = 0; j < N1; ++j)
        a[j] = (mine && FCM_INB(c * k.Gc + row + kzl + (long long)(j * N2 + n2) * xs, 3 * k.Gc, BS_SPECTRUM))
                   ? ldt<T>(src[(long long)(j * N2 + n2) * xs])
                   : V2<T>{(T)0, (T)0};
    }
    dft<T, N1, false>(a);
#pragma unroll
    for (int j = 1; j < N1; ++j) a[j] = cmul(a[j], ldt<T>(__ldg(&twN[n2 * j])));
#pragma unroll
    for (int j = 0; j < N1; ++j) s[(j * N2 + n2) * NC + col] = a[j];
  }
  __syncthreads();
  // per (k1, kz): forward step over n2, projection, inverse step over n2
  const double q2 = wavenumber(y, k.ny, k.fy);
  const T ie = (T)k.inv_etaG;
  for (int i = threadIdx.x; i < N1 * TK; i += blockDim.x) {
    const int kzl = i % TK, k1 = i / TK;
    const int kz = k0 + kzl;
    if (kz == 0 || kz >= kzn) continue;
    V2<T>* base = s + (k1 * N2) * NC + kzl;
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      V2<T> b[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) b[j] = base[j * NC + c * TK];
      dft<T, N2, false>(b);
#pragma unroll
      for (int j = 0; j < N2; ++j) base[j * NC + c * TK] = b[j];
    }
    const double q3 = (double)kz * k.fz;
#pragma unroll 4
    for (int j = 0; j < N2; ++j) {  // mode kx = k1 + N1*j
      V2<T> f[3], u[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) f[c] = base[j * NC + c * TK];
      project_mode<T>(wavenumber(k1 + N1 * j, k.nx, k.fx), q2, q3, f, u, ie);
#pragma unroll
      for (int c = 0; c < 3; ++c) base[j * NC + c * TK] = u[c];
    }
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      V2<T> b[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) b[j] = base[j * NC + c * TK];
      dft<T, N2, true>(b);
#pragma unroll
      for (int j = 1; j < N2; ++j) b[j] = cmulc(b[j], ldt<T>(__ldg(&twN[j * k1])));
#pragma unroll
      for (int j = 0; j < N2; ++j) base[j * NC + c * TK] = b[j];
    }
  }
  __syncthreads();
  // inverse step over n1: shared memory -> registers -> spectrum
  for (int i = threadIdx.x; i < N2 * NC; i += blockDim.x) {
    const int col = i % NC, n2 = i / NC, kzl = col % TK, c = col / TK;
    const int kz = k0 + kzl;
    if (kz == 0 || kz >= kzn) continue;
    V2<T> a[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) a[j] = s[(j * N2 + n2) * NC + col];
    dft<T, N1, true>(a);
    C* dst = spec + c * k.Gc + row + kzl;
#pragma unroll
    for (int j = 0; j < N1; ++j) {
      C o;
      o.x = a[j].x;
      o.y = a[j].y;
      if (FCM_INB(c * k.Gc + row + kzl + (long long)(j * N2 + n2) * xs, 3 * k.Gc, BS_SPECTRUM))
        dst[(long long)(j * N2 + n2) * xs] = o;
    }
  }
}

template <typename T, typename C, int N1, int N2, int TK>
__device__ __forceinline__ void xfft_interior_cta(C* __restrict__ spec, const KParams& k,
                                                  const C* __restrict__ twN) {
  extern __shared__ __align__(16) unsigned char xfft_smem[];
  V2<T>* s = reinterpret_cast<V2<T>*>(xfft_smem);
  const int y = blockIdx.y;
  const int k0 = (int)blockIdx.x * TK;
  if constexpr (N1 * N2 >= 384) {
    xfft_block_copy<T, C, N1, N2, TK>(spec, k, y, k0, s);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    __syncthreads();
    xfft_interior_block<T, C, N1, N2, TK, true>(spec, k, twN, y, k0, s);
  } else {
    xfft_interior_block<T, C, N1, N2, TK, false>(spec, k, twN, y, k0, s);
  }
}

// Threads per CTA: 256 (an FP32 CTA sized to one pencil DFT per thread and step,
// 384 threads at 256 points, measured slower); 128 for the FP64 interior CTAs,
// whose register-resident pencils take about 150 registers.
// FP32 interior CTAs of the 512-point transform: kz per CTA and threads (8 and 256:
// two CTAs per SM; 4 and 128, four smaller CTAs per SM, made the solve 16% slower).
#ifndef FCM_XFFT512_TK
#define FCM_XFFT512_TK 8
#endif
#ifndef FCM_XFFT512_THREADS
#define FCM_XFFT512_THREADS 256
#endif

template <typename T, int N1, int N2, int TK, bool PLANES>
constexpr int xfft_block() {
  return (sizeof(T) == 8 && !PLANES) ? 128 : (!PLANES && N1 * N2 == 512) ? FCM_XFFT512_THREADS : 256;
}

// CTAs per SM the register allocation must allow: three for the FP32 transforms up
// to 256 points, fewer for the longer ones and for FP64, whose pencils need more
// registers.
template <typename T, int N, int BLOCK, bool PLANES>
constexpr int xfft_min_blocks() {
  return sizeof(T) == 4 ? (N <= 256 ? 3 : (BLOCK == 128 ? 4 : 2)) : (N <= 256 ? 2 : 1);
}

template <typename T, typename C, int N1, int N2, int TK, bool PLANES>
__global__ void __launch_bounds__(xfft_block<T, N1, N2, TK, PLANES>(),
                                  (xfft_min_blocks<T, N1 * N2, xfft_block<T, N1, N2, TK, PLANES>(), PLANES>()))
    k_xfft_project(C* __restrict__ spec, KParams k, const C* __restrict__ twN) {
  if constexpr (PLANES)
    xfft_planes_cta<T, C, N1, N2, TK>(spec, k, twN);
  else
    xfft_interior_cta<T, C, N1, N2, TK>(spec, k, twN);
}

// Batched: blockIdx.z = member gidx[blockIdx.z] of a group of equal grids.
template <typename T, typename C, int P, int N1, int N2, int TK, bool PLANES>
__global__ void __launch_bounds__(xfft_block<T, N1, N2, TK, PLANES>(),
                                  (xfft_min_blocks<T, N1 * N2, xfft_block<T, N1, N2, TK, PLANES>(), PLANES>()))
    k_b_xfft_project(const BMember* __restrict__ mem, const int* __restrict__ gidx, int mask,
                     const C* __restrict__ twN) {
  const BMember& m = mem[gidx[blockIdx.z]];
  if (bskip(m, mask)) return;
  if constexpr (PLANES)
    xfft_planes_cta<T, C, N1, N2, TK>((C*)m.spec[P], m.kp, twN);
  else
    xfft_interior_cta<T, C, N1, N2, TK>((C*)m.spec[P], m.kp, twN);
}

// ------------------------------------------------------------------ (y, z) transforms
// The (y, z) transforms around k_xfft_project for FP32 grids up to 256 points
// along z, replacing cuFFT's R2C / C2R of every x-plane.  z: the real lines are taken two at a time as the
// real and imaginary parts of one complex pencil (the DFTs of the two real lines
// are (Z(k) + conj Z(-k))/2 and (Z(k) - conj Z(-k))/2i), transformed in two
// register steps with one shared-memory exchange, and written as nz/2 + 1 modes per
// line; the inverse assembles Z(k) = A(k) + i B(k) from the two half spectra,
// ignoring the imaginary parts of A, B at kz = 0 and nz/2 as a C2R transform does.
// y: one CTA per (x-plane, TK kz), the step over n1 straight from global memory,
// the step over n2 straight back to it, one barrier between.  Unnormalised, with
// cuFFT's sign convention.

// padded shared-memory index of pencil position pos (one gap after every Z2)
template <int Z2>
__device__ __forceinline__ int zpad(int pos) {
  return pos + pos / Z2;
}

template <int Z1, int Z2>
__device__ __forceinline__ int zpos(int k) {  // position of mode k after the two steps
  return (k % Z1) * Z2 + k / Z1;
}

// Whether the z passes' middle step shares each row between two lanes where it
// would otherwise leave half the CTA idle (Z2 = 2 Z1).
#ifndef FCM_ZFFT_PAIR
#define FCM_ZFFT_PAIR 1
#endif

// The Z2-point DFT of one shared-memory row (positions row[zpad(j)], j < Z2) by a
// pair of lanes (lane and lane ^ 1): lane half h transforms the samples 2m + h
// (Z2/2 points), the odd lane scales its result by W_Z2^k (conjugated for the
// inverse), the pair swaps halves with shuffles and lane h writes outputs
// k + h Z2/2 = E[k] +- W^k O[k].  Both lanes read their samples before either
// writes (the shuffles order them).  With tw, output j > 0 is then scaled by the
// outer twiddle tw[j k1] (conjugated for the inverse) before the store.
template <typename T, int Z2, bool INV, typename C>
__device__ __forceinline__ void pair_dft_row(V2<T>* row, int half, const C* __restrict__ tw, int k1) {
  constexpr int H = Z2 / 2;
  V2<T> a[H];
#pragma unroll
  for (int m = 0; m < H; ++m) a[m] = row[zpad<Z2>(2 * m + half)];
  dft<T, H, INV>(a);
  if (half) {
#pragma unroll
    for (int k = 1; k < H; ++k) {
      const V2<T> w = w96<T>(k * (96 / Z2));
      a[k] = INV ? cmulc(a[k], w) : cmul(a[k], w);
    }
  }
#pragma unroll
  for (int k = 0; k < H; ++k) {
    const V2<T> o{__shfl_xor_sync(0xffffffffu, a[k].x, 1), __shfl_xor_sync(0xffffffffu, a[k].y, 1)};
    V2<T> x = half ? csub(o, a[k]) : cadd(a[k], o);
    const int j = k + half * H;
    if (tw && j > 0) {
      const V2<T> w = ldt<T>(__ldg(&tw[j * k1]));
      x = INV ? cmulc(x, w) : cmul(x, w);
    }
    row[zpad<Z2>(j)] = x;
  }
}

template <typename T, typename C, int Z1, int Z2>
__global__ void __launch_bounds__(256) k_zfft_r2c(const T* __restrict__ in, C* __restrict__ out, long long nlines,
                                                  const C* __restrict__ twZ) {
  constexpr int N = Z1 * Z2;
  constexpr int Q = 256 / Z2;        // complex pencils (two lines each) per CTA
  constexpr int PS = Z1 * (Z2 + 1);  // padded pencil
  extern __shared__ __align__(16) unsigned char zfft_smem[];
  V2<T>* s = reinterpret_cast<V2<T>*>(zfft_smem);
  const long long l0 = (long long)blockIdx.x * 2 * Q;
  for (int i = threadIdx.x; i < Q * Z2; i += blockDim.x) {
    const int p = i / Z2, n2 = i % Z2;
    const long long la = l0 + 2 * p, lb = la + 1;
    V2<T> a[Z1];
#pragma unroll
    for (int j = 0; j < Z1; ++j) {
      const int z = j * Z2 + n2;
      a[j].x = la < nlines ? in[la * N + z] : (T)0;
      a[j].y = lb < nlines ? in[lb * N + z] : (T)0;
    }
    dft<T, Z1, false>(a);
#pragma unroll
    for (int j = 1; j < Z1; ++j) a[j] = cmul(a[j], ldt<T>(__ldg(&twZ[n2 * j])));
#pragma unroll
    for (int j = 0; j < Z1; ++j) s[p * PS + zpad<Z2>(j * Z2 + n2)] = a[j];
  }
  __syncthreads();
  if constexpr (FCM_ZFFT_PAIR && 2 * Q * Z1 == 256 && Z2 % 2 == 0 && 96 % Z2 == 0) {
    // half the threads would have an item: each row is shared by a lane pair
    const int i = threadIdx.x >> 1, p = i / Z1, k1 = i % Z1;
    pair_dft_row<T, Z2, false, C>(s + p * PS + zpad<Z2>(k1 * Z2), threadIdx.x & 1, nullptr, 0);
  } else {
    for (int i = threadIdx.x; i < Q * Z1; i += blockDim.x) {
      const int p = i / Z1, k1 = i % Z1;
      V2<T> b[Z2];
#pragma unroll
      for (int j = 0; j < Z2; ++j) b[j] = s[p * PS + zpad<Z2>(k1 * Z2 + j)];
      dft<T, Z2, false>(b);
#pragma unroll
      for (int j = 0; j < Z2; ++j) s[p * PS + zpad<Z2>(k1 * Z2 + j)] = b[j];
    }
  }
  __syncthreads();
  constexpr int NZH = N / 2 + 1;  // the spectrum's row length (nzh); a constant divisor below
  for (int i = threadIdx.x; i < Q * NZH; i += blockDim.x) {
    const int p = i / NZH, k = i % NZH;
    const long long la = l0 + 2 * p, lb = la + 1;
    const V2<T> zk = s[p * PS + zpad<Z2>(zpos<Z1, Z2>(k))];
    const V2<T> zm = s[p * PS + zpad<Z2>(zpos<Z1, Z2>((N - k) % N))];
    if (la < nlines) {
      C o;
      o.x = (T)0.5 * (zk.x + zm.x);
      o.y = (T)0.5 * (zk.y - zm.y);
      out[la * NZH + k] = o;
    }
    if (lb < nlines) {
      C o;
      o.x = (T)0.5 * (zk.y + zm.y);
      o.y = (T)0.5 * (zm.x - zk.x);
      out[lb * NZH + k] = o;
    }
  }
}

template <typename T, typename C, int Z1, int Z2>
__global__ void __launch_bounds__(256) k_zfft_c2r(const C* __restrict__ in, T* __restrict__ out, long long nlines,
                                                  const C* __restrict__ twZ) {
  constexpr int N = Z1 * Z2;
  constexpr int Q = 256 / Z2;
  constexpr int PS = Z1 * (Z2 + 1);
  extern __shared__ __align__(16) unsigned char zfft_smem[];
  V2<T>* s = reinterpret_cast<V2<T>*>(zfft_smem);
  const long long l0 = (long long)blockIdx.x * 2 * Q;
  // all of a thread's half-spectrum values are loaded before any is stored
  constexpr int NZH = N / 2 + 1, ITEMS = (Q * NZH + 255) / 256;
  V2<T> A[ITEMS], B[ITEMS];
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) {
    const int i = threadIdx.x + 256 * u;
    const int p = i / NZH, k = i % NZH;
    const long long la = l0 + 2 * p, lb = la + 1;
    const bool live = i < Q * NZH;
    A[u] = live && la < nlines ? ldt<T>(in[la * NZH + k]) : V2<T>{(T)0, (T)0};
    B[u] = live && lb < nlines ? ldt<T>(in[lb * NZH + k]) : V2<T>{(T)0, (T)0};
  }
#pragma unroll
  for (int u = 0; u < ITEMS; ++u) {
    const int i = threadIdx.x + 256 * u;
    if (i >= Q * NZH) break;
    const int p = i / NZH, k = i % NZH;
    V2<T> a = A[u], bb = B[u];
    if (k == 0 || 2 * k == N) {
      a.y = (T)0;
      bb.y = (T)0;
    }
    s[p * PS + zpad<Z2>(zpos<Z1, Z2>(k))] = V2<T>{a.x - bb.y, a.y + bb.x};
    if (k > 0 && 2 * k < N) s[p * PS + zpad<Z2>(zpos<Z1, Z2>(N - k))] = V2<T>{a.x + bb.y, bb.x - a.y};
  }
  __syncthreads();
  if constexpr (FCM_ZFFT_PAIR && 2 * Q * Z1 == 256 && Z2 % 2 == 0 && 96 % Z2 == 0) {
    // half the threads would have an item: each row is shared by a lane pair
    const int i = threadIdx.x >> 1, p = i / Z1, k1 = i % Z1;
    pair_dft_row<T, Z2, true, C>(s + p * PS + zpad<Z2>(k1 * Z2), threadIdx.x & 1, twZ, k1);
  } else {
    for (int i = threadIdx.x; i < Q * Z1; i += blockDim.x) {
      const int p = i / Z1, k1 = i % Z1;
      V2<T> b[Z2];
#pragma unroll
      for (int j = 0; j < Z2; ++j) b[j] = s[p * PS + zpad<Z2>(k1 * Z2 + j)];
      dft<T, Z2, true>(b);
#pragma unroll
      for (int j = 1; j < Z2; ++j) b[j] = cmulc(b[j], ldt<T>(__ldg(&twZ[j * k1])));
#pragma unroll
      for (int j = 0; j < Z2; ++j) s[p * PS + zpad<Z2>(k1 * Z2 + j)] = b[j];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Q * Z2; i += blockDim.x) {
    const int p = i / Z2, n2 = i % Z2;
    const long long la = l0 + 2 * p, lb = la + 1;
    V2<T> a[Z1];
#pragma unroll
    for (int j = 0; j < Z1; ++j) a[j] = s[p * PS + zpad<Z2>(j * Z2 + n2)];
    dft<T, Z1, true>(a);
#pragma unroll
    for (int j = 0; j < Z1; ++j) {
      const int z = j * Z2 + n2;
      if (la < nlines) out[la * N + z] = a[j].x;
      if (lb < nlines) out[lb * N + z] = a[j].y;
    }
  }
}

// Whether the y pass's first step loads two items per thread before transforming
// either (where the items divide evenly among the threads); off: at 512 points it
// measured 1% slower.
#ifndef FCM_YFFT_BATCH
#define FCM_YFFT_BATCH 0
#endif

// C2C along y, in place: blockIdx.y = x-plane (3 nx per grid), TK kz per CTA.
// Both directions split NY = Y1 Y2 the same way (input n = j Y2 + n2, output
// k = k1 + Y1 k2): Y1-point DFTs over j, the twiddles W_NY^(n2 k1) (conjugated for
// the inverse), Y2-point DFTs over n2.  The first step reads its pencils straight
// into registers and writes them to shared memory (an asynchronous-copy prologue
// measured slower here), the second writes the result to the spectrum.
template <typename T, typename C, int Y1, int Y2, int TK, bool INV>
__global__ void __launch_bounds__(256) k_yfft(C* __restrict__ spec, int nzh, const C* __restrict__ twY) {
  constexpr int NY = Y1 * Y2;
  extern __shared__ __align__(16) unsigned char yfft_smem[];
  V2<T>* s = reinterpret_cast<V2<T>*>(yfft_smem);  // [NY][TK]
  const int k0 = (int)blockIdx.x * TK;
  C* base = spec + (long long)blockIdx.y * NY * nzh + k0;
  // first step: IPT items per thread when they divide evenly (every item's loads
  // issued before any transform), else one item at a time
  constexpr int IPT = (FCM_YFFT_BATCH && (Y2 * TK) % 256 == 0 && Y2 * TK / 256 <= 2) ? Y2 * TK / 256 : 1;
  for (int i0 = threadIdx.x; i0 < Y2 * TK; i0 += IPT * blockDim.x) {
    V2<T> a[IPT][Y1];
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
      const int i = i0 + u * blockDim.x, kzl = i % TK, n2 = i / TK;
      const bool live = i < Y2 * TK && k0 + kzl < nzh;
#pragma unroll
      for (int j = 0; j < Y1; ++j)
        a[u][j] = live ? ldt<T>(base[(long long)(j * Y2 + n2) * nzh + kzl]) : V2<T>{(T)0, (T)0};
    }
#pragma unroll
    for (int u = 0; u < IPT; ++u) {
      const int i = i0 + u * blockDim.x, kzl = i % TK, n2 = i / TK;
      if (i >= Y2 * TK) break;
      dft<T, Y1, INV>(a[u]);
#pragma unroll
      for (int j = 1; j < Y1; ++j) {
        const V2<T> w = ldt<T>(__ldg(&twY[n2 * j]));
        a[u][j] = INV ? cmulc(a[u][j], w) : cmul(a[u][j], w);
      }
#pragma unroll
      for (int j = 0; j < Y1; ++j) s[(j * Y2 + n2) * TK + kzl] = a[u][j];
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < Y1 * TK; i += blockDim.x) {
    const int kzl = i % TK, k1 = i / TK;
    if (k0 + kzl >= nzh) continue;
    V2<T> b[Y2];
#pragma unroll
    for (int j = 0; j < Y2; ++j) b[j] = s[(k1 * Y2 + j) * TK + kzl];
    dft<T, Y2, INV>(b);
#pragma unroll
    for (int j = 0; j < Y2; ++j) {
      C o;
      o.x = b[j].x;
      o.y = b[j].y;
      base[(long long)(k1 + Y1 * j) * nzh + kzl] = o;
    }
  }
}

// ------------------------------------------------------------------ (y, z) transforms, a CTA per plane
// Grids with ny == nz = N up to 96 points: one (component, x-plane) per CTA, so the
// z and y transforms of a plane take one pass over HBM each way instead of two.
// The CTA's shared memory holds the plane's half spectrum [N][N/2 + 1].  Forward:
// the rows are transformed two at a time (as k_zfft_r2c does) and every mode of a
// pencil (y, y + 1) is stored into the plane buffer: Z(k) at row y, column k for
// k <= N/2, at row y + 1, column N - k above; then the two lines' spectra are
// separated in place, the columns transformed along y and written.  The inverse
// runs the same steps backwards.  The arithmetic is that of k_zfft_* and k_yfft
// step for step.  (Planes of 256 points split over a cluster of 4 CTAs, the modes
// exchanged through distributed shared memory, took 280 us against 174 us for the
// separate passes: two 102 KB CTAs per SM left the phases between barriers latency
// bound at 15% of DRAM throughput.)
template <typename T, typename C, int N1, int N2>
__global__ void __launch_bounds__(256) k_yz_r2c(const T* __restrict__ in, C* __restrict__ out,
                                                const C* __restrict__ twY, const C* __restrict__ twZ) {
  constexpr int N = N1 * N2, KS = N / 2 + 1, PEN = N / 2;
  constexpr int Q = 256 / N2, PS = N1 * (N2 + 1);
  extern __shared__ __align__(16) unsigned char yz_smem[];
  V2<T>* buf = reinterpret_cast<V2<T>*>(yz_smem);  // [N][KS]
  V2<T>* s = buf + N * KS;                         // [Q][PS]
  const long long plane = (long long)blockIdx.x;
  const T* src = in + plane * N * N;
  for (int p0 = 0; p0 < PEN; p0 += Q) {
    for (int i = threadIdx.x; i < Q * N2; i += blockDim.x) {
      const int p = i / N2, n2 = i % N2;
      if (p0 + p >= PEN) continue;
      const T* la = src + (long long)(2 * (p0 + p)) * N;
      V2<T> a[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) a[j] = V2<T>{la[j * N2 + n2], la[N + j * N2 + n2]};
      dft<T, N1, false>(a);
#pragma unroll
      for (int j = 1; j < N1; ++j) a[j] = cmul(a[j], ldt<T>(__ldg(&twZ[n2 * j])));
#pragma unroll
      for (int j = 0; j < N1; ++j) s[p * PS + zpad<N2>(j * N2 + n2)] = a[j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < Q * N1; i += blockDim.x) {
      const int p = i / N1, k1 = i % N1;
      if (p0 + p >= PEN) continue;
      V2<T> b[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) b[j] = s[p * PS + zpad<N2>(k1 * N2 + j)];
      dft<T, N2, false>(b);
      const int y = 2 * (p0 + p);
#pragma unroll
      for (int j = 0; j < N2; ++j) {
        const int k = k1 + N1 * j;
        buf[2 * k <= N ? y * KS + k : (y + 1) * KS + (N - k)] = b[j];
      }
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < (N / 2) * KS; i += blockDim.x) {
    const int q = i / KS, k = i % KS;
    V2<T>* ra = buf + 2 * q * KS + k;
    const V2<T> zk = ra[0];
    const V2<T> zm = (k == 0 || 2 * k == N) ? zk : ra[KS];
    ra[0] = V2<T>{(T)0.5 * (zk.x + zm.x), (T)0.5 * (zk.y - zm.y)};
    ra[KS] = V2<T>{(T)0.5 * (zk.y + zm.y), (T)0.5 * (zm.x - zk.x)};
  }
  __syncthreads();
  for (int i = threadIdx.x; i < N2 * KS; i += blockDim.x) {
    const int k = i % KS, n2 = i / KS;
    V2<T> a[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) a[j] = buf[(j * N2 + n2) * KS + k];
    dft<T, N1, false>(a);
#pragma unroll
    for (int j = 1; j < N1; ++j) a[j] = cmul(a[j], ldt<T>(__ldg(&twY[n2 * j])));
#pragma unroll
    for (int j = 0; j < N1; ++j) buf[(j * N2 + n2) * KS + k] = a[j];
  }
  __syncthreads();
  C* dst = out + plane * N * KS;
  for (int i = threadIdx.x; i < N1 * KS; i += blockDim.x) {
    const int k = i % KS, k1 = i / KS;
    V2<T> b[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) b[j] = buf[(k1 * N2 + j) * KS + k];
    dft<T, N2, false>(b);
#pragma unroll
    for (int j = 0; j < N2; ++j) {
      C o;
      o.x = b[j].x;
      o.y = b[j].y;
      dst[(k1 + N1 * j) * KS + k] = o;
    }
  }
}

template <typename T, typename C, int N1, int N2>
__global__ void __launch_bounds__(256) k_yz_c2r(const C* __restrict__ in, T* __restrict__ out,
                                                const C* __restrict__ twY, const C* __restrict__ twZ) {
  constexpr int N = N1 * N2, KS = N / 2 + 1, PEN = N / 2;
  constexpr int Q = 256 / N2, PS = N1 * (N2 + 1);
  extern __shared__ __align__(16) unsigned char yz_smem[];
  V2<T>* buf = reinterpret_cast<V2<T>*>(yz_smem);
  V2<T>* s = buf + N * KS;
  const long long plane = (long long)blockIdx.x;
  const C* src = in + plane * N * KS;
  for (int i = threadIdx.x; i < N1 * KS; i += blockDim.x) {
    const int k = i % KS, k1 = i / KS;
    V2<T> b[N2];
#pragma unroll
    for (int j = 0; j < N2; ++j) b[j] = ldt<T>(src[(k1 + N1 * j) * KS + k]);
    dft<T, N2, true>(b);
#pragma unroll
    for (int j = 1; j < N2; ++j) b[j] = cmulc(b[j], ldt<T>(__ldg(&twY[j * k1])));
#pragma unroll
    for (int j = 0; j < N2; ++j) buf[(k1 * N2 + j) * KS + k] = b[j];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < N2 * KS; i += blockDim.x) {
    const int k = i % KS, n2 = i / KS;
    V2<T> a[N1];
#pragma unroll
    for (int j = 0; j < N1; ++j) a[j] = buf[(j * N2 + n2) * KS + k];
    dft<T, N1, true>(a);
#pragma unroll
    for (int j = 0; j < N1; ++j) buf[(j * N2 + n2) * KS + k] = a[j];
  }
  __syncthreads();
  // row 2q <- Z(k) = A(k) + i B(k), row 2q + 1 <- Z(N - k), Im A, Im B ignored at kz = 0, N/2
  for (int i = threadIdx.x; i < (N / 2) * KS; i += blockDim.x) {
    const int q = i / KS, k = i % KS;
    V2<T>* ra = buf + 2 * q * KS + k;
    V2<T> a = ra[0], bb = ra[KS];
    if (k == 0 || 2 * k == N) {
      a.y = (T)0;
      bb.y = (T)0;
    }
    ra[0] = V2<T>{a.x - bb.y, a.y + bb.x};
    ra[KS] = V2<T>{a.x + bb.y, bb.x - a.y};
  }
  __syncthreads();
  T* dsts = out + plane * N * N;
  for (int p0 = 0; p0 < PEN; p0 += Q) {
    for (int i = threadIdx.x; i < Q * N1; i += blockDim.x) {
      const int p = i / N1, k1 = i % N1;
      if (p0 + p >= PEN) continue;
      const int y = 2 * (p0 + p);
      V2<T> b[N2];
#pragma unroll
      for (int j = 0; j < N2; ++j) {
        const int k = k1 + N1 * j;
        b[j] = buf[2 * k <= N ? y * KS + k : (y + 1) * KS + (N - k)];
      }
      dft<T, N2, true>(b);
#pragma unroll
      for (int j = 1; j < N2; ++j) b[j] = cmulc(b[j], ldt<T>(__ldg(&twZ[j * k1])));
#pragma unroll
      for (int j = 0; j < N2; ++j) s[p * PS + zpad<N2>(k1 * N2 + j)] = b[j];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < Q * N2; i += blockDim.x) {
      const int p = i / N2, n2 = i % N2;
      if (p0 + p >= PEN) continue;
      V2<T> a[N1];
#pragma unroll
      for (int j = 0; j < N1; ++j) a[j] = s[p * PS + zpad<N2>(j * N2 + n2)];
      dft<T, N1, true>(a);
      T* la = dsts + (long long)(2 * (p0 + p)) * N;
#pragma unroll
      for (int j = 0; j < N1; ++j) {
        la[j * N2 + n2] = a[j].x;
        la[N + j * N2 + n2] = a[j].y;
      }
    }
    __syncthreads();
  }
}

}  // namespace

KParams make_kparams(const Ctx& c) {
  const double PI = 3.14159265358979323846264338327950288;
  KParams k;
  k.nx = c.g.nx; k.ny = c.g.ny; k.nz = c.g.nz; k.nzh = c.g.nzh;
  k.Gc = c.g.Gc;
  k.fx = 2.0 * PI / c.g.Lx;
  k.fy = 2.0 * PI / c.g.Ly;
  k.fz = 2.0 * PI / c.g.Lz;
  k.inv_etaG = 1.0 / (c.p.viscosity * ((double)c.g.nx * (double)c.g.ny * (double)c.g.nz));
  k.slip = c.p.slip_channel;
  return k;
}


// ------------------------------------------------------------------ fused x-transform (host)
// (N1, N2) of the x-transform length n, both divisors of 96 up to 32; false when
// n is not one of the supported lengths.
bool xfft_factor(int n, int* n1, int* n2) {
  static const int tab[][3] = {{8, 2, 4},    {12, 3, 4},   {16, 4, 4},   {24, 4, 6},    {32, 4, 8},
                               {48, 6, 8},   {64, 8, 8},   {96, 8, 12},  {128, 8, 16},  {192, 12, 16},
                               {256, 16, 16}, {384, 16, 24}, {512, 16, 32}};
  for (const auto& t : tab)
    if (t[0] == n) {
      *n1 = t[1];
      *n2 = t[2];
      return true;
    }
  return false;
}

namespace {

// kz per interior CTA: shared memory N * 3 TK elements near 100 KB (two CTAs per
// SM), TK * N1 threads busy in the middle step.  At 256 points in FP32, 12 kz per
// CTA (three CTAs per SM) took 171 us against 129 us with 16.  FP64 beyond 256
// points: 4 kz (98 KB at 512); the autotuner weighs it against the 3D transforms.
template <typename T>
constexpr int xfft_tk(int n) {
  return sizeof(T) == 4 ? (n <= 256 ? 16 : n == 512 ? FCM_XFFT512_TK : 8) : (n <= 256 ? 8 : 4);
}

// Row pairs per plane CTA: one (ny/2 + 1 CTAs per plane; four pairs per CTA left
// most SMs idle at 256 points and took twice as long).
template <typename T>
constexpr int xfft_pairs(int n) {
  return 1;
}

template <typename K>
int xfft_smem_attr(K kernel, size_t smem) {
  FCM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  return FCM_OK;
}

// The interior and plane launches: the context's own spectrum (b == nullptr), or
// the members gidx[0..nm) of a batch group (all with c's grid) when b is given.
template <typename T, int N1, int N2>
int xfft_run(const Ctx& c, typename cplx_t<T>::type* spec, cudaStream_t s, bool prepare, const BatchGeom* b,
             const int* gidx, int nm, int mask) {
  using C = typename cplx_t<T>::type;
  constexpr int N = N1 * N2;
  constexpr int TK = xfft_tk<T>(N);
  constexpr int P = sizeof(T) == 8 ? 0 : 1;
  constexpr int PP = xfft_pairs<T>(N);
  const size_t smem_i = (size_t)N * 3 * TK * sizeof(C);
  const size_t smem_p = (size_t)N * (6 * PP + 1) * sizeof(C);
  if (prepare) {
    FCM_TRY(xfft_smem_attr(k_xfft_project<T, C, N1, N2, TK, false>, smem_i));
    FCM_TRY(xfft_smem_attr(k_xfft_project<T, C, N1, N2, PP, true>, smem_p));
    FCM_TRY(xfft_smem_attr(k_b_xfft_project<T, C, P, N1, N2, TK, false>, smem_i));
    FCM_TRY(xfft_smem_attr(k_b_xfft_project<T, C, P, N1, N2, PP, true>, smem_p));
    return FCM_OK;
  }
  const C* tw = (const C*)(sizeof(T) == 4 ? c.d_xtw32 : c.d_xtw64);
  const int kzn = c.g.nz / 2;
  const unsigned nb = (unsigned)(b ? nm : 1);
  const unsigned pair_ctas = (unsigned)((c.g.ny / 2 + 1 + PP - 1) / PP);
  const dim3 gi((unsigned)((kzn + TK - 1) / TK), (unsigned)c.g.ny, nb), gp(2u, pair_ctas, nb);
  constexpr int BI = xfft_block<T, N1, N2, TK, false>(), BP = xfft_block<T, N1, N2, PP, true>();
  if (b) {
    k_b_xfft_project<T, C, P, N1, N2, TK, false><<<gi, BI, smem_i, s>>>(b->mem, gidx, mask, tw);
    FCM_LAUNCH_CHECK();
    k_b_xfft_project<T, C, P, N1, N2, PP, true><<<gp, BP, smem_p, s>>>(b->mem, gidx, mask, tw);
  } else {
    const KParams k = make_kparams(c);
    k_xfft_project<T, C, N1, N2, TK, false><<<gi, BI, smem_i, s>>>(spec, k, tw);
    FCM_LAUNCH_CHECK();
    k_xfft_project<T, C, N1, N2, PP, true><<<gp, BP, smem_p, s>>>(spec, k, tw);
  }
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// First factor of the 512-point x-transform (32 by default; 16 is the other split).
#ifndef FCM_XFFT512_N1
#define FCM_XFFT512_N1 32
#endif

template <typename T>
int xfft_dispatch(const Ctx& c, typename cplx_t<T>::type* spec, cudaStream_t s, bool prepare,
                  const BatchGeom* b = nullptr, const int* gidx = nullptr, int nm = 0, int mask = 0) {
  switch (c.g.nx) {
    case 8: return xfft_run<T, 2, 4>(c, spec, s, prepare, b, gidx, nm, mask);
    case 12: return xfft_run<T, 3, 4>(c, spec, s, prepare, b, gidx, nm, mask);
    case 16: return xfft_run<T, 4, 4>(c, spec, s, prepare, b, gidx, nm, mask);
    case 24: return xfft_run<T, 4, 6>(c, spec, s, prepare, b, gidx, nm, mask);
    case 32: return xfft_run<T, 4, 8>(c, spec, s, prepare, b, gidx, nm, mask);
    case 48: return xfft_run<T, 6, 8>(c, spec, s, prepare, b, gidx, nm, mask);
    case 64: return xfft_run<T, 8, 8>(c, spec, s, prepare, b, gidx, nm, mask);
    case 96: return xfft_run<T, 8, 12>(c, spec, s, prepare, b, gidx, nm, mask);
    case 128: return xfft_run<T, 8, 16>(c, spec, s, prepare, b, gidx, nm, mask);
    case 192: return xfft_run<T, 12, 16>(c, spec, s, prepare, b, gidx, nm, mask);
    case 256: return xfft_run<T, 16, 16>(c, spec, s, prepare, b, gidx, nm, mask);
    case 384: return xfft_run<T, 16, 24>(c, spec, s, prepare, b, gidx, nm, mask);
    case 512:
      // 32 x 16: the middle step has N1 * TK = 256 items in FP32 (128 in FP64), one
      // per thread (16 x 32 left half the CTA idle there while it ran six 32-point
      // DFTs per item)
      return xfft_run<T, FCM_XFFT512_N1, 512 / FCM_XFFT512_N1>(c, spec, s, prepare, b, gidx, nm, mask);
    default: break;
  }
  set_error("fused x-transform: unsupported length " + std::to_string(c.g.nx));
  return FCM_ERR_INVALID;
}

}  // namespace

// exp(-2 pi i k / 96) into the constant tables of the current device (once per device).
int xfft_tables_init() {
  static std::mutex mu;
  static std::vector<bool> done;
  int dev = 0;
  FCM_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if ((int)done.size() <= dev) done.resize(dev + 1, false);
  if (done[dev]) return FCM_OK;
  const double PI = 3.14159265358979323846264338327950288;
  double2 wd[96];
  float2 wf[96];
  for (int j = 0; j < 96; ++j) {
    wd[j] = make_double2(std::cos(2.0 * PI * j / 96.0), -std::sin(2.0 * PI * j / 96.0));
    wf[j] = make_float2((float)wd[j].x, (float)wd[j].y);
  }
  FCM_CUDA(cudaMemcpyToSymbol(c_w96d, wd, sizeof(wd)));
  FCM_CUDA(cudaMemcpyToSymbol(c_w96f, wf, sizeof(wf)));
  done[dev] = true;
  return FCM_OK;
}

namespace {

// Calls f(integral_constant<N1>, integral_constant<N2>) for a supported length n.
template <typename F>
int with_factors(int n, F&& f) {
  using std::integral_constant;
  switch (n) {
    case 8: return f(integral_constant<int, 2>{}, integral_constant<int, 4>{});
    case 12: return f(integral_constant<int, 3>{}, integral_constant<int, 4>{});
    case 16: return f(integral_constant<int, 4>{}, integral_constant<int, 4>{});
    case 24: return f(integral_constant<int, 4>{}, integral_constant<int, 6>{});
    case 32: return f(integral_constant<int, 4>{}, integral_constant<int, 8>{});
    case 48: return f(integral_constant<int, 6>{}, integral_constant<int, 8>{});
    case 64: return f(integral_constant<int, 8>{}, integral_constant<int, 8>{});
    case 96: return f(integral_constant<int, 8>{}, integral_constant<int, 12>{});
    case 128: return f(integral_constant<int, 8>{}, integral_constant<int, 16>{});
    case 192: return f(integral_constant<int, 12>{}, integral_constant<int, 16>{});
    case 256: return f(integral_constant<int, 16>{}, integral_constant<int, 16>{});
    case 384: return f(integral_constant<int, 16>{}, integral_constant<int, 24>{});
    case 512: return f(integral_constant<int, 16>{}, integral_constant<int, 32>{});
    default: break;
  }
  set_error("(y, z) transforms: unsupported length " + std::to_string(n));
  return FCM_ERR_INVALID;
}

// Dynamic shared memory above the default 48 KB for `kernel`, set once per kernel
// and device (kernels of one signature share the template instance, so the cache
// is keyed by the kernel's address).
template <typename K>
int smem_attr_once(K kernel, size_t smem) {
  if (smem <= 48 * 1024) return FCM_OK;
  static std::mutex mu;
  static std::vector<std::pair<int, const void*>> done;
  int dev = 0;
  FCM_CUDA(cudaGetDevice(&dev));
  const std::pair<int, const void*> key(dev, reinterpret_cast<const void*>(kernel));
  std::lock_guard<std::mutex> lock(mu);
  if (std::find(done.begin(), done.end(), key) == done.end()) {
    FCM_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done.push_back(key);
  }
  return FCM_OK;
}

// z passes of Z1 x Z2 points, Q = 256 / Z2 complex pencils (two real lines each)
// per CTA.
template <typename T, int Z1, int Z2>
int zfft_run(const T* r, typename cplx_t<T>::type* spec, T* r_out, long long nlines, bool inverse,
             const typename cplx_t<T>::type* tw, cudaStream_t s) {
  using C = typename cplx_t<T>::type;
  constexpr int Q = 256 / Z2;
  const size_t smem = (size_t)Q * Z1 * (Z2 + 1) * sizeof(C);
  const unsigned grid = (unsigned)((nlines + 2 * Q - 1) / (2 * Q));
  if (inverse) {
    FCM_TRY(smem_attr_once(k_zfft_c2r<T, C, Z1, Z2>, smem));
    k_zfft_c2r<T, C, Z1, Z2><<<grid, 256, smem, s>>>(spec, r_out, nlines, tw);
  } else {
    FCM_TRY(smem_attr_once(k_zfft_r2c<T, C, Z1, Z2>, smem));
    k_zfft_r2c<T, C, Z1, Z2><<<grid, 256, smem, s>>>(r, spec, nlines, tw);
  }
  FCM_LAUNCH_CHECK();
  return (int)FCM_OK;
}

// At 512 points the split is 32 x 16 (the middle step then has Q Z1 = 512 items, two
// per thread; 16 x 32 left half the CTA idle there), elsewhere the table's.
#ifndef FCM_ZFFT512_Z1
#define FCM_ZFFT512_Z1 16
#endif

template <typename T>
int zfft(const Ctx& c, const T* r, typename cplx_t<T>::type* spec, T* r_out, long long nlines, bool inverse,
         cudaStream_t s) {
  using C = typename cplx_t<T>::type;
  const C* tw = (const C*)c.d_ztw32;
  return with_factors(c.g.nz, [&](auto a, auto b) -> int {
    constexpr int Z1 = decltype(a)::value, Z2 = decltype(b)::value;
    if constexpr (Z1 * Z2 == 512)
      return zfft_run<T, FCM_ZFFT512_Z1, 512 / FCM_ZFFT512_Z1>(r, spec, r_out, nlines, inverse, tw, s);
    else
      return zfft_run<T, Z1, Z2>(r, spec, r_out, nlines, inverse, tw, s);
  });
}

// y pass: 16 kz per CTA (rows of 128 bytes in FP32; the second step has Y1 * 16 =
// 256 items, one per thread, for Y1 = 16); 64 KB of shared memory at 512 points.
template <typename T>
int yfft(const Ctx& c, typename cplx_t<T>::type* spec, int nplanes, bool inverse, cudaStream_t s) {
  using C = typename cplx_t<T>::type;
  const C* tw = (const C*)c.d_ytw32;
  const int nzh = c.g.nzh;
  return with_factors(c.g.ny, [&](auto a, auto b) -> int {
    constexpr int Y1 = decltype(a)::value, Y2 = decltype(b)::value;
    constexpr int TK = 16;
    const size_t smem = (size_t)Y1 * Y2 * TK * sizeof(C);
    const dim3 grid((unsigned)((nzh + TK - 1) / TK), (unsigned)nplanes);
    if (inverse) {
      FCM_TRY(smem_attr_once(k_yfft<T, C, Y1, Y2, TK, true>, smem));
      k_yfft<T, C, Y1, Y2, TK, true><<<grid, 256, smem, s>>>(spec, nzh, tw);
    } else {
      FCM_TRY(smem_attr_once(k_yfft<T, C, Y1, Y2, TK, false>, smem));
      k_yfft<T, C, Y1, Y2, TK, false><<<grid, 256, smem, s>>>(spec, nzh, tw);
    }
    FCM_LAUNCH_CHECK();
    return (int)FCM_OK;
  });
}

// One launch of the per-plane kernels over `planes` (component, x-plane) planes of
// grids with ny == nz = N1 N2, or (prepare) their shared-memory attribute.
template <int N1, int N2>
int yz_plane_go(const Ctx& c, const float* r, cufftComplex* spec, float* r_out, long long planes, bool inverse,
                cudaStream_t s, bool prepare) {
  using C = cufftComplex;
  constexpr int N = N1 * N2;
  const size_t smem = ((size_t)N * (N / 2 + 1) + (size_t)(256 / N2) * N1 * (N2 + 1)) * sizeof(C);
  auto kf = k_yz_r2c<float, C, N1, N2>;
  auto ki = k_yz_c2r<float, C, N1, N2>;
  if (prepare) {
    FCM_TRY(xfft_smem_attr(kf, smem));
    return xfft_smem_attr(ki, smem);
  }
  const C* twY = (const C*)c.d_ytw32;
  const C* twZ = (const C*)c.d_ztw32;
  if (inverse)
    ki<<<(unsigned)planes, 256, smem, s>>>(spec, r_out, twY, twZ);
  else
    kf<<<(unsigned)planes, 256, smem, s>>>(r, spec, twY, twZ);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// Square (y, z) planes of these sizes take the per-plane kernels (55 KB of shared
// memory at 96 points, four CTAs per SM).
bool yz_plane_ok(const Ctx& c) {
  switch (c.g.nz) {
    case 16: case 32: case 48: case 64: case 96: return c.g.ny == c.g.nz;
    default: return false;
  }
}

int yz_plane(const Ctx& c, const float* r, cufftComplex* spec, float* r_out, long long planes, bool inverse,
             cudaStream_t s, bool prepare) {
  switch (c.g.nz) {
    case 16: return yz_plane_go<4, 4>(c, r, spec, r_out, planes, inverse, s, prepare);
    case 32: return yz_plane_go<4, 8>(c, r, spec, r_out, planes, inverse, s, prepare);
    case 48: return yz_plane_go<6, 8>(c, r, spec, r_out, planes, inverse, s, prepare);
    case 64: return yz_plane_go<8, 8>(c, r, spec, r_out, planes, inverse, s, prepare);
    case 96: return yz_plane_go<8, 12>(c, r, spec, r_out, planes, inverse, s, prepare);
    default: break;
  }
  set_error("(y, z) plane transforms: unsupported length " + std::to_string(c.g.nz));
  return FCM_ERR_INVALID;
}

}  // namespace

// The (y, z) transforms of `members` consecutive FP32 grids of c's shape: forward
// from the real grid r into the spectrum, inverse from the spectrum (overwritten)
// into r.  Square (y, z) planes up to 96 points take the per-plane kernels, other
// shapes the z and y passes one after the other.
int launch_yz_forward(const Ctx& c, const float* r, cufftComplex* spec, int members, cudaStream_t s) {
  if (yz_plane_ok(c)) return yz_plane(c, r, spec, nullptr, 3LL * c.g.nx * members, false, s, false);
  const long long nlines = 3LL * c.g.nx * c.g.ny * members;
  FCM_TRY(zfft<float>(c, r, spec, nullptr, nlines, false, s));
  return yfft<float>(c, spec, 3 * c.g.nx * members, false, s);
}

int launch_yz_inverse(const Ctx& c, cufftComplex* spec, float* r, int members, cudaStream_t s) {
  if (yz_plane_ok(c)) return yz_plane(c, nullptr, spec, r, 3LL * c.g.nx * members, true, s, false);
  const long long nlines = 3LL * c.g.nx * c.g.ny * members;
  FCM_TRY(yfft<float>(c, spec, 3 * c.g.nx * members, true, s));
  return zfft<float>(c, nullptr, spec, r, nlines, true, s);
}

template <typename T>
int launch_xfft_project(const Ctx& c, typename cplx_t<T>::type* spec, cudaStream_t s) {
  return xfft_dispatch<T>(c, spec, s, false);
}

template <typename T>
int xfft_prepare(const Ctx& c) {
  if constexpr (sizeof(T) == 4)
    if (c.yz32_cap && yz_plane_ok(c)) FCM_TRY(yz_plane(c, nullptr, nullptr, nullptr, 0, false, 0, true));
  return xfft_dispatch<T>(c, nullptr, 0, true);
}

template <typename T>
int b_xfft_project(const BatchGeom& b, const Ctx& c0, const int* gidx, int nm, int mask, cudaStream_t s) {
  return xfft_dispatch<T>(c0, nullptr, s, false, &b, gidx, nm, mask);
}
template int b_xfft_project<double>(const BatchGeom&, const Ctx&, const int*, int, int, cudaStream_t);
template int b_xfft_project<float>(const BatchGeom&, const Ctx&, const int*, int, int, cudaStream_t);

template int launch_xfft_project<double>(const Ctx&, cufftDoubleComplex*, cudaStream_t);
template int launch_xfft_project<float>(const Ctx&, cufftComplex*, cudaStream_t);
template int xfft_prepare<double>(const Ctx&);
template int xfft_prepare<float>(const Ctx&);

template <typename T>
int launch_project(const Ctx& c, typename cplx_t<T>::type* spec, cudaStream_t s) {
  const KParams k = make_kparams(c);
  const int nt = 256;
  k_project<T, typename cplx_t<T>::type><<<(unsigned)((k.Gc + nt - 1) / nt), nt, 0, s>>>(spec, k);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// Standard deviations of the stress (fcm_fluid_solver.cpp:169-170):
// var1 = sqrt(2 kT eta / (DX^3 dt)) off-diagonal, var2 = sqrt(2) var1 diagonal.
static void stress_amplitudes(const Ctx& c, double& diag, double& off) {
  const double dx = c.g.dx;
  const double var1 = sqrt(2.0 * c.p.kT * c.p.viscosity / (dx * dx * dx * c.p.dt));
  const double var2 = sqrt(2.0) * var1;
  const double G = (double)c.g.G;
  // complex modes: real and imaginary parts each carry G v^2 / 2
  diag = var2 * sqrt(0.5 * G);
  off = var1 * sqrt(0.5 * G);
}

template <typename T>
int launch_noise_kspace(const Ctx& c, typename cplx_t<T>::type* spec, uint64_t seed, uint64_t counter,
                        const uint64_t* d_args, cudaStream_t s) {
  const KParams k = make_kparams(c);
  double ad, ao;
  stress_amplitudes(c, ad, ao);
  const int nt = 256;
  k_fluct<T, typename cplx_t<T>::type, 1><<<(unsigned)((k.Gc + nt - 1) / nt), nt, 0, s>>>(spec, nullptr, k, seed,
                                                                                          counter, d_args, ad, ao);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int launch_stress_divergence_project(const Ctx& c, const cufftDoubleComplex* sigma6, cufftDoubleComplex* spec,
                                     cudaStream_t s) {
  const KParams k = make_kparams(c);
  const int nt = 256;
  k_fluct<double, cufftDoubleComplex, 0><<<(unsigned)((k.Gc + nt - 1) / nt), nt, 0, s>>>(spec, sigma6, k, 0, 0,
                                                                                         nullptr, 0, 0);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// Body force of the imposed shear flow (fcm_fluid_solver.cpp:713-734): fx takes
// the value row[j] of its y index everywhere, fy = fz = 0.
__global__ void k_shear_forcing(const double* __restrict__ row, double* __restrict__ grid, int ny, int nz,
                                long long G) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G; t += (long long)gridDim.x * blockDim.x) {
    const int j = (int)((t / nz) % ny);
    grid[t] = row[j];
    grid[G + t] = 0.0;
    grid[2 * G + t] = 0.0;
  }
}

int launch_shear_forcing(const Ctx& c, const double* d_row, double* grid, cudaStream_t s) {
  const long long G = c.g.G;
  const int nt = 256;
  const long long nb = std::min<long long>((G + nt - 1) / nt, 148LL * 16);
  k_shear_forcing<<<(unsigned)nb, nt, 0, s>>>(d_row, grid, c.g.ny, c.g.nz, G);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// x-velocity profile along y (main.cpp:395-429): one block per y index sums
// u + add over the nx*nz points of that plane, divided by nx*nz.
__global__ void __launch_bounds__(256) k_x_profile(const double* __restrict__ u, const double* __restrict__ add,
                                                   int nx, int ny, int nz, double* __restrict__ out) {
  const int j = blockIdx.x;
  double acc = 0.0;
  for (long long t = threadIdx.x; t < (long long)nx * nz; t += blockDim.x) {
    const int i = (int)(t / nz), k = (int)(t % nz);
    const long long idx = ((long long)i * ny + j) * nz + k;
    acc += u[idx] + (add ? add[idx] : 0.0);
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[j] = red[0] / (double)(nx * nz);
}

int launch_x_profile(const Ctx& c, const double* u, const double* add, double* d_out, cudaStream_t s) {
  k_x_profile<<<(unsigned)c.g.ny, 256, 0, s>>>(u, add, c.g.nx, c.g.ny, c.g.nz, d_out);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template <typename T>
int b_project(const BatchGeom& b, int mask, cudaStream_t s) {
  constexpr int P = sizeof(T) == 8 ? 0 : 1;
  k_b_project<T, typename cplx_t<T>::type, P><<<b.total_kblocks, 256, 0, s>>>(b.mem, b.kblock_map, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template int b_project<double>(const BatchGeom&, int, cudaStream_t);
template int b_project<float>(const BatchGeom&, int, cudaStream_t);
template int launch_project<double>(const Ctx&, cufftDoubleComplex*, cudaStream_t);
template int launch_project<float>(const Ctx&, cufftComplex*, cudaStream_t);
template int launch_noise_kspace<double>(const Ctx&, cufftDoubleComplex*, uint64_t, uint64_t, const uint64_t*,
                                         cudaStream_t);
template int launch_noise_kspace<float>(const Ctx&, cufftComplex*, uint64_t, uint64_t, const uint64_t*, cudaStream_t);

FCM_BOUNDS_READER(bounds_read_kspace)

}  // namespace fcm
