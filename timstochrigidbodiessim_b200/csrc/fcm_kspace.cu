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
  if (bskip(m, mask)) return;
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
  return k;
}


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

}  // namespace fcm
