// fcm_api.cu -- host orchestration and the extern "C" entry points of
// include/fcm_b200.h.  Every entry point catches C++ exceptions, records the
// error text (fcm_last_error) and returns a status code.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "fcm_internal.cuh"

namespace fcm {

// NVTX range over a scope: host-driven steps, refinement sweeps, GMRES iterations
// and the grid stages, for Nsight tools and ncu's --nvtx filters (no cost without a
// tool attached; ranges entered during graph capture mark the capture).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

static thread_local std::string g_err;
void set_error(const std::string& m) { g_err = m; }
static std::atomic<long long> g_launches{0};
static thread_local long long t_launches = 0;  // this thread's launches (graph capture bookkeeping)
void count_launch() {
  g_launches.fetch_add(1, std::memory_order_relaxed);
  ++t_launches;
}
void count_launches(long long n) {
  g_launches.fetch_add(n, std::memory_order_relaxed);
  t_launches += n;
}
long long launch_count() { return t_launches; }

namespace {
bool dense_inv(const std::vector<double>& A, int n, std::vector<double>& out);
}

// Cyclic Jacobi eigen-decomposition of a symmetric n x n matrix (column-major).
static void jacobi_eigen(std::vector<double> A, int n, std::vector<double>& evals, std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
  auto a = [&](int i, int j) -> double& { return A[(size_t)j * n + i]; };
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = i + 1; j < n; ++j) off += a(i, j) * a(i, j);
    if (off < 1e-300) break;
    for (int p = 0; p < n; ++p)
      for (int q = p + 1; q < n; ++q) {
        if (a(p, q) == 0.0) continue;
        const double theta = (a(q, q) - a(p, p)) / (2.0 * a(p, q));
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double cs = 1.0 / std::sqrt(t * t + 1.0), sn = t * cs;
        for (int k = 0; k < n; ++k) {
          const double akp = a(k, p), akq = a(k, q);
          a(k, p) = cs * akp - sn * akq;
          a(k, q) = sn * akp + cs * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a(p, k), aqk = a(q, k);
          a(p, k) = cs * apk - sn * aqk;
          a(q, k) = sn * apk + cs * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double vkp = V[(size_t)p * n + k], vkq = V[(size_t)q * n + k];
          V[(size_t)p * n + k] = cs * vkp - sn * vkq;
          V[(size_t)q * n + k] = sn * vkp + cs * vkq;
        }
      }
  }
  evals.resize(n);
  for (int i = 0; i < n; ++i) evals[i] = a(i, i);
}

// inv() of the reference (Gauss-Jordan) when A is well conditioned; for a
// singular symmetric A -- K^T K and K^T M^{-1} K of a body whose blobs are
// collinear, where spin about the axis moves no blob -- the Moore-Penrose
// pseudo-inverse (eigenvalues below 1e-10 of the largest are dropped).  The
// reference's bodies (twisted rods, tetrahedra, hedgehogs) never reach the
// second branch.
bool sym_inv_or_pinv(const std::vector<double>& A, int n, std::vector<double>& out, bool* used_pinv) {
  std::vector<double> ev, V;
  jacobi_eigen(A, n, ev, V);
  double mx = 0.0;
  for (double e : ev) mx = std::max(mx, std::fabs(e));
  bool singular = !(mx > 0.0);
  for (double e : ev)
    if (std::fabs(e) <= 1e-10 * mx) singular = true;
  if (used_pinv) *used_pinv = singular;
  if (!singular) return dense_inv(A, n, out);
  out.assign((size_t)n * n, 0.0);
  for (int k = 0; k < n; ++k) {
    if (!(std::fabs(ev[k]) > 1e-10 * mx)) continue;
    const double inv = 1.0 / ev[k];
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) out[(size_t)j * n + i] += V[(size_t)k * n + i] * inv * V[(size_t)k * n + j];
  }
  return true;
}

namespace {

const double PI = 3.14159265358979323846264338327950288;

// ------------------------------------------------------------------ helpers
// True for memory the kernels of the current device may use in place: device
// memory of the current device, or managed memory.  Device memory of another GPU
// is not: it goes through the copy path (cudaMemcpyDefault copies between
// devices), so no kernel of this device dereferences another GPU's memory.
bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  if (a.type != cudaMemoryTypeDevice) return false;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.device == dev;
}

int copy_in(Ctx* c, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return FCM_OK;
  if (!src) {
    set_error("null input pointer");
    return FCM_ERR_INVALID;
  }
  FCM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
  return FCM_OK;
}

int copy_out(Ctx* c, void* dst, const void* src, size_t bytes) {
  if (!dst || bytes == 0) return FCM_OK;
  FCM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, c->stream));
  if (!is_device_ptr(dst)) FCM_CUDA(cudaStreamSynchronize(c->stream));
  return FCM_OK;
}

template <typename T>
int dev_alloc(T** p, size_t n) {
  if (cudaMalloc((void**)p, sizeof(T) * (n > 0 ? n : 1)) != cudaSuccess) {
    cudaGetLastError();
    set_error("cudaMalloc of " + std::to_string(sizeof(T) * n) + " bytes failed");
    return FCM_ERR_NOMEM;
  }
  return FCM_OK;
}

// Dense helpers (column-major) for the reference matrices: inv() by
// Gauss-Jordan with partial pivoting, inv_sympd() by Cholesky.
bool dense_inv(const std::vector<double>& A, int n, std::vector<double>& out) {
  std::vector<double> a = A;
  out.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) out[(size_t)i * n + i] = 1.0;
  auto at = [n](std::vector<double>& M, int i, int j) -> double& { return M[(size_t)j * n + i]; };
  for (int col = 0; col < n; ++col) {
    int piv = col;
    for (int r = col + 1; r < n; ++r)
      if (std::fabs(at(a, r, col)) > std::fabs(at(a, piv, col))) piv = r;
    if (at(a, piv, col) == 0.0) return false;
    if (piv != col)
      for (int j = 0; j < n; ++j) {
        std::swap(at(a, col, j), at(a, piv, j));
        std::swap(at(out, col, j), at(out, piv, j));
      }
    const double d = at(a, col, col);
    for (int j = 0; j < n; ++j) {
      at(a, col, j) /= d;
      at(out, col, j) /= d;
    }
    for (int r = 0; r < n; ++r) {
      if (r == col) continue;
      const double f = at(a, r, col);
      if (f == 0.0) continue;
      for (int j = 0; j < n; ++j) {
        at(a, r, j) -= f * at(a, col, j);
        at(out, r, j) -= f * at(out, col, j);
      }
    }
  }
  return true;
}

bool dense_inv_sympd(const std::vector<double>& A, int n, std::vector<double>& out) {
  std::vector<double> L((size_t)n * n, 0.0), Li((size_t)n * n, 0.0);
  auto a = [&](int i, int j) { return A[(size_t)j * n + i]; };
  auto l = [&](int i, int j) -> double& { return L[(size_t)j * n + i]; };
  auto li = [&](int i, int j) -> double& { return Li[(size_t)j * n + i]; };
  for (int j = 0; j < n; ++j) {
    double d = a(j, j);
    for (int k = 0; k < j; ++k) d -= l(j, k) * l(j, k);
    if (!(d > 0.0)) return false;
    const double ljj = std::sqrt(d);
    l(j, j) = ljj;
    for (int i = j + 1; i < n; ++i) {
      double s = a(i, j);
      for (int k = 0; k < j; ++k) s -= l(i, k) * l(j, k);
      l(i, j) = s / ljj;
    }
  }
  for (int j = 0; j < n; ++j) {
    li(j, j) = 1.0 / l(j, j);
    for (int i = j + 1; i < n; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s -= l(i, k) * li(k, j);
      li(i, j) = s / l(i, i);
    }
  }
  out.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (int k = i; k < n; ++k) s += li(k, i) * li(k, j);
      out[(size_t)j * n + i] = s;
      out[(size_t)i * n + j] = s;
    }
  return true;
}

// K of the reference shape, (3nb) x 6 column-major: rows 3m..3m+2 = [I, rcross(r_m)]
// (rcross.cpp:5-9: rcross(x) = {{0,x2,-x1},{-x2,0,x0},{x1,-x0,0}}).
std::vector<double> reference_K(const std::vector<double>& ref, int nb) {
  const int n3 = 3 * nb;
  std::vector<double> K((size_t)n3 * 6, 0.0);
  for (int m = 0; m < nb; ++m) {
    const double* x = &ref[3 * m];
    const double C[3][3] = {{0, x[2], -x[1]}, {-x[2], 0, x[0]}, {x[1], -x[0], 0}};
    for (int d = 0; d < 3; ++d) K[(size_t)d * n3 + 3 * m + d] = 1.0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) K[(size_t)(3 + j) * n3 + 3 * m + i] = C[i][j];
  }
  return K;
}

// K^T K of a shape (6x6, column-major).
std::vector<double> shape_KTK(const std::vector<double>& K, int nb) {
  const int n3 = 3 * nb;
  std::vector<double> KTK(36, 0.0);
  for (int i = 0; i < 6; ++i)
    for (int j = 0; j < 6; ++j) {
      double s = 0.0;
      for (int t = 0; t < n3; ++t) s += K[(size_t)i * n3 + t] * K[(size_t)j * n3 + t];
      KTK[(size_t)j * 6 + i] = s;
    }
  return KTK;
}

// Free-space FCM mobility between two blobs whose force envelopes are Gaussians of
// variance sigma^2 = a^2/pi per dimension (the envelope of fcm_fluid_solver.cpp:
// 135-136).  The Stokes flow of one Gaussian force density, averaged over the
// other Gaussian, is the Stokeslet regularised by a Gaussian of variance
// s^2 = 2 sigma^2.  Writing u = (1/eta)(-phi I + grad grad psi) F with
// lap phi = Gaussian and lap psi = phi gives
//   M(r) = [A(r) I + B(r) r r^T / r^2] / (8 pi eta r),
//   A = (1 + s^2/r^2) erf(r / (sqrt2 s)) - sqrt(2/pi) (s/r) exp(-r^2 / (2 s^2)),
//   B = (1 - 3 s^2/r^2) erf(r / (sqrt2 s)) + 3 sqrt(2/pi) (s/r) exp(-r^2 / (2 s^2)),
// which tends to the Oseen tensor far away and to I / (6 pi eta a) as r -> 0.
void fcm_pair_mobility(const double* d, double a, double eta, double out[3][3]) {
  const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
  const double s = std::sqrt(2.0) * a / std::sqrt(PI);
  const double self = 1.0 / (6.0 * PI * eta * a);
  if (r2 < 1e-20 * s * s) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) out[i][j] = i == j ? self : 0.0;
    return;
  }
  const double r = std::sqrt(r2), sr = s / r, x = r / (std::sqrt(2.0) * s);
  const double er = std::erf(x), ex = std::sqrt(2.0 / PI) * sr * std::exp(-x * x);
  const double A = (1.0 + sr * sr) * er - ex, B = (1.0 - 3.0 * sr * sr) * er + 3.0 * ex;
  const double f = 1.0 / (8.0 * PI * eta * r);
  for (int i = 0; i < 3; ++i)
    for (int j = 0; j < 3; ++j) out[i][j] = f * ((i == j ? A : 0.0) + B * d[i] * d[j] / r2);
}

// Preconditioner blocks of one body shape (body frame): ref_Minv = inverse of the
// shape's blob-blob mobility (fcm_pair_mobility between every pair of its blobs),
// ref_N = inv(K^T ref_Minv K) and ref_KTKinv = inv(K^T K)
// (collection_of_rigid_bodies.cpp:117-130, fcm_fluid_solver.cpp:866-877 with the
// analytic mobility in place of the probed one).
bool body_preconditioner(const double* shape, int nb, double a, double eta, double* Minv_out, double* N_out,
                         double* KTKinv_out) {
  const int n3 = 3 * nb;
  std::vector<double> ref(shape, shape + n3), Mb((size_t)n3 * n3), Minv, N, KTKinv;
  for (int i = 0; i < nb; ++i)
    for (int j = 0; j < nb; ++j) {
      const double d[3] = {ref[3 * i] - ref[3 * j], ref[3 * i + 1] - ref[3 * j + 1], ref[3 * i + 2] - ref[3 * j + 2]};
      double m[3][3];
      fcm_pair_mobility(d, a, eta, m);
      for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) Mb[(size_t)(3 * j + q) * n3 + 3 * i + p] = m[p][q];
    }
  if (!dense_inv_sympd(Mb, n3, Minv)) return false;
  const std::vector<double> K = reference_K(ref, nb);
  std::vector<double> KtMK(36, 0.0), t(n3);
  for (int j = 0; j < 6; ++j) {
    for (int i = 0; i < n3; ++i) {
      double sum = 0.0;
      for (int k = 0; k < n3; ++k) sum += Minv[(size_t)k * n3 + i] * K[(size_t)j * n3 + k];
      t[i] = sum;
    }
    for (int i = 0; i < 6; ++i) {
      double sum = 0.0;
      for (int r = 0; r < n3; ++r) sum += K[(size_t)i * n3 + r] * t[r];
      KtMK[(size_t)j * 6 + i] = sum;
    }
  }
  if (!sym_inv_or_pinv(KtMK, 6, N, nullptr)) return false;
  if (!sym_inv_or_pinv(shape_KTK(K, nb), 6, KTKinv, nullptr)) return false;
  std::copy(Minv.begin(), Minv.end(), Minv_out);
  std::copy(N.begin(), N.end(), N_out);
  std::copy(KTKinv.begin(), KTKinv.end(), KTKinv_out);
  return true;
}

// f(lo, hi) over [0, n) on the host's hardware threads.
template <class F>
void parallel_ranges(long long n, F&& f) {
  const int nt = (int)std::max(1u, std::min(64u, std::thread::hardware_concurrency()));
  if (nt == 1 || n < 64) {
    f(0LL, n);
    return;
  }
  std::vector<std::thread> th;
  const long long chunk = (n + nt - 1) / nt;
  for (int t = 0; t < nt; ++t) {
    const long long lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo < hi) th.emplace_back([&f, lo, hi] { f(lo, hi); });
  }
  for (auto& x : th) x.join();
}

// ------------------------------------------------------------------ cuFFT exec
inline cufftResult exec_r2c(cufftHandle p, double* in, cufftDoubleComplex* out) { return cufftExecD2Z(p, in, out); }
inline cufftResult exec_r2c(cufftHandle p, float* in, cufftComplex* out) { return cufftExecR2C(p, in, out); }
inline cufftResult exec_c2r(cufftHandle p, cufftDoubleComplex* in, double* out) { return cufftExecZ2D(p, in, out); }
inline cufftResult exec_c2r(cufftHandle p, cufftComplex* in, float* out) { return cufftExecC2R(p, in, out); }
template <typename T>
cufftType r2c_type();
template <>
cufftType r2c_type<double>() { return CUFFT_D2Z; }
template <>
cufftType r2c_type<float>() { return CUFFT_R2C; }
template <typename T>
cufftType c2r_type();
template <>
cufftType c2r_type<double>() { return CUFFT_Z2D; }
template <>
cufftType c2r_type<float>() { return CUFFT_C2R; }

template <typename T>
GridBufs<T>& grid_of(Ctx* c);
template <>
GridBufs<double>& grid_of<double>(Ctx* c) { return c->g64; }
template <>
GridBufs<float>& grid_of<float>(Ctx* c) { return c->g32; }

// Stencil width of the FP32 tables: the reference's W, narrowed to the smallest
// even width whose excluded points all lie at least 5.5 sigma from the blob
// (a W-point stencil starting at int(Y/DX) - W/2 + 1 excludes only points W/2
// or more grid spacings away).  The Gaussian mass beyond 5.5 sigma is 3.8e-8 of
// the total per dimension, below FP32 rounding; the FP64 residual of the
// refinement keeps the full W.
int fp32_stencil(const Ctx* c) {
  const double PI = 3.14159265358979323846264338327950288;
  const double sigma = c->p.blob_radius / std::sqrt(PI);
  const int half = (int)std::ceil(5.5 * sigma / c->g.dx);
  return std::min(c->p.ngauss, std::max(2, 2 * half));
}

// The fused x-transform path of the Stokes solve (stokes_t) when nx has a kernel
// and nz is even -- for FP64 only up to 256 points, where it measured faster than
// the 3D transforms (at 512^3 FP64 it was slower) -- and the twiddles
// exp(-2 pi i j / nx) of both precisions.
int setup_xfft(Ctx* c) {
  int n1 = 0, n2 = 0;
  const bool ok = xfft_factor(c->g.nx, &n1, &n2) && c->g.nz % 2 == 0;
  c->xfft[1] = ok;
  c->xfft[0] = ok && c->g.nx <= 256;  // FP64 beyond 256 points: the 3D transforms unless tuned
  c->xfft_cap[0] = ok;
  c->xfft_cap[1] = c->xfft[1];
  if (!ok) return FCM_OK;
  FCM_TRY(xfft_tables_init());
  const int n = c->g.nx;
  const double PI = 3.14159265358979323846264338327950288;
  std::vector<double2> wd(n);
  std::vector<float2> wf(n);
  for (int j = 0; j < n; ++j) {
    wd[j] = make_double2(std::cos(2.0 * PI * j / n), -std::sin(2.0 * PI * j / n));
    wf[j] = make_float2((float)wd[j].x, (float)wd[j].y);
  }
  double2* d64 = nullptr;
  float2* d32 = nullptr;
  FCM_TRY(dev_alloc(&d64, (size_t)n));
  c->d_xtw64 = d64;
  FCM_TRY(dev_alloc(&d32, (size_t)n));
  c->d_xtw32 = d32;
  FCM_CUDA(cudaMemcpy(d64, wd.data(), sizeof(double2) * n, cudaMemcpyHostToDevice));
  FCM_CUDA(cudaMemcpy(d32, wf.data(), sizeof(float2) * n, cudaMemcpyHostToDevice));
  // FP32 (y, z) transforms by the library's kernels, where they beat cuFFT's 2D
  // plans: 64^3, 96^3 (the 64-suspension ensemble ran 11% faster), 256^3 (328
  // against 364 us per solve) and, with 16 kz per y CTA, 512^3 (the whole FP32 solve
  // 4091 against 4477 us)
  c->yz32_cap = xfft_factor(c->g.ny, &n1, &n2) && xfft_factor(c->g.nz, &n1, &n2) && 3 * c->g.nx <= 65535;
  c->yz32 = c->yz32_cap;
  if (c->yz32_cap) {
    for (int d = 0; d < 2; ++d) {
      const int m = d == 0 ? c->g.ny : c->g.nz;
      std::vector<float2> w(m);
      for (int j = 0; j < m; ++j)
        w[j] = make_float2((float)std::cos(2.0 * PI * j / m), (float)-std::sin(2.0 * PI * j / m));
      float2* dw = nullptr;
      FCM_TRY(dev_alloc(&dw, (size_t)m));
      (d == 0 ? c->d_ytw32 : c->d_ztw32) = dw;
      FCM_CUDA(cudaMemcpy(dw, w.data(), sizeof(float2) * m, cudaMemcpyHostToDevice));
    }
  }
  return FCM_OK;
}

template <typename T>
int ensure_grid(Ctx* c) {
  GridBufs<T>& gb = grid_of<T>(c);
  if (gb.ready) return FCM_OK;
  FCM_TRY(dev_alloc(&gb.r, 3 * (size_t)c->g.G));
  FCM_TRY(dev_alloc(&gb.c, 3 * (size_t)c->g.Gc));
  FCM_TRY(dev_alloc(&gb.urand, 3 * (size_t)c->g.G));
  FCM_CUDA(cudaMemsetAsync(gb.urand, 0, sizeof(T) * 3 * (size_t)c->g.G, c->stream));
  int n[3] = {c->g.nx, c->g.ny, c->g.nz};
  FCM_CUFFT(cufftPlanMany(&gb.r2c, 3, n, nullptr, 1, (int)c->g.G, nullptr, 1, (int)c->g.Gc, r2c_type<T>(), 3));
  FCM_CUFFT(cufftPlanMany(&gb.c2r, 3, n, nullptr, 1, (int)c->g.Gc, nullptr, 1, (int)c->g.G, c2r_type<T>(), 3));
  FCM_CUFFT(cufftSetStream(gb.r2c, c->stream));
  FCM_CUFFT(cufftSetStream(gb.c2r, c->stream));
  if (c->xfft_cap[sizeof(T) == 8 ? 0 : 1]) {  // (y, z) transforms of the 3 nx planes of each component
    int n2[2] = {c->g.ny, c->g.nz};
    const int planes = 3 * c->g.nx;
    FCM_CUFFT(cufftPlanMany(&gb.r2c2d, 2, n2, nullptr, 1, c->g.ny * c->g.nz, nullptr, 1, c->g.ny * c->g.nzh,
                            r2c_type<T>(), planes));
    FCM_CUFFT(cufftPlanMany(&gb.c2r2d, 2, n2, nullptr, 1, c->g.ny * c->g.nzh, nullptr, 1, c->g.ny * c->g.nz,
                            c2r_type<T>(), planes));
    FCM_CUFFT(cufftSetStream(gb.r2c2d, c->stream));
    FCM_CUFFT(cufftSetStream(gb.c2r2d, c->stream));
    FCM_TRY(xfft_prepare<T>(*c));
  }
  const int W = sizeof(T) == 4 ? fp32_stencil(c) : c->p.ngauss;
  FCM_TRY(blob_table_alloc(gb.blobs, c->Nb, W, c->g));
  FCM_TRY(blob_table_alloc(gb.ref_blobs, c->nb, W, c->g));
  gb.ready = true;
  return FCM_OK;
}

template <typename T>
void free_grid(GridBufs<T>& gb) {
  if (!gb.borrowed) {
    cudaFree(gb.r);
    cudaFree(gb.c);
    cudaFree(gb.urand);
  }
  if (gb.r2c) cufftDestroy(gb.r2c);
  if (gb.c2r) cufftDestroy(gb.c2r);
  if (gb.r2c2d) cufftDestroy(gb.r2c2d);
  if (gb.c2r2d) cufftDestroy(gb.c2r2d);
  blob_table_free(gb.blobs);
  blob_table_free(gb.ref_blobs);
  gb = GridBufs<T>();
}

int set_stream_all(Ctx* c) {
  if (c->g64.ready) {
    FCM_CUFFT(cufftSetStream(c->g64.r2c, c->stream));
    FCM_CUFFT(cufftSetStream(c->g64.c2r, c->stream));
    if (c->g64.r2c2d) FCM_CUFFT(cufftSetStream(c->g64.r2c2d, c->stream));
    if (c->g64.c2r2d) FCM_CUFFT(cufftSetStream(c->g64.c2r2d, c->stream));
  }
  if (c->g32.ready) {
    FCM_CUFFT(cufftSetStream(c->g32.r2c, c->stream));
    FCM_CUFFT(cufftSetStream(c->g32.c2r, c->stream));
    if (c->g32.r2c2d) FCM_CUFFT(cufftSetStream(c->g32.r2c2d, c->stream));
    if (c->g32.c2r2d) FCM_CUFFT(cufftSetStream(c->g32.c2r2d, c->stream));
  }
  if (c->plan_r2c6) FCM_CUFFT(cufftSetStream(c->plan_r2c6, c->stream));
  return FCM_OK;
}

// ------------------------------------------------------------------ FCM pieces
// Gaussian tables of all blobs from Y (device), FP64 always, FP32 for precision 1.
int set_up_gaussians_dev(Ctx* c, const double* dY) {
  FCM_TRY(launch_set_up_gaussians<double>(*c, c->g64.blobs, dY, c->stream));
  if (c->p.precision == 1) FCM_TRY(launch_set_up_gaussians<float>(*c, c->g32.blobs, dY, c->stream));
  c->gauss_ready = true;
  return FCM_OK;
}

template <typename T>
int spread_t(Ctx* c, const BlobTable<T>& t, const double* dF) {
  NvtxRange r(sizeof(T) == 8 ? "fcm spread fp64" : "fcm spread fp32");
  FCM_TRY(launch_spread<T>(*c, t, dF, grid_of<T>(c).r, c->stream));
  if (c->p.slip_channel) FCM_TRY(launch_slip_image<T>(*c, grid_of<T>(c).r, c->stream));  // :602-632
  return FCM_OK;
}

template <typename T>
int stokes_t(Ctx* c) {
  NvtxRange r(sizeof(T) == 8 ? "fcm stokes solve fp64" : "fcm stokes solve fp32");
  GridBufs<T>& gb = grid_of<T>(c);
  if (c->xfft[sizeof(T) == 8 ? 0 : 1]) {  // (y, z) transforms, then x + projection + inverse x
    if constexpr (sizeof(T) == 4) {
      if (c->yz32) {
        FCM_TRY(launch_yz_forward(*c, gb.r, gb.c, 1, c->stream));
        FCM_TRY(launch_xfft_project<T>(*c, gb.c, c->stream));
        return launch_yz_inverse(*c, gb.c, gb.r, 1, c->stream);
      }
    }
    FCM_CUFFT(exec_r2c(gb.r2c2d, gb.r, gb.c));
    FCM_TRY(launch_xfft_project<T>(*c, gb.c, c->stream));
    FCM_CUFFT(exec_c2r(gb.c2r2d, gb.c, gb.r));
    return FCM_OK;
  }
  FCM_CUFFT(exec_r2c(gb.r2c, gb.r, gb.c));
  FCM_TRY(launch_project<T>(*c, gb.c, c->stream));
  FCM_CUFFT(exec_c2r(gb.c2r, gb.c, gb.r));
  return FCM_OK;
}

template <typename T>
int interp_t(Ctx* c, const BlobTable<T>& t, const T* grid, double* dV) {
  NvtxRange r(sizeof(T) == 8 ? "fcm interp fp64" : "fcm interp fp32");
  return launch_interp<T>(*c, t, grid, dV, c->stream);
}

// V (3Nb, device) = M F with the grid precision `prec`.
int mobility_dev(Ctx* c, int prec, const double* dF, double* dV) {
  if (prec == 0) {
    FCM_TRY(spread_t<double>(c, c->g64.blobs, dF));
    FCM_TRY(stokes_t<double>(c));
    FCM_TRY(interp_t<double>(c, c->g64.blobs, c->g64.r, dV));
  } else {
    FCM_TRY(spread_t<float>(c, c->g32.blobs, dF));
    FCM_TRY(stokes_t<float>(c));
    FCM_TRY(interp_t<float>(c, c->g32.blobs, c->g32.r, dV));
  }
  return FCM_OK;
}

int random_velocities_dev(Ctx* c, double* dV) {
  if (!c->urand_ready) {
    FCM_CUDA(cudaMemsetAsync(dV, 0, sizeof(double) * 3 * (size_t)c->Nb, c->stream));
    return FCM_OK;
  }
  if (c->urand_prec == 0) return interp_t<double>(c, c->g64.blobs, c->g64.urand, dV);
  return interp_t<float>(c, c->g32.blobs, c->g32.urand, dV);
}

// Precision of the random velocity field: FP32 for mixed-precision EM steps; FP64
// otherwise, and for GDC also in mixed precision, whose div(U) differentiates
// random velocities over 1e-5 a (collection_of_rigid_bodies.cpp:869-953), which
// FP32 interpolation rounding would swamp.
int noise_precision(const Ctx* c) { return (c->p.precision == 1 && c->p.algorithm == 2) ? 1 : 0; }

int noise_dev(Ctx* c, uint64_t seed, uint64_t counter, const uint64_t* d_args = nullptr) {
  if (noise_precision(c) == 1) {
    FCM_TRY(launch_noise_kspace<float>(*c, c->g32.c, seed, counter, d_args, c->stream));
    FCM_CUFFT(exec_c2r(c->g32.c2r, c->g32.c, c->g32.urand));
    c->urand_prec = 1;
  } else {
    FCM_TRY(launch_noise_kspace<double>(*c, c->g64.c, seed, counter, d_args, c->stream));
    FCM_CUFFT(exec_c2r(c->g64.c2r, c->g64.c, c->g64.urand));
    c->urand_prec = 0;
  }
  c->urand_ready = true;
  return FCM_OK;
}

// gmres_solver.cpp:72-83 on device vectors (system size).
int saddle_matvec(Ctx* c, int prec, const double* in, double* out) {
  FCM_TRY(mobility_dev(c, prec, in, out));
  FCM_TRY(launch_multiply_K(*c, c->d_qm, in + 3 * (size_t)c->Nb, out, 1.0, c->stream));
  FCM_TRY(launch_multiply_KT(*c, c->d_qm, in, out + 3 * (size_t)c->Nb, -1.0, nullptr, 0.0, c->stream));
  return FCM_OK;
}

// One Arnoldi iteration of the device-side GMRES on c->stream:
//   z_in = Q[k]; z = P^-1 z_in; w = A z; orthogonalise, normalise, Givens.
int enqueue_gm_iteration(Ctx* c, int prec) {
  FCM_TRY(gm_fetch(*c, c->d_sys_b, c->stream));
  FCM_TRY(launch_pinv(*c, c->d_qm, c->d_sys_b, c->d_sys_a, c->stream));
  FCM_TRY(saddle_matvec(c, prec, c->d_sys_a, c->d_sys_b));
  FCM_TRY(gm_orthogonalize(*c, c->d_sys_b, c->stream));
  return FCM_OK;
}

// The Arnoldi iteration captured once per precision in a CUDA graph on the
// private capture stream.
int capture_iteration(Ctx* c, int prec) {
  cudaGraphExec_t& ex = c->iter_graph[prec];
  if (ex) return FCM_OK;
  const cudaStream_t orig = c->stream;
  c->stream = c->cap_stream;
  FCM_TRY(set_stream_all(c));
  int st = FCM_OK;
  cudaGraph_t g = nullptr;
  const long long l0 = launch_count();
  cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = enqueue_gm_iteration(c, prec);
    const cudaError_t e2 = cudaStreamEndCapture(c->cap_stream, &g);
    if (st == FCM_OK && e2 != cudaSuccess) {
      set_error(std::string("GMRES iteration capture: ") + cudaGetErrorString(e2));
      st = FCM_ERR_CUDA;
    }
  } else {
    set_error(std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
    st = FCM_ERR_CUDA;
  }
  // captured kernels are counted when the graph is launched, not here
  c->iter_graph_kernels[prec] = launch_count() - l0;
  count_launches(-(launch_count() - l0));
  if (st == FCM_OK) {
    e = cudaGraphInstantiate(&ex, g, 0);
    if (e != cudaSuccess) {
      set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
      ex = nullptr;
      st = FCM_ERR_CUDA;
    }
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  c->stream = orig;
  const int s2 = set_stream_all(c);
  return st != FCM_OK ? st : s2;
}

// gmres_solver.cpp:148-306 (right preconditioning, Givens, no restarts) on the
// device vector d_b; the solution is written to d_x.  The Krylov basis, the
// Hessenberg matrix, the rotations and the convergence test stay on the device;
// each iteration is one graph launch followed by a 32-byte state read.
int gmres_dev(Ctx* c, int prec, const double* d_b, double* d_x, double tol, int maxit_req, int* iters_out,
              double* rel_out) {
  const long long n = c->nsys;
  const int max_iter = (int)std::max<long long>(1, std::min<long long>(n, std::min(maxit_req, c->maxit_alloc)));
  FCM_TRY(capture_iteration(c, prec));
  FCM_TRY(gm_init(*c, d_b, tol, max_iter, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->h_gm, c->gm, sizeof(GmState), cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  for (int it = 0; it < max_iter && !c->h_gm->done; ++it) {
    NvtxRange r(prec ? "fcm gmres iteration fp32 grid" : "fcm gmres iteration fp64");
    FCM_CUDA(cudaGraphLaunch(c->iter_graph[prec], c->stream));
    count_launches(c->iter_graph_kernels[prec]);
    FCM_CUDA(cudaMemcpyAsync(c->h_gm, c->gm, sizeof(GmState), cudaMemcpyDeviceToHost, c->stream));
    FCM_CUDA(cudaStreamSynchronize(c->stream));
  }
  const GmState g = *c->h_gm;
  if (iters_out) *iters_out = g.k;
  if (rel_out) *rel_out = g.rel;
  if (g.status == FCM_ERR_NONFINITE) {
    set_error(g.k == 0 ? "non-finite right-hand side" : "GMRES residual became non-finite");
    return FCM_ERR_NONFINITE;
  }
  FCM_TRY(gm_finish(*c, c->d_sys_b, c->stream));
  FCM_TRY(launch_pinv(*c, c->d_qm, c->d_sys_b, d_x, c->stream));
  return g.status;
}

// Saddle-point solve of d_rhs into d_soln.  precision 0: one GMRES; precision 1:
// FP64 iterative refinement around FP32-grid GMRES sweeps.
int solve_dev(Ctx* c, const double* d_rhs, double* d_soln, int* iters, double* rel, int* sweeps) {
  const long long n = c->nsys;
  if (c->p.precision == 0) {
    if (sweeps) *sweeps = 1;
    return gmres_dev(c, 0, d_rhs, d_soln, c->p.gmres_tol, c->p.gmres_max_iter, iters, rel);
  }
  // r = b; x = 0; repeat: dx = GMRES32(r); x += dx; r = b - A64 x.
  double* x = d_soln;
  double* res = c->d_res;
  double* dx = c->d_dx;
  FCM_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, c->stream));
  FCM_CUDA(cudaMemcpyAsync(res, d_rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
  FCM_TRY(blas_norm_sq_partial(*c, d_rhs, n, c->d_H, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_H, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  const double nb = c->h_pinned[0];
  int total = 0, sw = 0, st = FCM_OK;
  double relr = 1.0;
  for (sw = 1; sw <= 8; ++sw) {
    NvtxRange r("fcm refinement sweep");
    // The FP32-grid inner solve only has to shrink the current residual by the
    // remaining factor; below ~1e-6 the FP32 operator error dominates anyway.
    const double inner_tol = std::min(0.5, std::max(1e-6, 0.3 * c->p.gmres_tol / relr));
    int it = 0;
    double rr = 0;
    int s = gmres_dev(c, 1, res, dx, inner_tol, c->p.gmres_max_iter, &it, &rr);
    total += it;
    if (s != FCM_OK && s != FCM_ERR_NOT_CONVERGED) return s;
    FCM_TRY(blas_axpby(x, dx, 1.0, 1.0, n, c->stream));
    FCM_TRY(saddle_matvec(c, 0, x, res));
    FCM_TRY(blas_axpby(res, d_rhs, 1.0, -1.0, n, c->stream));
    FCM_TRY(blas_norm_sq_partial(*c, res, n, c->d_H, c->stream));
    FCM_CUDA(cudaMemcpyAsync(c->h_pinned, c->d_H, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FCM_CUDA(cudaStreamSynchronize(c->stream));
    relr = nb > 0 ? c->h_pinned[0] / nb : 0.0;
    if (!std::isfinite(relr)) {
      st = FCM_ERR_NONFINITE;
      break;
    }
    if (relr < c->p.gmres_tol) {
      st = FCM_OK;
      break;
    }
    st = FCM_ERR_NOT_CONVERGED;
  }
  if (iters) *iters = total;
  if (rel) *rel = relr;
  if (sweeps) *sweeps = std::min(sw, 8);
  return st;
}

int calculate_forces_dev(Ctx* c) {
  if (c->p.algorithm == 2) {  // collection_of_rigid_bodies.cpp:625-629
    FCM_CUDA(cudaMemcpyAsync(c->d_xm, c->d_x, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
    FCM_CUDA(cudaMemcpyAsync(c->d_qm, c->d_q, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  }
  FCM_TRY(cells_build(*c, c->stream));
  FCM_TRY(cells_steric_forces(*c, c->d_F, false, c->stream, true));  // + slip-channel walls (:640-662)
  return FCM_OK;
}

int assemble_rhs_dev(Ctx* c) {
  const size_t n3 = 3 * (size_t)c->Nb;
  FCM_CUDA(cudaMemcpyAsync(c->d_rhs, c->d_V, sizeof(double) * n3, cudaMemcpyDeviceToDevice, c->stream));
  FCM_TRY(blas_axpby(c->d_rhs, c->d_rhs, 0.0, -1.0, (long long)n3, c->stream));
  if (c->shear) FCM_TRY(blas_axpby(c->d_rhs, c->d_vshear, -1.0, 1.0, (long long)n3, c->stream));  // :62-64
  FCM_TRY(launch_multiply_KT(*c, c->d_qm, c->d_F, c->d_rhs + n3, -1.0, c->d_fe, -1.0, c->stream));
  return FCM_OK;
}

// fcm_fluid_solver.cpp:489-550: Vshear = J u_shear on the current Gaussians.
int shear_velocities_dev(Ctx* c) {
  return launch_interp<double>(*c, c->g64.blobs, c->d_ushear, c->d_vshear, c->stream);
}

// Overlaps of all_blob_pos: between bodies (check_for_overlap) and, with walls, a
// slip channel's wall contacts (check_for_channel_wall_overlap).
int overlap_dev(Ctx* c, int* ov, bool pairs = true, bool walls = false) {
  if (pairs) FCM_TRY(cells_overlap(*c, c->d_flag, c->stream));
  else FCM_CUDA(cudaMemsetAsync(c->d_flag, 0, sizeof(int), c->stream));
  if (walls) FCM_TRY(cells_wall_overlap(*c, c->d_flag, c->stream));
  int h = 0;
  FCM_CUDA(cudaMemcpyAsync(&h, c->d_flag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  *ov = h;
  return FCM_OK;
}

// The body update scales by nu * dt, with nu read from *d_nu when d_nu is given.
int end_of_step_update_dev(Ctx* c, const double* dU, double nu, int* overlap, const double* d_nu = nullptr) {
  FCM_CUDA(cudaMemcpyAsync(c->d_xs, c->d_x, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->d_qs, c->d_q, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  const double scale = d_nu ? c->p.dt : nu * c->p.dt;
  FCM_TRY(launch_body_update(*c, c->d_x, c->d_q, dU, scale, c->stream, d_nu));
  FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
  FCM_TRY(cells_build(*c, c->stream));
  // collection_of_rigid_bodies.cpp:780-786: wall contact always, body overlap with SKIP_ON_OVERLAP
  int ov = 0;
  if (c->p.skip_on_overlap || c->p.slip_channel)
    FCM_TRY(overlap_dev(c, &ov, c->p.skip_on_overlap != 0, c->p.slip_channel != 0));
  if (overlap) *overlap = ov;
  return FCM_OK;
}

int advance_to_midstep_dev(Ctx* c, const double* dV, int* overlap) {
  FCM_CUDA(cudaMemcpyAsync(c->d_xm, c->d_x, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->d_qm, c->d_q, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_TRY(launch_rigid_projection(*c, c->d_q, dV, c->d_U0, c->stream));
  FCM_TRY(launch_body_update(*c, c->d_xm, c->d_qm, c->d_U0, 0.5 * c->p.dt, c->stream));
  FCM_TRY(launch_fill_blob_pos(*c, c->d_xm, c->d_qm, c->d_Y, c->stream));
  FCM_TRY(cells_build(*c, c->stream));
  // collection_of_rigid_bodies.cpp:611-617
  int ov = 0;
  if (c->p.skip_on_overlap || c->p.slip_channel)
    FCM_TRY(overlap_dev(c, &ov, c->p.skip_on_overlap != 0, c->p.slip_channel != 0));
  if (overlap) *overlap = ov;
  return FCM_OK;
}

// collection_of_rigid_bodies.cpp:869-953 with the sum left in *acc (device).
int divU_enqueue(Ctx* c, double* acc) {
  FCM_CUDA(cudaMemcpyAsync(c->d_xs, c->d_x, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->d_qs, c->d_q, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_CUDA(cudaMemsetAsync(acc, 0, sizeof(double), c->stream));
  for (int i = 0; i < 6; ++i) {
    double e[6] = {0, 0, 0, 0, 0, 0};
    e[i] = (i < 3) ? c->p.fd_delta * c->p.blob_radius : c->p.fd_delta;
    FCM_TRY(launch_body_update_uniform(*c, c->d_x, c->d_q, e, c->stream));
    FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
    FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
    FCM_TRY(random_velocities_dev(c, c->d_V));
    FCM_TRY(launch_rigid_projection(*c, c->d_q, c->d_V, c->d_tmp6, c->stream));
    FCM_TRY(launch_divU_accumulate(*c, c->d_tmp6, c->d_U0, i, e[i], c->d_tmp3, c->stream));
    FCM_TRY(blas_sum_accumulate(*c, c->d_tmp3, c->M, acc, c->stream));
    FCM_CUDA(cudaMemcpyAsync(c->d_x, c->d_xs, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
    FCM_CUDA(cudaMemcpyAsync(c->d_q, c->d_qs, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  }
  return FCM_OK;
}

int divU_dev(Ctx* c, double* out) {
  double* acc = c->d_H + c->maxit_alloc + 1;
  FCM_TRY(divU_enqueue(c, acc));
  FCM_CUDA(cudaMemcpyAsync(c->h_pinned, acc, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  *out = c->h_pinned[0];
  return FCM_OK;
}

// ------------------------------------------------------------------ device-resident step
// The whole time step as one CUDA graph.  The GMRES iterations and the FP64
// refinement sweeps are conditional while-nodes whose conditions the device sets
// from the GMRES state (cudaGraphSetConditional), so a step runs from launch to
// completion with no host round trip; the host reads one StepRecord at the end.
// The per-step inputs (noise seed and step index) are read from device memory.
// Built once per context, after a host-driven step has allocated every buffer.

// Condition of a GMRES while-loop: go on while the solve is not done, for at
// most `limit` iterations of this loop.
__global__ void k_gm_loop_cond(cudaGraphConditionalHandle h, const GmState* __restrict__ gm, StepRecord* sd,
                               int enter, int limit) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (enter) sd->guard = 0;
  else ++sd->guard;
  cudaGraphSetConditional(h, (!gm->done && sd->guard < limit) ? 1u : 0u);
}

__global__ void k_step_begin(StepRecord* sd) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sd->iters = 0;
  sd->sweeps = 0;
  sd->status = FCM_OK;
  sd->guard = 0;
  sd->rel = 0.0;
  sd->divU = 0.0;
  sd->normb = 0.0;
  sd->relr = 1.0;
}

// FP64 solve: record the GMRES result.
__global__ void k_gm_record(StepRecord* sd, const GmState* __restrict__ gm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sd->iters = gm->k;
  sd->sweeps = 1;
  sd->rel = gm->rel;
  sd->status = gm->status;
}

// GDC: nu = 1 + dt/2 divU (main.cpp:265-268), divU = 0 without noise.
__global__ void k_gdc_nu(StepRecord* sd, const double* __restrict__ acc, int noise, double dt, double* __restrict__ nu) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double divU = noise ? *acc : 0.0;
  sd->divU = divU;
  *nu = __dadd_rn(1.0, __dmul_rn(__dmul_rn(0.5, dt), divU));
}

// Refinement loop entry: ||b|| from rs[0], enter the loop.
__global__ void k_ref_enter(cudaGraphConditionalHandle h, StepRecord* sd, const double* __restrict__ rs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sd->normb = rs[0];
  sd->relr = 1.0;
  sd->sweeps = 0;
  sd->iters = 0;
  sd->status = FCM_OK;
  cudaGraphSetConditional(h, 1u);
}

// Inner tolerance of the next FP32-grid sweep: it only has to shrink the
// current residual by the remaining factor (clamped to [1e-6, 0.5]).
__global__ void k_ref_tol(const StepRecord* __restrict__ sd, double tol, double* __restrict__ rs) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  rs[2] = fmin(0.5, fmax(1e-6, 0.3 * tol / sd->relr));
}

// After a sweep: relative residual ||r|| / ||b|| (rs[1] / normb) and the loop
// condition; at most `max_sweeps` sweeps.
__global__ void k_ref_next(cudaGraphConditionalHandle h, StepRecord* sd, const GmState* __restrict__ gm,
                           const double* __restrict__ rs, double tol, int max_sweeps) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  sd->sweeps += 1;
  sd->iters += gm->k;
  unsigned go = 0u;
  if (gm->status == FCM_ERR_NONFINITE) {
    sd->status = FCM_ERR_NONFINITE;
    sd->rel = gm->rel;
  } else {
    const double relr = sd->normb > 0.0 ? rs[1] / sd->normb : 0.0;
    sd->relr = relr;
    sd->rel = relr;
    if (!isfinite(relr)) {
      sd->status = FCM_ERR_NONFINITE;
    } else if (relr < tol) {
      sd->status = FCM_OK;
    } else {
      sd->status = FCM_ERR_NOT_CONVERGED;
      go = sd->sweeps < max_sweeps ? 1u : 0u;
    }
  }
  cudaGraphSetConditional(h, go);
}

constexpr int kMaxSweeps = 8;

// Capture scope: c->stream and the cuFFT plans follow stream `s` until restored.
struct StreamSwap {
  Ctx* c;
  cudaStream_t old;
  StreamSwap(Ctx* c_, cudaStream_t s) : c(c_), old(c_->stream) {
    c->stream = s;
    set_stream_all(c);
  }
  ~StreamSwap() {
    c->stream = old;
    set_stream_all(c);
  }
};

// A conditional while-node appended to the graph being captured on `s`; its
// condition handle `h` must have been created on that graph (new_handle) and set
// by a kernel captured before.  Returns the (empty) body graph.
int add_while_node(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraph_t* body) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  FCM_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
  if (cs != cudaStreamCaptureStatusActive) {
    set_error("step graph: stream is not capturing");
    return FCM_ERR_CUDA;
  }
  cudaGraphNodeParams np = {cudaGraphNodeTypeConditional};
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  FCM_CUDA(cudaGraphAddNode(&node, g, deps, nd, &np));
  *body = np.conditional.phGraph_out[0];
  FCM_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
  return FCM_OK;
}

// A condition handle on the graph being captured on `s`.
int new_handle(cudaStream_t s, cudaGraphConditionalHandle* h) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  cudaGraph_t g = nullptr;
  FCM_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
  if (cs != cudaStreamCaptureStatusActive) {
    set_error("step graph: stream is not capturing");
    return FCM_ERR_CUDA;
  }
  // default 0 at every launch of the owning graph: a loop runs only once a
  // kernel has set its condition
  FCM_CUDA(cudaGraphConditionalHandleCreate(h, g, 0, cudaGraphCondAssignDefault));
  return FCM_OK;
}

// Capture into `body` on stream `bs` whatever `fn` enqueues on c->stream.
template <typename F>
int capture_body(Ctx* c, cudaGraph_t body, cudaStream_t bs, F&& fn) {
  FCM_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  int st = FCM_OK;
  {
    StreamSwap sw(c, bs);
    st = fn();
  }
  cudaGraph_t out = nullptr;
  const cudaError_t e = cudaStreamEndCapture(bs, &out);
  if (st == FCM_OK && e != cudaSuccess) {
    set_error(std::string("step graph body capture: ") + cudaGetErrorString(e));
    st = FCM_ERR_CUDA;
  }
  return st;
}

// GMRES on c->stream as a device loop: init (tolerance `tol`, or *d_tol), the
// iterations as a while-node whose body is captured on `bs`, then the solution
// P^-1 sum y_i q_i into d_x.  *iter_kernels receives the kernels of one iteration.
int enqueue_gmres_loop(Ctx* c, int prec, const double* d_b, double* d_x, double tol, const double* d_tol,
                       cudaStream_t bs, long long* iter_kernels) {
  const long long n = c->nsys;
  const int max_iter =
      (int)std::max<long long>(1, std::min<long long>(n, std::min(c->p.gmres_max_iter, c->maxit_alloc)));
  FCM_TRY(gm_init(*c, d_b, tol, max_iter, c->stream, d_tol));
  cudaGraphConditionalHandle h;
  FCM_TRY(new_handle(c->stream, &h));
  k_gm_loop_cond<<<1, 32, 0, c->stream>>>(h, c->gm, c->d_step, 1, max_iter);
  FCM_LAUNCH_CHECK();
  cudaGraph_t body = nullptr;
  FCM_TRY(add_while_node(c->stream, h, &body));
  const long long l0 = launch_count();
  FCM_TRY(capture_body(c, body, bs, [&] {
    FCM_TRY(enqueue_gm_iteration(c, prec));
    k_gm_loop_cond<<<1, 32, 0, c->stream>>>(h, c->gm, c->d_step, 0, max_iter);
    FCM_LAUNCH_CHECK();
    return (int)FCM_OK;
  }));
  *iter_kernels = launch_count() - l0;
  FCM_TRY(gm_finish(*c, c->d_sys_b, c->stream));
  FCM_TRY(launch_pinv(*c, c->d_qm, c->d_sys_b, d_x, c->stream));
  return FCM_OK;
}

// Enqueue one whole time step (the sequence of fcm_step) on c->stream, with the
// solve as device loops.  Requires skip_on_overlap = 0 (no host decision).
int enqueue_resident_step(Ctx* c, long long* k_top, long long* k_sweep, long long* k_iter) {
  const long long l_start = launch_count();
  long long l_loops = 0;  // kernels captured inside loop bodies
  const bool noise = c->p.noise != 0;
  k_step_begin<<<1, 32, 0, c->stream>>>(c->d_step);
  FCM_LAUNCH_CHECK();
  FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
  if (noise) FCM_TRY(noise_dev(c, 0, 0, c->d_stepargs));
  else c->urand_ready = false;
  FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
  FCM_TRY(random_velocities_dev(c, c->d_V));
  const double* d_nu = nullptr;
  if (c->p.algorithm == 1) {
    int ov = 0;
    FCM_TRY(advance_to_midstep_dev(c, c->d_V, &ov));
    double* acc = c->d_H + c->maxit_alloc + 1;
    if (noise) FCM_TRY(divU_enqueue(c, acc));
    k_gdc_nu<<<1, 32, 0, c->stream>>>(c->d_step, acc, noise ? 1 : 0, c->p.dt, c->d_rs + 3);
    FCM_LAUNCH_CHECK();
    d_nu = c->d_rs + 3;
    FCM_TRY(launch_fill_blob_pos(*c, c->d_xm, c->d_qm, c->d_Y, c->stream));
    FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
    FCM_TRY(random_velocities_dev(c, c->d_V));
    if (c->shear) FCM_TRY(shear_velocities_dev(c));  // main.cpp:270-272
  }
  FCM_TRY(calculate_forces_dev(c));
  FCM_TRY(assemble_rhs_dev(c));
  const long long n = c->nsys;
  *k_sweep = 0;
  if (c->p.precision == 0) {
    FCM_TRY(enqueue_gmres_loop(c, 0, c->d_rhs, c->d_soln, c->p.gmres_tol, nullptr, c->cap_body[0], k_iter));
    l_loops += *k_iter;
    k_gm_record<<<1, 32, 0, c->stream>>>(c->d_step, c->gm);
    FCM_LAUNCH_CHECK();
  } else {
    // r = b; x = 0; repeat: dx = GMRES32(r); x += dx; r = b - A64 x (solve_dev).
    double* x = c->d_soln;
    FCM_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, c->stream));
    FCM_CUDA(cudaMemcpyAsync(c->d_res, c->d_rhs, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream));
    FCM_TRY(blas_norm_sq_partial(*c, c->d_rhs, n, c->d_rs + 0, c->stream));
    cudaGraphConditionalHandle h;
    FCM_TRY(new_handle(c->stream, &h));
    k_ref_enter<<<1, 32, 0, c->stream>>>(h, c->d_step, c->d_rs);
    FCM_LAUNCH_CHECK();
    cudaGraph_t body = nullptr;
    FCM_TRY(add_while_node(c->stream, h, &body));
    const long long l0 = launch_count();
    FCM_TRY(capture_body(c, body, c->cap_body[0], [&] {
      k_ref_tol<<<1, 32, 0, c->stream>>>(c->d_step, c->p.gmres_tol, c->d_rs);
      FCM_LAUNCH_CHECK();
      FCM_TRY(enqueue_gmres_loop(c, 1, c->d_res, c->d_dx, 0.0, c->d_rs + 2, c->cap_body[1], k_iter));
      FCM_TRY(blas_axpby(x, c->d_dx, 1.0, 1.0, n, c->stream));
      FCM_TRY(saddle_matvec(c, 0, x, c->d_res));
      FCM_TRY(blas_axpby(c->d_res, c->d_rhs, 1.0, -1.0, n, c->stream));
      FCM_TRY(blas_norm_sq_partial(*c, c->d_res, n, c->d_rs + 1, c->stream));
      k_ref_next<<<1, 32, 0, c->stream>>>(h, c->d_step, c->gm, c->d_rs, c->p.gmres_tol, kMaxSweeps);
      FCM_LAUNCH_CHECK();
      return (int)FCM_OK;
    }));
    *k_sweep = launch_count() - l0 - *k_iter;
    l_loops += launch_count() - l0;
  }
  int ov = 0;
  FCM_TRY(end_of_step_update_dev(c, c->d_soln + 3 * (size_t)c->Nb, 1.0, &ov, d_nu));
  FCM_CUDA(cudaMemcpyAsync(c->h_step, c->d_step, sizeof(StepRecord), cudaMemcpyDeviceToHost, c->stream));
  *k_top = launch_count() - l_start - l_loops;
  return FCM_OK;
}

// Capture the resident step into c->step_graph (state 1), or mark the context
// for host-driven steps (state -1) when the step cannot be a graph.
int build_step_graph(Ctx* c) {
  if (c->p.skip_on_overlap || c->p.slip_channel) {  // steps that may be rejected stay host-driven
    c->step_graph_state = -1;
    return FCM_OK;
  }
  if (!c->d_step) {
    if (cudaMalloc(&c->d_step, sizeof(StepRecord)) != cudaSuccess ||
        cudaMallocHost(&c->h_step, sizeof(StepRecord)) != cudaSuccess ||
        cudaMalloc(&c->d_stepargs, 2 * sizeof(uint64_t)) != cudaSuccess ||
        cudaMallocHost(&c->h_stepargs, 2 * sizeof(uint64_t)) != cudaSuccess ||
        cudaMalloc(&c->d_rs, 8 * sizeof(double)) != cudaSuccess ||
        (!c->cap_body[0] && cudaStreamCreateWithFlags(&c->cap_body[0], cudaStreamNonBlocking) != cudaSuccess) ||
        (!c->cap_body[1] && cudaStreamCreateWithFlags(&c->cap_body[1], cudaStreamNonBlocking) != cudaSuccess)) {
      cudaGetLastError();
      set_error("step graph: buffer allocation failed");
      c->step_graph_state = -1;
      return FCM_ERR_NOMEM;
    }
  }
  const long long l0 = launch_count();
  int st = FCM_OK;
  cudaGraph_t g = nullptr;
  long long kt = 0, ks = 0, ki = 0;
  cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    {
      StreamSwap sw(c, c->cap_stream);
      st = enqueue_resident_step(c, &kt, &ks, &ki);
    }
    const cudaError_t e2 = cudaStreamEndCapture(c->cap_stream, &g);
    if (st == FCM_OK && e2 != cudaSuccess) {
      set_error(std::string("step graph capture: ") + cudaGetErrorString(e2));
      st = FCM_ERR_CUDA;
    }
  } else {
    set_error(std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
    st = FCM_ERR_CUDA;
  }
  count_launches(-(launch_count() - l0));  // counted per executed step instead
  if (st == FCM_OK) {
    e = cudaGraphInstantiate(&c->step_graph, g, 0);
    if (e != cudaSuccess) {
      set_error(std::string("step graph instantiate: ") + cudaGetErrorString(e));
      c->step_graph = nullptr;
      st = FCM_ERR_CUDA;
    }
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  if (st != FCM_OK) {
    c->step_graph_state = -1;
    return st;
  }
  c->step_kernels_top = kt;
  c->step_kernels_sweep = ks;
  c->step_kernels_iter = ki;
  c->step_graph_state = 1;
  return FCM_OK;
}

int reference_matrices_dev(Ctx* c) {
  const int nb = c->nb, n3 = 3 * nb;
  // Body 0 alone at the box centre (in a slip channel at the channel's centre,
  // y = L_y/4) with q = 1 (collection_of_rigid_bodies.cpp:132-151).
  std::vector<double> ref(3 * nb), Y(3 * nb);
  FCM_CUDA(cudaMemcpyAsync(ref.data(), c->d_ref, sizeof(double) * 3 * nb, cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  const double centre[3] = {0.5 * c->g.Lx, (c->p.slip_channel ? 0.25 : 0.5) * c->g.Ly, 0.5 * c->g.Lz};
  const double L[3] = {c->g.Lx, c->g.Ly, c->g.Lz};
  for (int m = 0; m < nb; ++m)
    for (int d = 0; d < 3; ++d) {
      const double p = centre[d] + ref[3 * m + d];
      Y[3 * m + d] = p - L[d] * std::floor(p / L[d]);
    }
  double *dY = nullptr, *dF = nullptr, *dV = nullptr;
  FCM_TRY(dev_alloc(&dY, 3 * (size_t)nb));
  FCM_TRY(dev_alloc(&dF, 3 * (size_t)nb));
  FCM_TRY(dev_alloc(&dV, 3 * (size_t)nb));
  int st = FCM_OK;
  std::vector<double> Mb((size_t)n3 * n3);
  do {
    if ((st = copy_in(c, dY, Y.data(), sizeof(double) * 3 * nb)) != FCM_OK) break;
    if ((st = launch_set_up_gaussians<double>(*c, c->g64.ref_blobs, dY, c->stream)) != FCM_OK) break;
    std::vector<double> e(n3, 0.0);
    for (int n = 0; n < n3 && st == FCM_OK; ++n) {
      std::fill(e.begin(), e.end(), 0.0);
      e[n] = 1.0;
      if ((st = copy_in(c, dF, e.data(), sizeof(double) * n3)) != FCM_OK) break;
      if ((st = spread_t<double>(c, c->g64.ref_blobs, dF)) != FCM_OK) break;
      if ((st = stokes_t<double>(c)) != FCM_OK) break;
      if ((st = interp_t<double>(c, c->g64.ref_blobs, c->g64.r, dV)) != FCM_OK) break;
      if (cudaMemcpyAsync(&Mb[(size_t)n * n3], dV, sizeof(double) * n3, cudaMemcpyDeviceToHost, c->stream) !=
          cudaSuccess) {
        st = FCM_ERR_CUDA;
        break;
      }
      if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
        st = FCM_ERR_CUDA;
        break;
      }
    }
  } while (0);
  cudaFree(dY);
  cudaFree(dF);
  cudaFree(dV);
  if (st != FCM_OK) return st;
  // ref_Minv = inv_sympd(M_body); ref_N = inv(K^T ref_Minv K) (fcm_fluid_solver.cpp:866-877)
  std::vector<double> Minv, N;
  if (!dense_inv_sympd(Mb, n3, Minv)) {
    set_error("single-body mobility is not positive definite");
    return FCM_ERR_NONFINITE;
  }
  const std::vector<double> K = reference_K(ref, nb);
  std::vector<double> KtMK(36, 0.0), t(n3);
  for (int j = 0; j < 6; ++j) {
    for (int i = 0; i < n3; ++i) {
      double s = 0.0;
      for (int k = 0; k < n3; ++k) s += Minv[(size_t)k * n3 + i] * K[(size_t)j * n3 + k];
      t[i] = s;
    }
    for (int i = 0; i < 6; ++i) {
      double s = 0.0;
      for (int r = 0; r < n3; ++r) s += K[(size_t)i * n3 + r] * t[r];
      KtMK[(size_t)j * 6 + i] = s;
    }
  }
  if (!sym_inv_or_pinv(KtMK, 6, N, nullptr)) {
    set_error("K^T Minv K could not be inverted");
    return FCM_ERR_NONFINITE;
  }
  c->h_Minv = Minv;
  c->h_N = N;
  FCM_CUDA(cudaMemcpyAsync(c->d_Minv, c->h_Minv.data(), sizeof(double) * n3 * n3, cudaMemcpyHostToDevice, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->d_N, c->h_N.data(), sizeof(double) * 36, cudaMemcpyHostToDevice, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  c->have_ref = true;
  c->gauss_ready = false;  // the main tables are untouched, but V was not produced for them
  return FCM_OK;
}

// Copy between the reference's padded [x][y][pad] layout and the unpadded grid.
int padded_to_grid(Ctx* c, double* dst, const double* src_padded) {
  FCM_CUDA(cudaMemcpy2DAsync(dst, sizeof(double) * c->g.nz, src_padded, sizeof(double) * 2 * c->g.nzh,
                             sizeof(double) * c->g.nz, (size_t)c->g.nx * c->g.ny, cudaMemcpyDefault, c->stream));
  return FCM_OK;
}

template <typename T>
int grid_to_padded(Ctx* c, double* dst_padded, const T* src) {
  const size_t G = (size_t)c->g.G;
  const int pad = 2 * c->g.nzh;
  std::vector<T> h(G);
  FCM_CUDA(cudaMemcpyAsync(h.data(), src, sizeof(T) * G, cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  std::vector<double> out((size_t)c->g.nx * c->g.ny * pad, 0.0);
  for (size_t l = 0; l < (size_t)c->g.nx * c->g.ny; ++l)
    for (int k = 0; k < c->g.nz; ++k) out[l * pad + k] = (double)h[l * c->g.nz + k];
  FCM_CUDA(cudaMemcpyAsync(dst_padded, out.data(), sizeof(double) * out.size(), cudaMemcpyDefault, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  return FCM_OK;
}

int check_params(const fcm_params* p) {
  if (!p) return FCM_ERR_INVALID;
  auto bad = [](const char* m) {
    set_error(m);
    return FCM_ERR_INVALID;
  };
  if (p->nx < 2 || p->ny < 2 || p->nz < 2) return bad("grid dimensions must be >= 2");
  if (p->ngauss < 1 || p->ngauss > p->nx || p->ngauss > p->ny || p->ngauss > p->nz)
    return bad("ngauss must be in [1, min(nx,ny,nz)]");
  if (!(p->dx > 0) || !(p->blob_radius > 0) || !(p->viscosity > 0) || !(p->dt > 0) || !(p->kT >= 0))
    return bad("dx, blob_radius, viscosity, dt must be > 0 and kT >= 0");
  if (p->num_bodies < 1 || p->blobs_per_body < 1) return bad("num_bodies and blobs_per_body must be >= 1");
  if (p->ncells < 3) return bad("ncells must be >= 3 (the 13-cell half shell degenerates below 3)");
  if (p->potential < 0 || p->potential > 3) return bad("potential must be 0..3");
  if (p->gmres_max_iter < 1) return bad("gmres_max_iter must be >= 1");
  if (p->algorithm != 1 && p->algorithm != 2) return bad("algorithm must be 1 (GDC) or 2 (EM)");
  if (p->precision != 0 && p->precision != 1) return bad("precision must be 0 or 1");
  if (p->slip_channel != 0 && p->slip_channel != 1) return bad("slip_channel must be 0 or 1");
  if (p->slip_channel && p->ny % 2) return bad("slip_channel needs an even ny (walls at rows 0 and ny/2)");
  const long long G = (long long)p->nx * p->ny * p->nz;
  if (3 * G > 2000000000LL) return bad("grid too large for 32-bit cuFFT batch strides");
  return FCM_OK;
}

void destroy_ctx(Ctx* c) {
  if (!c) return;
  double* ptrs[] = {c->d_ref, c->d_x, c->d_q, c->d_xm, c->d_qm, c->d_xs, c->d_qs, c->d_Y, c->d_V, c->d_F,
                    c->d_fe, c->d_U0, c->d_tmp3, c->d_tmp6, c->d_sys_a, c->d_sys_b, c->d_rhs, c->d_soln, c->d_res, c->d_dx, c->d_Minv, c->d_N,
                    c->d_KTKinv, c->d_Qm, c->d_H, c->d_y, c->d_partials, c->d_stress};
  for (double* p : ptrs) cudaFree(p);
  cudaFree(c->d_counter);
  for (int i = 0; i < 2; ++i)
    if (c->iter_graph[i]) cudaGraphExecDestroy(c->iter_graph[i]);
  cudaFree(c->gm);
  double* gptrs[] = {c->d_Hd, c->d_beta, c->d_CS, c->d_SN, c->d_hA, c->d_hB, c->d_hnorm, c->d_mdpart};
  for (double* p : gptrs) cudaFree(p);
  cudaFree(c->d_mdcount);
  if (c->h_gm) cudaFreeHost(c->h_gm);
  if (c->cap_stream) cudaStreamDestroy(c->cap_stream);
  cudaFree(c->d_dip);
  cudaFree(c->d_xtw64);
  cudaFree(c->d_xtw32);
  cudaFree(c->d_ytw32);
  cudaFree(c->d_ztw32);
  cudaFree(c->d_ushear);
  cudaFree(c->d_vshear);
  cudaFree(c->d_mcmc);
  cudaFree(c->d_usum);
  if (c->mcmc_graph) cudaGraphExecDestroy(c->mcmc_graph);
  if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
  if (!c->in_batch) {
    cudaFree(c->d_step);
    cudaFree(c->d_stepargs);
  }
  cudaFree(c->d_rs);
  if (c->h_step) cudaFreeHost(c->h_step);
  if (c->h_stepargs) cudaFreeHost(c->h_stepargs);
  for (int i = 0; i < 2; ++i)
    if (c->cap_body[i]) cudaStreamDestroy(c->cap_body[i]);
  cudaFree(c->d_cell);
  cudaFree(c->d_cell_start);
  cudaFree(c->d_cell_count);
  cudaFree(c->d_cell_sorted);
  cudaFree(c->d_cell_cursor);
  cudaFree(c->d_flag);
  cudaFree(c->d_pair_count);
  cudaFree(c->d_stress_c);
  if (c->plan_r2c6) cufftDestroy(c->plan_r2c6);
  if (c->h_pinned) cudaFreeHost(c->h_pinned);
  free_grid(c->g64);
  free_grid(c->g32);
  delete c;
}

int create_ctx(const fcm_params* p, const double* ref, Ctx** out) {
  FCM_TRY(check_params(p));
  if (!ref) {
    set_error("blob_ref_pos is null");
    return FCM_ERR_INVALID;
  }
  Ctx* c = new Ctx();
  c->p = *p;
  cudaGetDevice(&c->device);
  c->M = p->num_bodies;
  c->nb = p->blobs_per_body;
  c->Nb = c->M * c->nb;
  c->nsys = 3 * c->Nb + 6 * c->M;
  c->g.nx = p->nx;
  c->g.ny = p->ny;
  c->g.nz = p->nz;
  c->g.nzh = p->nz / 2 + 1;
  c->g.G = (long long)p->nx * p->ny * p->nz;
  c->g.Gc = (long long)p->nx * p->ny * c->g.nzh;
  c->g.dx = p->dx;
  c->g.Lx = p->dx * p->nx;  // config.hpp:89-91
  c->g.Ly = p->dx * p->ny;
  c->g.Lz = p->dx * p->nz;
  int st = FCM_OK;
  auto fail = [&](int s) {
    destroy_ctx(c);
    return s;
  };
  const int M = c->M, Nb = c->Nb, nb = c->nb;
  const long long n = c->nsys;
  if ((st = dev_alloc(&c->d_ref, 3 * (size_t)nb)) || (st = dev_alloc(&c->d_x, 3 * (size_t)M)) ||
      (st = dev_alloc(&c->d_q, 4 * (size_t)M)) || (st = dev_alloc(&c->d_xm, 3 * (size_t)M)) ||
      (st = dev_alloc(&c->d_qm, 4 * (size_t)M)) || (st = dev_alloc(&c->d_xs, 3 * (size_t)M)) ||
      (st = dev_alloc(&c->d_qs, 4 * (size_t)M)) || (st = dev_alloc(&c->d_Y, 3 * (size_t)Nb)) ||
      (st = dev_alloc(&c->d_V, 3 * (size_t)Nb)) || (st = dev_alloc(&c->d_F, 3 * (size_t)Nb)) ||
      (st = dev_alloc(&c->d_fe, 6 * (size_t)M)) || (st = dev_alloc(&c->d_U0, 6 * (size_t)M)) ||
      (st = dev_alloc(&c->d_tmp3, std::max<size_t>(3 * (size_t)Nb, (size_t)M))) ||
      (st = dev_alloc(&c->d_tmp6, 6 * (size_t)M)) || (st = dev_alloc(&c->d_sys_a, n)) ||
      (st = dev_alloc(&c->d_sys_b, n)) || (st = dev_alloc(&c->d_rhs, n)) ||
      (st = dev_alloc(&c->d_soln, n)) || (st = dev_alloc(&c->d_res, n)) || (st = dev_alloc(&c->d_dx, n)) ||
      (st = dev_alloc(&c->d_Minv, 9 * (size_t)nb * nb)) || (st = dev_alloc(&c->d_N, 36)) ||
      (st = dev_alloc(&c->d_KTKinv, 36)))
    return fail(st);
  c->maxit_alloc = (int)std::min<long long>(n, p->gmres_max_iter);
  if ((st = dev_alloc(&c->d_Qm, n * (size_t)(c->maxit_alloc + 1))) ||
      (st = dev_alloc(&c->d_H, (size_t)c->maxit_alloc + 4)) || (st = dev_alloc(&c->d_y, (size_t)c->maxit_alloc + 1)))
    return fail(st);
  c->red_blocks = (int)std::max<long long>(1, std::min<long long>(296, (n + 1023) / 1024));
  c->md_blocks = (int)std::max<long long>(1, std::min<long long>(148, (n + 2047) / 2048));
  {
    const size_t hn = (size_t)c->maxit_alloc + 1;
    if ((st = dev_alloc(&c->gm, 1)) || (st = dev_alloc(&c->d_Hd, hn * hn)) || (st = dev_alloc(&c->d_beta, hn)) ||
        (st = dev_alloc(&c->d_CS, hn)) || (st = dev_alloc(&c->d_SN, hn)) || (st = dev_alloc(&c->d_hA, hn)) ||
        (st = dev_alloc(&c->d_hB, hn)) || (st = dev_alloc(&c->d_hnorm, 1)) ||
        (st = dev_alloc(&c->d_mdpart, hn * c->md_blocks)) || (st = dev_alloc(&c->d_mdcount, hn)))
      return fail(st);
    if (cudaMemset(c->d_mdcount, 0, sizeof(unsigned int) * hn) != cudaSuccess ||
        cudaMemset(c->d_Hd, 0, sizeof(double) * hn * hn) != cudaSuccess ||
        cudaMallocHost(&c->h_gm, sizeof(GmState)) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->cap_stream, cudaStreamNonBlocking) != cudaSuccess) {
      set_error("GMRES state allocation failed");
      return fail(FCM_ERR_NOMEM);
    }
  }
  if ((st = dev_alloc(&c->d_partials, (size_t)c->red_blocks)) ||
      (st = dev_alloc(&c->d_counter, 1)))
    return fail(st);
  if (cudaMallocHost(&c->h_pinned, sizeof(double) * std::max(256, c->maxit_alloc + 8)) != cudaSuccess)
    return fail(FCM_ERR_NOMEM);
  for (int m = 0; m < nb; ++m) {
    const double* r = ref + 3 * m;
    c->body_radius = std::max(c->body_radius, std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]));
  }
  c->ncell_total = p->ncells * p->ncells * p->ncells;
  if ((st = dev_alloc(&c->d_cell, (size_t)Nb)) || (st = dev_alloc(&c->d_cell_start, (size_t)c->ncell_total + 1)) ||
      (st = dev_alloc(&c->d_cell_count, (size_t)c->ncell_total)) ||
      (st = dev_alloc(&c->d_cell_sorted, (size_t)Nb)) || (st = dev_alloc(&c->d_cell_cursor, (size_t)c->ncell_total)) ||
      (st = dev_alloc(&c->d_flag, 1)) || (st = dev_alloc(&c->d_pair_count, 1)))
    return fail(st);
  if (cudaMemsetAsync(c->d_counter, 0, sizeof(unsigned int), c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_fe, 0, sizeof(double) * 6 * M, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_V, 0, sizeof(double) * 3 * Nb, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_F, 0, sizeof(double) * 3 * Nb, c->stream) != cudaSuccess ||
      cudaMemsetAsync(c->d_U0, 0, sizeof(double) * 6 * M, c->stream) != cudaSuccess) {
    set_error("cudaMemsetAsync failed");
    return fail(FCM_ERR_CUDA);
  }
  // shape, identity bodies, reference matrices (identity until produced)
  std::vector<double> href(ref, ref + 3 * nb);
  if (cudaMemcpy(c->d_ref, href.data(), sizeof(double) * 3 * nb, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(FCM_ERR_CUDA);
  std::vector<double> hx(3 * (size_t)M, 0.0), hq(4 * (size_t)M, 0.0);
  for (int i = 0; i < M; ++i) hq[4 * i] = 1.0;
  for (double* d : {c->d_x, c->d_xm, c->d_xs})
    if (cudaMemcpy(d, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(FCM_ERR_CUDA);
  for (double* d : {c->d_q, c->d_qm, c->d_qs})
    if (cudaMemcpy(d, hq.data(), sizeof(double) * hq.size(), cudaMemcpyHostToDevice) != cudaSuccess)
      return fail(FCM_ERR_CUDA);
  const int n3 = 3 * nb;
  c->h_Minv.assign((size_t)n3 * n3, 0.0);
  for (int i = 0; i < n3; ++i) c->h_Minv[(size_t)i * n3 + i] = 1.0;
  c->h_N.assign(36, 0.0);
  for (int i = 0; i < 6; ++i) c->h_N[i * 6 + i] = 1.0;
  // ref_KTKinv = inv(K^T K) (collection_of_rigid_bodies.cpp:117-130)
  {
    const std::vector<double> K = reference_K(href, nb);
    if (!sym_inv_or_pinv(shape_KTK(K, nb), 6, c->h_KTKinv, nullptr)) {
      set_error("K^T K of the body shape could not be inverted");
      return fail(FCM_ERR_INVALID);
    }
  }
  if (cudaMemcpy(c->d_Minv, c->h_Minv.data(), sizeof(double) * n3 * n3, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_N, c->h_N.data(), sizeof(double) * 36, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(c->d_KTKinv, c->h_KTKinv.data(), sizeof(double) * 36, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(FCM_ERR_CUDA);
  if ((st = setup_xfft(c)) != FCM_OK) return fail(st);
  if ((st = ensure_grid<double>(c)) != FCM_OK) return fail(st);
  if (p->precision == 1 && (st = ensure_grid<float>(c)) != FCM_OK) return fail(st);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) return fail(FCM_ERR_CUDA);
  *out = c;
  return FCM_OK;
}

template <class F>
int guard(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return FCM_ERR_NOMEM;
  } catch (const std::exception& e) {
    set_error(e.what());
    return FCM_ERR_INVALID;
  } catch (...) {
    set_error("unknown exception");
    return FCM_ERR_INVALID;
  }
}

#define CTX_CHECK(ctx)                   \
  if (!(ctx)) {                          \
    ::fcm::set_error("null context");    \
    return FCM_ERR_INVALID;              \
  }

// main.cpp:222-451, one step driven from the host.
int step_host(Ctx* c, uint64_t seed, uint64_t step_index, fcm_step_info* info) {
  NvtxRange range("fcm step");
  {
    fcm_step_info inf;
    std::memset(&inf, 0, sizeof(inf));
    const bool noise = c->p.noise != 0;
    // main.cpp:230-233
    FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
    if (noise) FCM_TRY(noise_dev(c, seed, step_index));
    else c->urand_ready = false;
    FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
    FCM_TRY(random_velocities_dev(c, c->d_V));
    double nu = 1.0;
    if (c->p.algorithm == 1) {  // main.cpp:235-268
      int ov = 0;
      FCM_TRY(advance_to_midstep_dev(c, c->d_V, &ov));
      if (ov) {
        inf.overlap = 1;
        if (info) *info = inf;
        return (int)FCM_ERR_OVERLAP;
      }
      double divU = 0.0;
      if (noise) FCM_TRY(divU_dev(c, &divU));
      inf.divU = divU;
      nu = 1.0 + 0.5 * c->p.dt * divU;
      FCM_TRY(launch_fill_blob_pos(*c, c->d_xm, c->d_qm, c->d_Y, c->stream));
      FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
      FCM_TRY(random_velocities_dev(c, c->d_V));
      if (c->shear) FCM_TRY(shear_velocities_dev(c));  // main.cpp:270-272
    }
    FCM_TRY(calculate_forces_dev(c));  // main.cpp:282
    FCM_TRY(assemble_rhs_dev(c));      // main.cpp:308
    int it = 0, sw = 0;
    double rel = 0.0;
    const int st = solve_dev(c, c->d_rhs, c->d_soln, &it, &rel, &sw);  // main.cpp:310
    inf.gmres_iters = it;
    inf.refinement_sweeps = sw;
    inf.gmres_rel_residual = rel;
    inf.status = st;
    if (st != FCM_OK && st != FCM_ERR_NOT_CONVERGED) {
      if (info) *info = inf;
      return st;
    }
    int ov = 0;
    FCM_TRY(end_of_step_update_dev(c, c->d_soln + 3 * (size_t)c->Nb, nu, &ov));  // main.cpp:312
    if (ov) {  // main.cpp:316-328
      FCM_CUDA(cudaMemcpyAsync(c->d_x, c->d_xs, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
      FCM_CUDA(cudaMemcpyAsync(c->d_q, c->d_qs, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
      inf.overlap = 1;
      if (info) *info = inf;
      return (int)FCM_ERR_OVERLAP;
    }
    if (info) *info = inf;
    return (int)FCM_OK;
  }
}

// Issue one step on c->stream: a launch of the step graph when the context has
// one; otherwise (first step, or skip_on_overlap) a host-driven step whose
// result step_wait returns.  The first host-driven step allocates every buffer,
// after which the step graph is captured.
int step_issue(Ctx* c, uint64_t seed, uint64_t step_index) {
  if (c->step_pending) {
    set_error("a step is already in flight on this context: call fcm_step_wait first");
    return FCM_ERR_STATE;
  }
  if (c->graph_stale && !c->in_batch) {  // recapture after a change of the step's work
    if (c->step_graph) cudaGraphExecDestroy(c->step_graph);
    c->step_graph = nullptr;
    if (c->step_graph_state == 1) c->step_graph_state = 0;
    c->graph_stale = false;
  }
  if (c->step_graph_state == 1) {
    c->h_stepargs[0] = seed;
    c->h_stepargs[1] = step_index;
    FCM_CUDA(cudaMemcpyAsync(c->d_stepargs, c->h_stepargs, 2 * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    FCM_CUDA(cudaGraphLaunch(c->step_graph, c->stream));
    c->step_pending = true;
    c->step_pending_graph = true;
    return FCM_OK;
  }
  fcm_step_info inf;
  std::memset(&inf, 0, sizeof(inf));
  const int st = step_host(c, seed, step_index, &inf);
  if (st != FCM_OK && st != FCM_ERR_OVERLAP) return st;
  c->step_pending = true;
  c->step_pending_graph = false;
  c->step_pending_status = st;
  c->step_pending_info = inf;
  if (c->step_graph_state == 0 && st == FCM_OK) {
    const std::string keep = g_err;
    if (build_step_graph(c) != FCM_OK) set_error(keep);  // host-driven steps from now on
  }
  return FCM_OK;
}

int step_wait(Ctx* c, fcm_step_info* info) {
  if (!c->step_pending) {
    set_error("no step in flight on this context");
    return FCM_ERR_STATE;
  }
  c->step_pending = false;
  if (!c->step_pending_graph) {
    if (info) *info = c->step_pending_info;
    return c->step_pending_status;
  }
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  const StepRecord r = *c->h_step;
  count_launches(c->step_kernels_top + (long long)r.sweeps * c->step_kernels_sweep +
                 (long long)r.iters * c->step_kernels_iter);
  c->gauss_ready = true;
  c->urand_ready = c->p.noise != 0;
  c->urand_prec = noise_precision(c);
  fcm_step_info inf;
  std::memset(&inf, 0, sizeof(inf));
  inf.gmres_iters = r.iters;
  inf.refinement_sweeps = r.sweeps;
  inf.gmres_rel_residual = r.rel;
  inf.divU = r.divU;
  inf.status = r.status;
  if (info) *info = inf;
  if (r.status != FCM_OK && r.status != FCM_ERR_NOT_CONVERGED) {
    // the host-driven step stops before the body update: put the bodies back
    FCM_CUDA(cudaMemcpyAsync(c->d_x, c->d_xs, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
    FCM_CUDA(cudaMemcpyAsync(c->d_q, c->d_qs, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
    FCM_CUDA(cudaStreamSynchronize(c->stream));
    set_error(r.status == FCM_ERR_NONFINITE ? "GMRES residual became non-finite" : "step failed");
    return r.status;
  }
  return FCM_OK;
}

// ------------------------------------------------------------------ Metropolis
__global__ void k_mcmc_enter(cudaGraphConditionalHandle h, const McmcDev* __restrict__ st) {
  if (threadIdx.x == 0)
    cudaGraphSetConditional(h, (st->n < st->n_target && st->attempt < st->attempt_cap) ? 1u : 0u);
}

__global__ void k_mcmc_set_energy(McmcDev* st, const double* __restrict__ usum) {
  if (threadIdx.x == 0) st->U_old = 0.5 * *usum;
}

// main.cpp:162-200: Metropolis test, running acceptance ratio (20 steps), scale.
__global__ void k_mcmc_decide(cudaGraphConditionalHandle h, McmcDev* st, const double* __restrict__ usum,
                              const int* __restrict__ ovflag, unsigned int i_acc) {
  if (threadIdx.x != 0) return;
  const double rs = 20.0;
  if (st->skip_on_overlap && *ovflag) {
    st->restore = 1;
  } else {
    const double U = 0.5 * *usum;
    const double u = mcmc_uniform(st->seed, (uint64_t)st->attempt, i_acc);
    if (u < exp((st->U_old - U) / st->kT)) {
      st->U_old = U;
      st->acc = ((rs - 1.0) * st->acc + 1.0) / rs;
      st->restore = 0;
    } else {
      st->restore = 1;
      st->acc *= (rs - 1.0) / rs;
    }
    st->n += 1;
    st->scale *= st->acc > 0.5 ? 1.02 : 0.98;
  }
  st->attempt += 1;
  cudaGraphSetConditional(h, (st->n < st->n_target && st->attempt < st->attempt_cap) ? 1u : 0u);
}

// Energy of the current bodies into *d_usum (twice the potential).
int potential_sum_dev(Ctx* c) {
  FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
  FCM_TRY(cells_build(*c, c->stream));
  FCM_TRY(cells_potential_terms(*c, c->d_tmp3, c->stream));
  FCM_TRY(blas_dot(*c, c->d_tmp3, nullptr, c->Nb, c->d_usum, c->stream));
  return FCM_OK;
}

int mcmc_alloc(Ctx* c) {
  if (c->d_mcmc) return FCM_OK;
  FCM_TRY(dev_alloc(&c->d_mcmc, 1));
  FCM_TRY(dev_alloc(&c->d_usum, 1));
  return FCM_OK;
}

// The Metropolis loop as one graph: while (n < n_target) { propose, positions,
// cells, [overlap], energy, decide, undo if rejected }.
int build_mcmc_graph(Ctx* c) {
  if (c->mcmc_graph) return FCM_OK;
  if (!c->cap_body[0] && cudaStreamCreateWithFlags(&c->cap_body[0], cudaStreamNonBlocking) != cudaSuccess) {
    cudaGetLastError();
    set_error("MCMC graph: stream creation failed");
    return FCM_ERR_CUDA;
  }
  const long long l0 = launch_count();
  int st = FCM_OK;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(c->cap_stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    {
      StreamSwap sw(c, c->cap_stream);
      do {
        cudaGraphConditionalHandle h;
        if ((st = new_handle(c->stream, &h)) != FCM_OK) break;
        k_mcmc_enter<<<1, 32, 0, c->stream>>>(h, c->d_mcmc);
        count_launch();
        cudaGraph_t body = nullptr;
        if ((st = add_while_node(c->stream, h, &body)) != FCM_OK) break;
        const long long lb = launch_count();
        st = capture_body(c, body, c->cap_body[0], [&] {
          FCM_TRY(launch_mcmc_propose(*c, c->d_mcmc, c->stream));
          FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
          FCM_TRY(cells_build(*c, c->stream));
          if (c->p.skip_on_overlap) FCM_TRY(cells_overlap(*c, c->d_flag, c->stream));
          else if (c->p.slip_channel) FCM_CUDA(cudaMemsetAsync(c->d_flag, 0, sizeof(int), c->stream));
          FCM_TRY(cells_wall_overlap(*c, c->d_flag, c->stream));  // slip channel (main.cpp:160)
          FCM_TRY(cells_potential_terms(*c, c->d_tmp3, c->stream));
          FCM_TRY(blas_dot(*c, c->d_tmp3, nullptr, c->Nb, c->d_usum, c->stream));
          k_mcmc_decide<<<1, 32, 0, c->stream>>>(h, c->d_mcmc, c->d_usum, c->d_flag, (unsigned int)(6 * c->M));
          FCM_LAUNCH_CHECK();
          FCM_TRY(launch_mcmc_restore(*c, c->d_mcmc, c->stream));
          return (int)FCM_OK;
        });
        c->mcmc_kernels = launch_count() - lb;
      } while (0);
    }
    const cudaError_t e2 = cudaStreamEndCapture(c->cap_stream, &g);
    if (st == FCM_OK && e2 != cudaSuccess) {
      set_error(std::string("MCMC graph capture: ") + cudaGetErrorString(e2));
      st = FCM_ERR_CUDA;
    }
  } else {
    set_error(std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
    st = FCM_ERR_CUDA;
  }
  count_launches(-(launch_count() - l0));
  if (st == FCM_OK) {
    e = cudaGraphInstantiate(&c->mcmc_graph, g, 0);
    if (e != cudaSuccess) {
      set_error(std::string("MCMC graph instantiate: ") + cudaGetErrorString(e));
      c->mcmc_graph = nullptr;
      st = FCM_ERR_CUDA;
    }
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  return st;
}

int mcmc_run_dev(Ctx* c, uint64_t seed, long long n_steps, fcm_mcmc_state* state) {
  FCM_TRY(mcmc_alloc(c));
  FCM_TRY(build_mcmc_graph(c));
  McmcDev h;
  std::memset(&h, 0, sizeof(h));
  h.seed = seed;
  h.n = state->steps;
  h.n_target = state->steps + n_steps;
  h.attempt = state->attempts;
  h.attempt_cap = state->attempts + 100 * n_steps + 1000;
  h.scale = state->scale;
  h.acc = state->acceptance_ratio;
  h.body_radius = c->body_radius > 0.0 ? c->body_radius : c->p.blob_radius;
  h.dt = c->p.dt;
  h.kT = c->p.kT;
  h.skip_on_overlap = c->p.skip_on_overlap || c->p.slip_channel;  // redraw on rejected proposals
  FCM_CUDA(cudaMemcpyAsync(c->d_mcmc, &h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
  FCM_TRY(potential_sum_dev(c));  // U_old of main.cpp:116
  k_mcmc_set_energy<<<1, 32, 0, c->stream>>>(c->d_mcmc, c->d_usum);
  FCM_LAUNCH_CHECK();
  if (n_steps > 0) FCM_CUDA(cudaGraphLaunch(c->mcmc_graph, c->stream));
  FCM_CUDA(cudaMemcpyAsync(&h, c->d_mcmc, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  count_launches((h.attempt - state->attempts) * c->mcmc_kernels + (n_steps > 0 ? 1 : 0));
  // leave positions and cells of the accepted configuration
  FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
  FCM_TRY(cells_build(*c, c->stream));
  state->scale = h.scale;
  state->acceptance_ratio = h.acc;
  state->potential = h.U_old;
  state->steps = h.n;
  state->attempts = h.attempt;
  if (h.n < h.n_target) {
    set_error("MCMC: too many overlapping proposals (attempt bound reached)");
    return FCM_ERR_OVERLAP;
  }
  return FCM_OK;
}

// ------------------------------------------------------------------ batches
// A batch steps many independent suspensions (its members) together.  The
// per-member work of a step (blob positions, noise, Gaussian tables, cells and
// forces, right-hand side, body update) runs as one graph branch per member;
// the saddle-point solves run in lockstep as batched kernels: every member's
// tiles in one spread / interpolation launch, every member's modes in one
// projection launch, one cuFFT plan per group of members with equal grids (their
// grids are contiguous), and the GMRES vector work of all members per launch.
// Members whose solve has finished are skipped inside the kernels.  The step is
// one CUDA graph whose GMRES iterations and refinement sweeps are conditional
// loops that run until every member is done.
struct BatchGroup {
  int nx = 0, ny = 0, nz = 0;
  std::vector<int> idx;                   // members
  void* r[2] = {nullptr, nullptr};        // [precision] 3G per member, contiguous
  void* c[2] = {nullptr, nullptr};        // 3Gc per member
  void* urand[2] = {nullptr, nullptr};
  cufftHandle r2c[2] = {0, 0}, c2r[2] = {0, 0};
  // fused x-transform path: (y, z) transforms of every member's planes, member ids
  cufftHandle r2c2d[2] = {0, 0}, c2r2d[2] = {0, 0};
  int* d_gidx = nullptr;
};

struct Batch {
  BatchGeom geom;
  std::vector<Ctx*> m;
  int precision = 0;
  BMember* d_mem = nullptr;
  int2* d_tile_map = nullptr;
  int2* d_kblock_map = nullptr;
  double* d_partials = nullptr;
  unsigned* d_counter = nullptr;
  double* d_mdpart = nullptr;
  unsigned* d_mdcount = nullptr;
  StepRecord* d_rec = nullptr;
  StepRecord* h_rec = nullptr;
  uint64_t* d_args = nullptr;
  uint64_t* h_args = nullptr;
  int* d_loop = nullptr;  // [0] inner-loop guard [1] inner iterations run [2] sweeps run
  int* h_loop = nullptr;
  std::vector<BatchGroup> groups;
  cudaStream_t stream = 0;
  cudaStream_t cap = 0, cap_body[2] = {0, 0};
  std::vector<cudaStream_t> branch;
  std::vector<cudaEvent_t> events;  // 2 forks + 2n joins
  cudaGraphExec_t graph = nullptr;
  int state = 0;  // 0 not built, 1 built, -1 host-driven
  long long k_top = 0, k_sweep = 0, k_iter = 0;
};

__global__ void k_b_step_begin(const BMember* __restrict__ mem, int n, int* __restrict__ loop) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    StepRecord* sd = mem[i].sd;
    sd->iters = 0;
    sd->sweeps = 0;
    sd->status = FCM_OK;
    sd->guard = 0;
    sd->rel = 0.0;
    sd->divU = 0.0;
    sd->normb = 0.0;
    sd->relr = 1.0;
    sd->ref_active = 0;
  }
  if (threadIdx.x == 0) loop[0] = loop[1] = loop[2] = 0;
}

// Lockstep GMRES loop condition: some member not done, at most `limit` rounds.
__global__ void k_b_loop_cond(cudaGraphConditionalHandle h, const BMember* __restrict__ mem, int n,
                              int* __restrict__ loop, int enter, int limit) {
  __shared__ int any;
  if (threadIdx.x == 0) {
    any = 0;
    if (enter) {
      loop[0] = 0;
    } else {
      loop[0] += 1;
      loop[1] += 1;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (!mem[i].gm->done) atomicOr(&any, 1);
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, (any && loop[0] < limit) ? 1u : 0u);
}

__global__ void k_b_gm_record(const BMember* __restrict__ mem, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const BMember& m = mem[i];
    m.sd->iters = m.gm->k;
    m.sd->sweeps = 1;
    m.sd->rel = m.gm->rel;
    m.sd->status = m.gm->status;
  }
}

// soln = 0, res = rhs
__global__ void k_b_refine_start(const BMember* __restrict__ mem) {
  const BMember& m = mem[blockIdx.y];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m.nsys) return;
  m.soln[i] = 0.0;
  m.res[i] = m.rhs[i];
}

__global__ void k_b_ref_enter(cudaGraphConditionalHandle h, const BMember* __restrict__ mem, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    StepRecord* sd = mem[i].sd;
    sd->normb = mem[i].rs[0];
    sd->relr = 1.0;
    sd->sweeps = 0;
    sd->iters = 0;
    sd->status = FCM_OK;
    sd->ref_active = 1;
  }
  if (threadIdx.x == 0) cudaGraphSetConditional(h, n > 0 ? 1u : 0u);
}

__global__ void k_b_ref_tol(const BMember* __restrict__ mem, int n, double tol) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const BMember& m = mem[i];
    if (m.sd->ref_active) m.rs[2] = fmin(0.5, fmax(1e-6, 0.3 * tol / m.sd->relr));
  }
}

// k_ref_next for every member still sweeping; the loop goes on while any does.
__global__ void k_b_ref_next(cudaGraphConditionalHandle h, const BMember* __restrict__ mem, int n, double tol,
                             int max_sweeps, int* __restrict__ loop) {
  __shared__ int any;
  if (threadIdx.x == 0) {
    any = 0;
    loop[2] += 1;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const BMember& m = mem[i];
    StepRecord* sd = m.sd;
    if (!sd->ref_active) continue;
    const GmState* gm = m.gm;
    sd->sweeps += 1;
    sd->iters += gm->k;
    int go = 0;
    if (gm->status == FCM_ERR_NONFINITE) {
      sd->status = FCM_ERR_NONFINITE;
      sd->rel = gm->rel;
    } else {
      const double relr = sd->normb > 0.0 ? m.rs[1] / sd->normb : 0.0;
      sd->relr = relr;
      sd->rel = relr;
      if (!isfinite(relr)) {
        sd->status = FCM_ERR_NONFINITE;
      } else if (relr < tol) {
        sd->status = FCM_OK;
      } else {
        sd->status = FCM_ERR_NOT_CONVERGED;
        go = sd->sweeps < max_sweeps ? 1 : 0;
      }
    }
    sd->ref_active = go;
    if (go) atomicOr(&any, 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

// Batched saddle-point product out = A in on the grids of precision T.
template <typename T>
int batch_saddle(Batch* B, int in, int out, int mask, cudaStream_t s) {
  constexpr int P = sizeof(T) == 8 ? 0 : 1;
  FCM_TRY(b_spread<T>(B->geom, in, mask, s));
  bool any3d = false;  // groups without the fused x-transform
  for (BatchGroup& g : B->groups) {
    const bool fused = g.r2c2d[P] != 0;
    any3d = any3d || !fused;
    const Ctx& c0 = *B->m[g.idx[0]];
    const int k = (int)g.idx.size();
    if (P == 1 && fused && c0.yz32 && 3LL * c0.g.nx * k <= 65535) {  // the library's (y, z) transforms
      FCM_TRY(launch_yz_forward(c0, (const float*)g.r[P], (cufftComplex*)g.c[P], k, s));
    } else {
      const cufftHandle h = fused ? g.r2c2d[P] : g.r2c[P];
      FCM_CUFFT(cufftSetStream(h, s));
      FCM_CUFFT(exec_r2c(h, (T*)g.r[P], (typename cplx_t<T>::type*)g.c[P]));
    }
    if (fused) FCM_TRY(b_xfft_project<T>(B->geom, c0, g.d_gidx, k, mask, s));
  }
  if (any3d) FCM_TRY(b_project<T>(B->geom, mask, s));  // members of the other groups
  for (BatchGroup& g : B->groups) {
    const Ctx& c0 = *B->m[g.idx[0]];
    const int k = (int)g.idx.size();
    if (P == 1 && g.c2r2d[P] && c0.yz32 && 3LL * c0.g.nx * k <= 65535) {
      FCM_TRY(launch_yz_inverse(c0, (cufftComplex*)g.c[P], (float*)g.r[P], k, s));
      continue;
    }
    const cufftHandle h = g.c2r2d[P] ? g.c2r2d[P] : g.c2r[P];
    FCM_CUFFT(cufftSetStream(h, s));
    FCM_CUFFT(exec_c2r(h, (typename cplx_t<T>::type*)g.c[P], (T*)g.r[P]));
  }
  FCM_TRY(b_interp<T>(B->geom, out, mask, s));
  FCM_TRY(b_multiply_K_KT(B->geom, in, out, mask, s));
  return FCM_OK;
}

// Lockstep GMRES of every member (on stream s, body captured on bs): init from
// vector `vec`, iterations until all are done, solution P^-1 sum y_i q_i in out.
int batch_gmres_loop(Batch* B, int prec, int vec, double tol, int use_rs, int mask, int out, cudaStream_t s,
                     cudaStream_t bs) {
  const BatchGeom& G = B->geom;
  FCM_TRY(b_gm_init(G, vec, tol, use_rs, mask, s));
  cudaGraphConditionalHandle h;
  FCM_TRY(new_handle(s, &h));
  const int limit = G.max_hn - 1;
  k_b_loop_cond<<<1, 256, 0, s>>>(h, G.mem, G.n, B->d_loop, 1, limit);
  FCM_LAUNCH_CHECK();
  cudaGraph_t body = nullptr;
  FCM_TRY(add_while_node(s, h, &body));
  const long long l0 = launch_count();
  FCM_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
  auto iteration = [&]() -> int {
    FCM_TRY(b_gm_fetch(G, bs));
    FCM_TRY(b_pinv(G, BV_SYS_B, BV_SYS_A, BM_GM, bs));
    if (prec == 0) FCM_TRY(batch_saddle<double>(B, BV_SYS_A, BV_SYS_B, BM_GM, bs));
    else FCM_TRY(batch_saddle<float>(B, BV_SYS_A, BV_SYS_B, BM_GM, bs));
    FCM_TRY(b_gm_orthogonalize(G, bs));
    k_b_loop_cond<<<1, 256, 0, bs>>>(h, G.mem, G.n, B->d_loop, 0, limit);
    FCM_LAUNCH_CHECK();
    return (int)FCM_OK;
  };
  const int st = iteration();
  cudaGraph_t tmp = nullptr;
  const cudaError_t e2 = cudaStreamEndCapture(bs, &tmp);
  if (st != FCM_OK) return st;
  if (e2 != cudaSuccess) {
    set_error(std::string("batch GMRES body capture: ") + cudaGetErrorString(e2));
    return FCM_ERR_CUDA;
  }
  B->k_iter = launch_count() - l0;
  FCM_TRY(b_gm_finish(G, s));
  FCM_TRY(b_pinv(G, BV_SYS_B, out, mask == BM_REF ? BM_REF : BM_ALL, s));
  return FCM_OK;
}

// Fork the members' branches off `s`, run fn(member index) on each branch
// (the member's c->stream swapped to the branch), join back into `s`.
template <typename F>
int batch_branches(Batch* B, cudaStream_t s, int fork_id, F&& fn) {
  const int n = B->geom.n;
  cudaEvent_t fork = B->events[fork_id];
  FCM_CUDA(cudaEventRecord(fork, s));
  for (int i = 0; i < n; ++i) {
    FCM_CUDA(cudaStreamWaitEvent(B->branch[i], fork, 0));
    {
      StreamSwap sw(B->m[i], B->branch[i]);
      FCM_TRY(fn(i));
    }
    cudaEvent_t join = B->events[2 + (size_t)fork_id * n + i];
    FCM_CUDA(cudaEventRecord(join, B->branch[i]));
    FCM_CUDA(cudaStreamWaitEvent(s, join, 0));
  }
  return FCM_OK;
}

// The pre-solve part of a step for one member (as enqueue_resident_step).
int member_pre_solve(Ctx* c) {
  const bool noise = c->p.noise != 0;
  FCM_TRY(launch_fill_blob_pos(*c, c->d_x, c->d_q, c->d_Y, c->stream));
  if (noise) FCM_TRY(noise_dev(c, 0, 0, c->d_stepargs));
  else c->urand_ready = false;
  FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
  FCM_TRY(random_velocities_dev(c, c->d_V));
  if (c->p.algorithm == 1) {
    int ov = 0;
    FCM_TRY(advance_to_midstep_dev(c, c->d_V, &ov));
    double* acc = c->d_H + c->maxit_alloc + 1;
    if (noise) FCM_TRY(divU_enqueue(c, acc));
    k_gdc_nu<<<1, 32, 0, c->stream>>>(c->d_step, acc, noise ? 1 : 0, c->p.dt, c->d_rs + 3);
    FCM_LAUNCH_CHECK();
    FCM_TRY(launch_fill_blob_pos(*c, c->d_xm, c->d_qm, c->d_Y, c->stream));
    FCM_TRY(set_up_gaussians_dev(c, c->d_Y));
    FCM_TRY(random_velocities_dev(c, c->d_V));
    if (c->shear) FCM_TRY(shear_velocities_dev(c));  // main.cpp:270-272
  }
  FCM_TRY(calculate_forces_dev(c));
  FCM_TRY(assemble_rhs_dev(c));
  return FCM_OK;
}

int enqueue_batch_step(Batch* B, cudaStream_t s) {
  const BatchGeom& G = B->geom;
  const int n = G.n;
  const long long l_start = launch_count();
  long long l_loops = 0;
  k_b_step_begin<<<1, 256, 0, s>>>(G.mem, n, B->d_loop);
  FCM_LAUNCH_CHECK();
  FCM_TRY(batch_branches(B, s, 0, [&](int i) { return member_pre_solve(B->m[i]); }));
  const double tol = B->m[0]->p.gmres_tol;
  if (B->precision == 0) {
    FCM_TRY(batch_gmres_loop(B, 0, BV_RHS, tol, 0, BM_ALL, BV_SOLN, s, B->cap_body[0]));
    l_loops += B->k_iter;
    B->k_sweep = 0;
    k_b_gm_record<<<1, 256, 0, s>>>(G.mem, n);
    FCM_LAUNCH_CHECK();
  } else {
    // r = b; x = 0; repeat: dx = GMRES32(r); x += dx; r = b - A64 x (solve_dev).
    k_b_refine_start<<<dim3(G.max_sys_blocks, n), 256, 0, s>>>(G.mem);
    FCM_LAUNCH_CHECK();
    FCM_TRY(b_norm(G, BV_RHS, BO_RS0, BM_ALL, s));
    cudaGraphConditionalHandle h;
    FCM_TRY(new_handle(s, &h));
    k_b_ref_enter<<<1, 256, 0, s>>>(h, G.mem, n);
    FCM_LAUNCH_CHECK();
    cudaGraph_t body = nullptr;
    FCM_TRY(add_while_node(s, h, &body));
    const long long l0 = launch_count();
    const cudaStream_t bs = B->cap_body[0];
    FCM_CUDA(cudaStreamBeginCaptureToGraph(bs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    auto sweep = [&]() -> int {
      k_b_ref_tol<<<1, 256, 0, bs>>>(G.mem, n, tol);
      FCM_LAUNCH_CHECK();
      FCM_TRY(batch_gmres_loop(B, 1, BV_RES, 0.0, 1, BM_REF, BV_DX, bs, B->cap_body[1]));
      FCM_TRY(b_axpby(G, BV_SOLN, BV_DX, 1.0, 1.0, BM_REF, bs));
      FCM_TRY(batch_saddle<double>(B, BV_SOLN, BV_RES, BM_REF, bs));
      FCM_TRY(b_axpby(G, BV_RES, BV_RHS, 1.0, -1.0, BM_REF, bs));
      FCM_TRY(b_norm(G, BV_RES, BO_RS1, BM_REF, bs));
      k_b_ref_next<<<1, 256, 0, bs>>>(h, G.mem, n, tol, kMaxSweeps, B->d_loop);
      FCM_LAUNCH_CHECK();
      return (int)FCM_OK;
    };
    const int st = sweep();
    cudaGraph_t tmp = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(bs, &tmp);
    if (st != FCM_OK) return st;
    if (e2 != cudaSuccess) {
      set_error(std::string("batch refinement body capture: ") + cudaGetErrorString(e2));
      return FCM_ERR_CUDA;
    }
    B->k_sweep = launch_count() - l0 - B->k_iter;
    l_loops += launch_count() - l0;
  }
  FCM_TRY(batch_branches(B, s, 1, [&](int i) {
    Ctx* c = B->m[i];
    int ov = 0;
    return end_of_step_update_dev(c, c->d_soln + 3 * (size_t)c->Nb, 1.0, &ov,
                                  c->p.algorithm == 1 ? c->d_rs + 3 : nullptr);
  }));
  FCM_CUDA(cudaMemcpyAsync(B->h_rec, B->d_rec, sizeof(StepRecord) * n, cudaMemcpyDeviceToHost, s));
  FCM_CUDA(cudaMemcpyAsync(B->h_loop, B->d_loop, sizeof(int) * 4, cudaMemcpyDeviceToHost, s));
  B->k_top = launch_count() - l_start - l_loops;
  return FCM_OK;
}

int build_batch_graph(Batch* B) {
  const long long l0 = launch_count();
  int st = FCM_OK;
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(B->cap, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    st = enqueue_batch_step(B, B->cap);
    const cudaError_t e2 = cudaStreamEndCapture(B->cap, &g);
    if (st == FCM_OK && e2 != cudaSuccess) {
      set_error(std::string("batch step capture: ") + cudaGetErrorString(e2));
      st = FCM_ERR_CUDA;
    }
  } else {
    set_error(std::string("cudaStreamBeginCapture: ") + cudaGetErrorString(e));
    st = FCM_ERR_CUDA;
  }
  count_launches(-(launch_count() - l0));  // counted per executed step instead
  if (st == FCM_OK) {
    e = cudaGraphInstantiate(&B->graph, g, 0);
    if (e != cudaSuccess) {
      set_error(std::string("batch step graph instantiate: ") + cudaGetErrorString(e));
      B->graph = nullptr;
      st = FCM_ERR_CUDA;
    }
  }
  if (g) cudaGraphDestroy(g);
  cudaGetLastError();
  B->state = st == FCM_OK ? 1 : -1;
  return st;
}

// The members' grids of precision T moved into one contiguous array per group
// of equal grids, with one cuFFT plan per group over all of them.
template <typename T>
int rehome_grids(Batch* B, int P) {
  for (BatchGroup& grp : B->groups) {
    const Ctx* c0 = B->m[grp.idx[0]];
    const size_t G = (size_t)c0->g.G, Gc = (size_t)c0->g.Gc, k = grp.idx.size();
    T* r = nullptr;
    typename cplx_t<T>::type* sp = nullptr;
    T* ur = nullptr;
    FCM_TRY(dev_alloc(&r, 3 * G * k));
    FCM_TRY(dev_alloc(&sp, 3 * Gc * k));
    FCM_TRY(dev_alloc(&ur, 3 * G * k));
    grp.r[P] = r;
    grp.c[P] = sp;
    grp.urand[P] = ur;
    FCM_CUDA(cudaMemset(ur, 0, sizeof(T) * 3 * G * k));
    for (size_t j = 0; j < k; ++j) {
      GridBufs<T>& gb = grid_of<T>(B->m[grp.idx[j]]);
      if (!gb.borrowed) {
        cudaFree(gb.r);
        cudaFree(gb.c);
        cudaFree(gb.urand);
      }
      gb.r = r + 3 * G * j;
      gb.c = sp + 3 * Gc * j;
      gb.urand = ur + 3 * G * j;
      gb.borrowed = true;
    }
    int nn[3] = {grp.nx, grp.ny, grp.nz};
    FCM_CUFFT(cufftPlanMany(&grp.r2c[P], 3, nn, nullptr, 1, (int)G, nullptr, 1, (int)Gc, r2c_type<T>(), (int)(3 * k)));
    FCM_CUFFT(cufftPlanMany(&grp.c2r[P], 3, nn, nullptr, 1, (int)Gc, nullptr, 1, (int)G, c2r_type<T>(), (int)(3 * k)));
    if (c0->xfft[P]) {
      int n2[2] = {grp.ny, grp.nz};
      const int pz = grp.ny * grp.nz, pc = grp.ny * (grp.nz / 2 + 1), planes = (int)(3 * grp.nx * k);
      FCM_CUFFT(cufftPlanMany(&grp.r2c2d[P], 2, n2, nullptr, 1, pz, nullptr, 1, pc, r2c_type<T>(), planes));
      FCM_CUFFT(cufftPlanMany(&grp.c2r2d[P], 2, n2, nullptr, 1, pc, nullptr, 1, pz, c2r_type<T>(), planes));
      if (!grp.d_gidx) {
        FCM_TRY(dev_alloc(&grp.d_gidx, k));
        FCM_CUDA(cudaMemcpy(grp.d_gidx, grp.idx.data(), sizeof(int) * k, cudaMemcpyHostToDevice));
      }
    }
  }
  return FCM_OK;
}

void destroy_batch(Batch* B) {
  if (!B) return;
  if (B->graph) cudaGraphExecDestroy(B->graph);
  for (Ctx* c : B->m) {
    c->d_step = nullptr;
    c->d_stepargs = nullptr;
    c->in_batch = false;
    destroy_ctx(c);
  }
  for (BatchGroup& g : B->groups)
    for (int P = 0; P < 2; ++P) {
      cudaFree(g.r[P]);
      cudaFree(g.c[P]);
      cudaFree(g.urand[P]);
      if (g.r2c[P]) cufftDestroy(g.r2c[P]);
      if (g.c2r[P]) cufftDestroy(g.c2r[P]);
      if (g.r2c2d[P]) cufftDestroy(g.r2c2d[P]);
      if (g.c2r2d[P]) cufftDestroy(g.c2r2d[P]);
    }
  for (BatchGroup& g : B->groups) cudaFree(g.d_gidx);
  cudaFree(B->d_mem);
  cudaFree(B->d_tile_map);
  cudaFree(B->d_kblock_map);
  cudaFree(B->d_partials);
  cudaFree(B->d_counter);
  cudaFree(B->d_mdpart);
  cudaFree(B->d_mdcount);
  cudaFree(B->d_rec);
  cudaFree(B->d_args);
  cudaFree(B->d_loop);
  if (B->h_rec) cudaFreeHost(B->h_rec);
  if (B->h_args) cudaFreeHost(B->h_args);
  if (B->h_loop) cudaFreeHost(B->h_loop);
  if (B->cap) cudaStreamDestroy(B->cap);
  for (int i = 0; i < 2; ++i)
    if (B->cap_body[i]) cudaStreamDestroy(B->cap_body[i]);
  for (cudaStream_t s : B->branch)
    if (s) cudaStreamDestroy(s);
  for (cudaEvent_t e : B->events)
    if (e) cudaEventDestroy(e);
  delete B;
}

int create_batch(int n, const fcm_params* params, const double* const* refs, Batch** out) {
  if (n < 1 || n > 4096 || !params || !refs) {
    set_error("batch: 1 <= n <= 4096 members with params and blob_ref_pos each");
    return FCM_ERR_INVALID;
  }
  for (int i = 0; i < n; ++i) {
    if (params[i].precision != params[0].precision || params[i].gmres_tol != params[0].gmres_tol) {
      set_error("batch: every member needs the same precision and gmres_tol");
      return FCM_ERR_INVALID;
    }
    if (params[i].skip_on_overlap || params[i].slip_channel) {
      set_error("batch: members step without overlap rejection (skip_on_overlap = 0, slip_channel = 0)");
      return FCM_ERR_INVALID;
    }
  }
  Batch* B = new Batch();
  auto fail = [&](int s) {
    destroy_batch(B);
    return s;
  };
  B->precision = params[0].precision;
  for (int i = 0; i < n; ++i) {
    Ctx* c = nullptr;
    const int st = create_ctx(&params[i], refs[i], &c);
    if (st != FCM_OK) return fail(st);
    B->m.push_back(c);
    c->in_batch = true;
    c->step_graph_state = -1;
    if (!c->g64.blobs.tiled || (B->precision == 1 && !c->g32.blobs.tiled)) {
      set_error("batch: member " + std::to_string(i) +
                " has a grid the tiled kernels cannot take (dimensions multiples of 8, at least ngauss + 8, "
                "ngauss <= 25)");
      return fail(FCM_ERR_INVALID);
    }
  }
  for (int i = 0; i < n; ++i) {  // groups of equal grids
    const Ctx* c = B->m[i];
    BatchGroup* g = nullptr;
    for (BatchGroup& x : B->groups)
      if (x.nx == c->g.nx && x.ny == c->g.ny && x.nz == c->g.nz) g = &x;
    if (!g) {
      B->groups.emplace_back();
      g = &B->groups.back();
      g->nx = c->g.nx;
      g->ny = c->g.ny;
      g->nz = c->g.nz;
    }
    g->idx.push_back(i);
  }
  int st = rehome_grids<double>(B, 0);
  if (st == FCM_OK && B->precision == 1) st = rehome_grids<float>(B, 1);
  if (st != FCM_OK) return fail(st);
  BatchGeom& G = B->geom;
  G.n = n;
  long long max_sys = 1, max_Nb = 1, max_M = 1;
  for (const Ctx* c : B->m) {
    max_sys = std::max<long long>(max_sys, c->nsys);
    max_Nb = std::max<long long>(max_Nb, c->Nb);
    max_M = std::max<long long>(max_M, c->M);
    G.max_nb = std::max(G.max_nb, c->nb);
    G.max_hn = std::max(G.max_hn, c->maxit_alloc + 1);
    G.red_blocks = std::max(G.red_blocks, c->red_blocks);
    G.md_blocks = std::max(G.md_blocks, c->md_blocks);
    G.total_tiles += c->g64.blobs.ntiles;
    if (!(c->xfft[0] && c->xfft[1])) G.total_kblocks += (int)((c->g.Gc + 255) / 256);  // k_b_project's share
  }
  G.max_sys_blocks = (int)((max_sys + 255) / 256);
  G.max_blob_blocks = (int)((max_Nb + 127) / 128);
  G.max_body_blocks = (int)((max_M + 127) / 128);
  G.max_pinv_blocks = (int)((max_M + 3) / 4);
  if ((st = dev_alloc(&B->d_mem, (size_t)n)) || (st = dev_alloc(&B->d_tile_map, (size_t)G.total_tiles)) ||
      (st = dev_alloc(&B->d_kblock_map, (size_t)G.total_kblocks)) ||
      (st = dev_alloc(&B->d_partials, (size_t)n * G.red_blocks)) || (st = dev_alloc(&B->d_counter, (size_t)n)) ||
      (st = dev_alloc(&B->d_mdpart, (size_t)n * G.max_hn * G.md_blocks)) ||
      (st = dev_alloc(&B->d_mdcount, (size_t)n * G.max_hn)) || (st = dev_alloc(&B->d_rec, (size_t)n)) ||
      (st = dev_alloc(&B->d_args, 2 * (size_t)n)) || (st = dev_alloc(&B->d_loop, 4)))
    return fail(st);
  if (cudaMemset(B->d_counter, 0, sizeof(unsigned) * n) != cudaSuccess ||
      cudaMemset(B->d_loop, 0, sizeof(int) * 4) != cudaSuccess ||
      cudaMemset(B->d_mdcount, 0, sizeof(unsigned) * n * G.max_hn) != cudaSuccess ||
      cudaMemset(B->d_rec, 0, sizeof(StepRecord) * n) != cudaSuccess ||
      cudaMallocHost(&B->h_rec, sizeof(StepRecord) * n) != cudaSuccess ||
      cudaMallocHost(&B->h_args, 2 * sizeof(uint64_t) * n) != cudaSuccess ||
      cudaMallocHost(&B->h_loop, 4 * sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    set_error("batch: allocation failed");
    return fail(FCM_ERR_NOMEM);
  }
  std::vector<BMember> hm(n);
  std::vector<int2> tmap, kmap;
  tmap.reserve(G.total_tiles);
  kmap.reserve(G.total_kblocks);
  for (int i = 0; i < n; ++i) {
    Ctx* c = B->m[i];
    if ((st = dev_alloc(&c->d_rs, 8)) != FCM_OK) return fail(st);
    c->d_step = B->d_rec + i;
    c->d_stepargs = B->d_args + 2 * i;
    BMember& m = hm[i];
    std::memset(&m, 0, sizeof(m));
    m.Nb = c->Nb;
    m.M = c->M;
    m.nb = c->nb;
    m.nsys = c->nsys;
    m.hn = c->maxit_alloc + 1;
    m.red_blocks = c->red_blocks;
    m.md_blocks = c->md_blocks;
    m.qm = c->d_qm;
    m.ref = c->d_ref;
    m.Minv = c->d_Minv;
    m.N = c->d_N;
    m.ref_stride = c->ref_stride;
    m.minv_stride = c->minv_stride;
    m.n_stride = c->n_stride;
    m.sys_a = c->d_sys_a;
    m.sys_b = c->d_sys_b;
    m.rhs = c->d_rhs;
    m.soln = c->d_soln;
    m.res = c->d_res;
    m.dx = c->d_dx;
    m.gm = c->gm;
    m.Qm = c->d_Qm;
    m.Hd = c->d_Hd;
    m.beta = c->d_beta;
    m.CS = c->d_CS;
    m.SN = c->d_SN;
    m.hA = c->d_hA;
    m.hB = c->d_hB;
    m.hnorm = c->d_hnorm;
    m.y = c->d_y;
    m.partials = B->d_partials + (size_t)i * G.red_blocks;
    m.counter = B->d_counter + i;
    m.mdpart = B->d_mdpart + (size_t)i * G.max_hn * G.md_blocks;
    m.mdcount = B->d_mdcount + (size_t)i * G.max_hn;
    m.sd = B->d_rec + i;
    m.rs = c->d_rs;
    m.wc[0] = c->g64.blobs.wc;
    m.toff[0] = c->g64.blobs.tile_offset;
    m.tlist[0] = c->g64.blobs.tile_list;
    m.base[0] = c->g64.blobs.base;
    m.grid[0] = c->g64.r;
    m.spec[0] = c->g64.c;
    m.partial[0] = c->g64.blobs.partial;
    if (B->precision == 1) {
      m.wc[1] = c->g32.blobs.wc;
      m.toff[1] = c->g32.blobs.tile_offset;
      m.tlist[1] = c->g32.blobs.tile_list;
      m.base[1] = c->g32.blobs.base;
      m.grid[1] = c->g32.r;
      m.spec[1] = c->g32.c;
      m.partial[1] = c->g32.blobs.partial;
    }
    m.tg[0] = tile_geom(c->g, c->g64.blobs);
    m.tg[1] = B->precision == 1 ? tile_geom(c->g, c->g32.blobs) : tile_geom(c->g, c->g64.blobs);
    m.kp = make_kparams(*c);
    m.dx3 = c->g.dx * c->g.dx * c->g.dx;
    m.xfft[0] = c->xfft[0] ? 1 : 0;
    m.xfft[1] = c->xfft[1] ? 1 : 0;
    for (int t = 0; t < c->g64.blobs.ntiles; ++t) tmap.push_back(make_int2(i, t));
    const int kb = (c->xfft[0] && c->xfft[1]) ? 0 : (int)((c->g.Gc + 255) / 256);
    for (int t = 0; t < kb; ++t) kmap.push_back(make_int2(i, t));
  }
  if (cudaMemcpy(B->d_mem, hm.data(), sizeof(BMember) * n, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(B->d_tile_map, tmap.data(), sizeof(int2) * tmap.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(B->d_kblock_map, kmap.data(), sizeof(int2) * kmap.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
    set_error("batch: descriptor upload failed");
    return fail(FCM_ERR_CUDA);
  }
  G.mem = B->d_mem;
  G.tile_map = B->d_tile_map;
  G.kblock_map = B->d_kblock_map;
  B->branch.assign(n, nullptr);
  B->events.assign(2 + 2 * (size_t)n, nullptr);
  bool ok = cudaStreamCreateWithFlags(&B->cap, cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&B->cap_body[0], cudaStreamNonBlocking) == cudaSuccess &&
            cudaStreamCreateWithFlags(&B->cap_body[1], cudaStreamNonBlocking) == cudaSuccess;
  for (int i = 0; ok && i < n; ++i) ok = cudaStreamCreateWithFlags(&B->branch[i], cudaStreamNonBlocking) == cudaSuccess;
  for (size_t i = 0; ok && i < B->events.size(); ++i)
    ok = cudaEventCreateWithFlags(&B->events[i], cudaEventDisableTiming) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    set_error("batch: stream or event creation failed");
    return fail(FCM_ERR_CUDA);
  }
  *out = B;
  return FCM_OK;
}

// One step of every member.  The first call steps the members host-driven
// (allocating what they need) and then captures the batch graph.
int batch_step(Batch* B, const uint64_t* seeds, uint64_t step_index, fcm_step_info* infos) {
  const int n = B->geom.n;
  bool stale = false;
  for (Ctx* c : B->m) {
    stale = stale || c->graph_stale;
    c->graph_stale = false;
  }
  if (stale && B->state == 1) {  // recapture after a change of a member's step
    cudaGraphExecDestroy(B->graph);
    B->graph = nullptr;
    B->state = 0;
  }
  if (B->state != 1) {
    int first = FCM_OK;
    std::string err;
    for (int i = 0; i < n; ++i) {
      fcm_step_info inf;
      std::memset(&inf, 0, sizeof(inf));
      const int st = step_host(B->m[i], seeds[i], step_index, &inf);
      if (infos) infos[i] = inf;
      if (st != FCM_OK && first == FCM_OK) {
        first = st;
        err = g_err;
      }
    }
    for (int i = 0; i < n; ++i) FCM_CUDA(cudaStreamSynchronize(B->m[i]->stream));
    if (first != FCM_OK) {
      set_error(err);
      return first;
    }
    if (B->state == 0) {
      const std::string keep = g_err;
      if (build_batch_graph(B) != FCM_OK) set_error(keep);  // host-driven steps from now on
    }
    return FCM_OK;
  }
  for (int i = 0; i < n; ++i) {
    B->h_args[2 * i] = seeds[i];
    B->h_args[2 * i + 1] = step_index;
  }
  FCM_CUDA(cudaMemcpyAsync(B->d_args, B->h_args, 2 * sizeof(uint64_t) * n, cudaMemcpyHostToDevice, B->stream));
  FCM_CUDA(cudaGraphLaunch(B->graph, B->stream));
  FCM_CUDA(cudaStreamSynchronize(B->stream));
  count_launches(B->k_top + (long long)B->h_loop[2] * B->k_sweep + (long long)B->h_loop[1] * B->k_iter);
  int first = FCM_OK;
  for (int i = 0; i < n; ++i) {
    Ctx* c = B->m[i];
    const StepRecord& r = B->h_rec[i];
    c->gauss_ready = true;
    c->urand_ready = c->p.noise != 0;
    c->urand_prec = noise_precision(c);
    if (infos) {
      fcm_step_info& inf = infos[i];
      std::memset(&inf, 0, sizeof(inf));
      inf.gmres_iters = r.iters;
      inf.refinement_sweeps = r.sweeps;
      inf.gmres_rel_residual = r.rel;
      inf.divU = r.divU;
      inf.status = r.status;
    }
    if (r.status != FCM_OK && r.status != FCM_ERR_NOT_CONVERGED) {
      // as in a host-driven step, a failed solve leaves the bodies where they were
      FCM_CUDA(cudaMemcpyAsync(c->d_x, c->d_xs, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, B->stream));
      FCM_CUDA(cudaMemcpyAsync(c->d_q, c->d_qs, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, B->stream));
      if (first == FCM_OK) first = r.status;
    }
  }
  if (first != FCM_OK) {
    FCM_CUDA(cudaStreamSynchronize(B->stream));
    set_error("a batch member's solve failed (non-finite residual); its bodies were left unchanged");
  }
  return first;
}

}  // namespace
}  // namespace fcm

struct fcm_ctx {
  fcm::Ctx* c;
};

struct fcm_batch {
  fcm::Batch* b;
  std::vector<fcm_ctx> members;
};

using namespace fcm;

// ------------------------------------------------------------------ kernel variants
// Solve variant of precision P: 0 = 3D transforms, 1 = fused x-transform with
// cuFFT's (y, z) plans, 2 = with the library's (y, z) kernels.
static int solve_variant(const Ctx* c, int P) {
  if (!c->xfft[P]) return 0;
  return (P == 1 && c->yz32) ? 2 : 1;
}

static void get_variants(const Ctx* c, int32_t* v) {
  v[0] = c->spread_variant[0];
  v[1] = solve_variant(c, 0);
  v[2] = c->spread_variant[1];
  v[3] = solve_variant(c, 1);
  v[4] = c->interp_variant[0];
  v[5] = c->interp_variant[1];
}

static int set_variants(Ctx* c, const int32_t* v) {
  for (int P = 0; P < 2; ++P) {
    const int sp = v[2 * P], sv = v[2 * P + 1], iv = v[4 + P];
    // the tensor-core spread (5) and interpolation (3) exist for FP32 grids only
    if (sp < 0 || sp > (P == 1 ? 5 : 4) || sv < 0 || sv > (P == 1 ? 2 : 1) || iv < 0 || iv > (P == 1 ? 3 : 2)) {
      set_error("kernel variant out of range");
      return FCM_ERR_INVALID;
    }
    if (P == 1 && c->p.precision != 1) continue;  // no FP32 grid
    if ((sv >= 1 && !c->xfft_cap[P]) || (sv == 2 && !c->yz32_cap)) {
      set_error("this grid does not allow solve variant " + std::to_string(sv));
      return FCM_ERR_INVALID;
    }
  }
  for (int P = 0; P < 2; ++P) {
    if (P == 1 && c->p.precision != 1) continue;
    c->spread_variant[P] = v[2 * P];
    c->xfft[P] = v[2 * P + 1] >= 1;
    if (P == 1) c->yz32 = v[3] == 2;
    c->interp_variant[P] = v[4 + P];
  }
  c->graph_stale = true;
  return FCM_OK;
}

struct EventPair {
  cudaEvent_t a = nullptr, b = nullptr;
  ~EventPair() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Mean microseconds of one call of body() on c's stream: one untimed call, then
// reps timed ones between two events.
template <class F>
static int time_calls(Ctx* c, int reps, F&& body, double* out) {
  FCM_TRY(body());
  EventPair ev;
  FCM_CUDA(cudaEventCreate(&ev.a));
  FCM_CUDA(cudaEventCreate(&ev.b));
  FCM_CUDA(cudaEventRecord(ev.a, c->stream));
  for (int i = 0; i < reps; ++i) FCM_TRY(body());
  FCM_CUDA(cudaEventRecord(ev.b, c->stream));
  FCM_CUDA(cudaEventSynchronize(ev.b));
  float ms = 0.f;
  FCM_CUDA(cudaEventElapsedTime(&ms, ev.a, ev.b));
  *out = 1e3 * (double)ms / reps;
  return FCM_OK;
}

// The spread, solve and interpolation variants of one precision timed on c's own
// grid and blob table; the fastest kept.  t[0..5] spread, t[6..8] solve, t[9..12]
// interpolation (-1: not available; the tensor-core spread 5 and interpolation 3
// are FP32 only).
template <typename T>
static int tune_precision(Ctx* c, int reps, double* t) {
  constexpr int P = sizeof(T) == 8 ? 0 : 1;
  GridBufs<T>& gb = grid_of<T>(c);
  const BlobTable<T>& bt = gb.blobs;
  FCM_CUDA(cudaMemsetAsync(c->d_tmp3, 0, sizeof(double) * 3 * (size_t)(c->Nb > 0 ? c->Nb : 1), c->stream));
  constexpr int NSP = P == 1 ? 6 : 5, NIP = P == 1 ? 4 : 3;
  if (bt.tiled) {
    for (int v = 0; v < NSP; ++v) {
      c->spread_variant[P] = v;
      FCM_TRY(time_calls(c, reps, [&] { return spread_t<T>(c, bt, c->d_tmp3); }, &t[v]));
    }
    int bs = 0;
    for (int v = 1; v < NSP; ++v)
      if (t[v] < t[bs]) bs = v;
    c->spread_variant[P] = bs;
  }
  FCM_CUDA(cudaMemsetAsync(gb.r, 0, sizeof(T) * 3 * (size_t)c->g.G, c->stream));
  for (int v = 0; v < 3; ++v) {
    if ((v >= 1 && !c->xfft_cap[P]) || (v == 2 && (P == 0 || !c->yz32_cap))) continue;
    c->xfft[P] = v >= 1;
    if (P == 1) c->yz32 = v == 2;
    FCM_TRY(time_calls(c, reps, [&] { return stokes_t<T>(c); }, &t[6 + v]));
  }
  int best = 0;
  for (int v = 1; v < 3; ++v)
    if (t[6 + v] >= 0.0 && t[6 + v] < t[6 + best]) best = v;
  c->xfft[P] = best >= 1;
  if (P == 1) c->yz32 = best == 2;
  if (bt.tiled) {  // interpolation of the (zeroed) grid into scratch
    for (int v = 0; v < NIP; ++v) {
      c->interp_variant[P] = v;
      FCM_TRY(time_calls(c, reps, [&] { return interp_t<T>(c, bt, gb.r, c->d_tmp3); }, &t[9 + v]));
    }
    int bi = 0;
    for (int v = 1; v < NIP; ++v)
      if (t[9 + v] < t[9 + bi]) bi = v;
    c->interp_variant[P] = bi;
  }
  return FCM_OK;
}

extern "C" {

void fcm_default_params(fcm_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  const double a = 1.0, eta = 1.0, kT = 1.0;
  p->nx = p->ny = p->nz = 256;  // config.hpp:65-67
  p->ngauss = 20;               // :69
  p->dx = a * 0.3033277330901916;
  p->blob_radius = a;
  p->viscosity = eta;
  p->kT = kT;
  p->dt = (PI * eta * a * a * a / kT) / 100.0;
  p->num_bodies = 3;
  p->blobs_per_body = 22;
  p->ncells = 6;
  p->potential = 0;
  p->steric_fs = 40.0 * kT / a;
  p->steric_rc = 2.2 * a;
  p->gmres_max_iter = 40;
  p->gmres_tol = 1e-3;
  p->fd_delta = 1e-5;
  p->algorithm = 2;
  p->precision = 0;
  p->noise = 1;
  p->skip_on_overlap = 0;
  p->slip_channel = 0;
}

const char* fcm_last_error(void) { return g_err.c_str(); }
const char* fcm_version(void) { return "fcm_b200 0.1 (sm_100a)"; }
int64_t fcm_kernel_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int fcm_debug_bounds(int32_t* checked, int64_t* count, int32_t* site, int64_t* index, int64_t* limit,
                     int32_t reset) {
  return guard([&] {
#ifdef FCM_BOUNDS_CHECK
    const int on = 1;
    FCM_CUDA(cudaDeviceSynchronize());
#else
    const int on = 0;
#endif
    int (*readers[])(BoundsRecord*, int) = {bounds_read_grid, bounds_read_cells, bounds_read_kspace,
                                            bounds_read_blas};
    unsigned long long total = 0;
    BoundsRecord first{};
    for (auto rd : readers) {
      BoundsRecord r{};
      FCM_TRY(rd(&r, reset));
      if (r.count && !total) first = r;
      total += r.count;
    }
    if (checked) *checked = on;
    if (count) *count = (int64_t)total;
    if (site) *site = total ? first.site : 0;
    if (index) *index = total ? first.index : 0;
    if (limit) *limit = total ? first.limit : 0;
    return (int)FCM_OK;
  });
}

int fcm_create(const fcm_params* p, const double* blob_ref_pos, fcm_ctx** out) {
  return guard([&] {
    if (!out) return (int)FCM_ERR_INVALID;
    *out = nullptr;
    Ctx* c = nullptr;
    const int st = create_ctx(p, blob_ref_pos, &c);
    if (st != FCM_OK) return st;
    *out = new fcm_ctx{c};
    return (int)FCM_OK;
  });
}

int fcm_destroy(fcm_ctx* ctx) {
  if (!ctx) return FCM_OK;
  if (ctx->c && ctx->c->in_batch) {
    set_error("this context belongs to a batch: destroy the batch instead");
    return FCM_ERR_INVALID;
  }
  if (ctx->c) cudaStreamSynchronize(ctx->c->stream);
  destroy_ctx(ctx->c);
  delete ctx;
  return FCM_OK;
}

int fcm_set_stream(fcm_ctx* ctx, void* stream) {
  CTX_CHECK(ctx);
  ctx->c->stream = (cudaStream_t)stream;
  return set_stream_all(ctx->c);
}

int fcm_get_params(const fcm_ctx* ctx, fcm_params* p) {
  CTX_CHECK(ctx);
  if (!p) return FCM_ERR_INVALID;
  *p = ctx->c->p;
  return FCM_OK;
}

// ------------------------------------------------------------------ bodies
int fcm_set_bodies(fcm_ctx* ctx, const double* x, const double* q) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_in(c, c->d_x, x, sizeof(double) * 3 * c->M));
  FCM_TRY(copy_in(c, c->d_q, q, sizeof(double) * 4 * c->M));
  FCM_CUDA(cudaMemcpyAsync(c->d_xm, c->d_x, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->d_qm, c->d_q, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  return FCM_OK;
}

int fcm_get_bodies(fcm_ctx* ctx, double* x, double* q) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_out(c, x, c->d_x, sizeof(double) * 3 * c->M));
  FCM_TRY(copy_out(c, q, c->d_q, sizeof(double) * 4 * c->M));
  return FCM_OK;
}

int fcm_get_midstep_bodies(fcm_ctx* ctx, double* x, double* q) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_out(c, x, c->d_xm, sizeof(double) * 3 * c->M));
  FCM_TRY(copy_out(c, q, c->d_qm, sizeof(double) * 4 * c->M));
  return FCM_OK;
}

int fcm_set_external_forces(fcm_ctx* ctx, const double* fe) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!fe) {
    FCM_CUDA(cudaMemsetAsync(c->d_fe, 0, sizeof(double) * 6 * c->M, c->stream));
    return FCM_OK;
  }
  return copy_in(c, c->d_fe, fe, sizeof(double) * 6 * c->M);
}

int fcm_fill_all_blob_pos(fcm_ctx* ctx, int32_t at_midstep) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  return launch_fill_blob_pos(*c, at_midstep ? c->d_xm : c->d_x, at_midstep ? c->d_qm : c->d_q, c->d_Y, c->stream);
}

int fcm_set_all_blob_pos(fcm_ctx* ctx, const double* Y) {
  CTX_CHECK(ctx);
  return copy_in(ctx->c, ctx->c->d_Y, Y, sizeof(double) * 3 * ctx->c->Nb);
}

int fcm_get_all_blob_pos(fcm_ctx* ctx, double* Y) {
  CTX_CHECK(ctx);
  return copy_out(ctx->c, Y, ctx->c->d_Y, sizeof(double) * 3 * ctx->c->Nb);
}

int fcm_multiply_by_K_at_midstep(fcm_ctx* ctx, const double* in, double* out) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_in(c, c->d_tmp6, in, sizeof(double) * 6 * c->M));
  FCM_TRY(launch_multiply_K(*c, c->d_qm, c->d_tmp6, c->d_tmp3, 0.0, c->stream));
  return copy_out(c, out, c->d_tmp3, sizeof(double) * 3 * c->Nb);
}

int fcm_multiply_by_KT_at_midstep(fcm_ctx* ctx, const double* in, double* out) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_in(c, c->d_tmp3, in, sizeof(double) * 3 * c->Nb));
  FCM_TRY(launch_multiply_KT(*c, c->d_qm, c->d_tmp3, c->d_tmp6, 1.0, nullptr, 0.0, c->stream));
  return copy_out(c, out, c->d_tmp6, sizeof(double) * 6 * c->M);
}

int fcm_calculate_forces(fcm_ctx* ctx) {
  CTX_CHECK(ctx);
  return calculate_forces_dev(ctx->c);
}

int fcm_get_blob_forces(fcm_ctx* ctx, double* F) {
  CTX_CHECK(ctx);
  return copy_out(ctx->c, F, ctx->c->d_F, sizeof(double) * 3 * ctx->c->Nb);
}

int fcm_set_blob_forces(fcm_ctx* ctx, const double* F) {
  CTX_CHECK(ctx);
  return copy_in(ctx->c, ctx->c->d_F, F, sizeof(double) * 3 * ctx->c->Nb);
}

int fcm_advance_to_midstep(fcm_ctx* ctx, const double* V, int32_t* overlap) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (V) FCM_TRY(copy_in(c, c->d_V, V, sizeof(double) * 3 * c->Nb));
  int ov = 0;
  FCM_TRY(advance_to_midstep_dev(c, c->d_V, &ov));
  if (overlap) *overlap = ov;
  return FCM_OK;
}

int fcm_calculate_divU(fcm_ctx* ctx, double* divU) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->urand_ready) {
    set_error("calculate_divU needs a random velocity field");
    return FCM_ERR_STATE;
  }
  double d = 0.0;
  FCM_TRY(divU_dev(c, &d));
  if (divU) *divU = d;
  return FCM_OK;
}

int fcm_end_of_step_update(fcm_ctx* ctx, const double* U, double nu, int32_t* overlap) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_in(c, c->d_tmp6, U, sizeof(double) * 6 * c->M));
  int ov = 0;
  FCM_TRY(end_of_step_update_dev(c, c->d_tmp6, nu, &ov));
  if (overlap) *overlap = ov;
  return FCM_OK;
}

int fcm_reset_to_start_of_step(fcm_ctx* ctx) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_CUDA(cudaMemcpyAsync(c->d_x, c->d_xs, sizeof(double) * 3 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  FCM_CUDA(cudaMemcpyAsync(c->d_q, c->d_qs, sizeof(double) * 4 * c->M, cudaMemcpyDeviceToDevice, c->stream));
  return FCM_OK;
}

int fcm_check_for_overlap(fcm_ctx* ctx, int32_t* overlap) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(cells_build(*c, c->stream));
  int ov = 0;
  FCM_TRY(overlap_dev(c, &ov));
  if (overlap) *overlap = ov;
  return FCM_OK;
}

int fcm_check_for_channel_wall_overlap(fcm_ctx* ctx, int32_t* overlap) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  int ov = 0;
  if (c->p.slip_channel) FCM_TRY(overlap_dev(c, &ov, false, true));
  if (overlap) *overlap = ov;
  return FCM_OK;
}

// ------------------------------------------------------------------ linked_list
int fcm_list_populate(fcm_ctx* ctx) {
  CTX_CHECK(ctx);
  return cells_build(*ctx->c, ctx->c->stream);
}

int fcm_list_get_cells(fcm_ctx* ctx, int32_t* cell) {
  CTX_CHECK(ctx);
  return copy_out(ctx->c, cell, ctx->c->d_cell, sizeof(int) * ctx->c->Nb);
}

int fcm_list_get_pairs(fcm_ctx* ctx, int32_t* pairs, int64_t cap, int64_t* npairs) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    FCM_TRY(cells_count_pairs(*c, c->d_pair_count, nullptr, 0, c->stream));
    long long n = 0;
    FCM_CUDA(cudaMemcpyAsync(&n, c->d_pair_count, sizeof(long long), cudaMemcpyDeviceToHost, c->stream));
    FCM_CUDA(cudaStreamSynchronize(c->stream));
    if (npairs) *npairs = n;
    if (!pairs) return (int)FCM_OK;
    if (n > cap) {
      set_error("pair buffer too small");
      return (int)FCM_ERR_CAPACITY;
    }
    int* dp = nullptr;
    FCM_TRY(dev_alloc(&dp, 2 * (size_t)std::max<long long>(n, 1)));
    int st = cells_count_pairs(*c, c->d_pair_count, dp, n, c->stream);
    std::vector<int> h(2 * (size_t)n);
    if (st == FCM_OK && n > 0 &&
        cudaMemcpyAsync(h.data(), dp, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
      st = FCM_ERR_CUDA;
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) st = FCM_ERR_CUDA;
    cudaFree(dp);
    if (st != FCM_OK) return st;
    std::vector<std::pair<int, int>> v((size_t)n);
    for (long long i = 0; i < n; ++i) v[i] = std::make_pair(h[2 * i], h[2 * i + 1]);
    std::sort(v.begin(), v.end());
    std::vector<int> outv(2 * (size_t)n);
    for (long long i = 0; i < n; ++i) {
      outv[2 * i] = v[i].first;
      outv[2 * i + 1] = v[i].second;
    }
    if (n > 0) {
      FCM_CUDA(cudaMemcpyAsync(pairs, outv.data(), sizeof(int) * 2 * n, cudaMemcpyDefault, c->stream));
      FCM_CUDA(cudaStreamSynchronize(c->stream));
    }
    return (int)FCM_OK;
  });
}

int fcm_apply_barrier_forces(fcm_ctx* ctx, double* blob_forces) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!blob_forces) return FCM_ERR_INVALID;
  FCM_TRY(copy_in(c, c->d_tmp3, blob_forces, sizeof(double) * 3 * c->Nb));
  FCM_TRY(cells_steric_forces(*c, c->d_tmp3, true, c->stream));
  return copy_out(c, blob_forces, c->d_tmp3, sizeof(double) * 3 * c->Nb);
}

// ------------------------------------------------------------------ fcm_fluid_solver
int fcm_set_up_gaussians(fcm_ctx* ctx, const double* Y) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (Y) FCM_TRY(copy_in(c, c->d_Y, Y, sizeof(double) * 3 * c->Nb));
  return set_up_gaussians_dev(c, c->d_Y);
}

int fcm_get_gaussians(fcm_ctx* ctx, int32_t precision, int32_t* ind, double* w) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->gauss_ready) {
    set_error("fcm_get_gaussians: set_up_gaussians must come first");
    return FCM_ERR_STATE;
  }
  if (precision != 0 && !(precision == 1 && c->p.precision == 1)) {
    set_error("fcm_get_gaussians: precision must be 0, or 1 in a context of precision 1");
    return FCM_ERR_INVALID;
  }
  const int n = c->Nb;
  const int W = precision == 0 ? c->g64.blobs.W : c->g32.blobs.W;
  const int* d_base = precision == 0 ? c->g64.blobs.base : c->g32.blobs.base;
  std::vector<int> base(3 * (size_t)n);
  FCM_CUDA(cudaMemcpyAsync(base.data(), d_base, sizeof(int) * base.size(), cudaMemcpyDeviceToHost, c->stream));
  std::vector<double> wt;
  if (w) {
    wt.resize(3 * (size_t)n * W);
    if (precision == 0) {
      FCM_CUDA(cudaMemcpyAsync(wt.data(), c->g64.blobs.w, sizeof(double) * wt.size(), cudaMemcpyDeviceToHost,
                               c->stream));
    } else {
      std::vector<float> wf(wt.size());
      FCM_CUDA(cudaMemcpyAsync(wf.data(), c->g32.blobs.w, sizeof(float) * wf.size(), cudaMemcpyDeviceToHost,
                               c->stream));
      FCM_CUDA(cudaStreamSynchronize(c->stream));
      for (size_t i = 0; i < wf.size(); ++i) wt[i] = wf[i];
    }
  }
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  const int nd[3] = {c->g.nx, c->g.ny, c->g.nz};
  for (int b = 0; b < n; ++b)
    for (int d = 0; d < 3; ++d) {
      const size_t row = (3 * (size_t)b + d) * W;
      for (int i = 0; i < W; ++i) {
        const int xg = base[3 * (size_t)b + d] + i;  // fcm_fluid_solver.cpp:141-151
        const int r = xg % nd[d];
        if (ind) ind[row + i] = r < 0 ? r + nd[d] : r;
        if (w) w[row + i] = wt[row + i];
      }
    }
  return FCM_OK;
}

int fcm_produce_random_velocity_field(fcm_ctx* ctx, uint64_t seed, uint64_t counter) {
  CTX_CHECK(ctx);
  return noise_dev(ctx->c, seed, counter);
}

int fcm_inject_random_stress(fcm_ctx* ctx, const double* sxx, const double* syy, const double* szz,
                             const double* sxy, const double* sxz, const double* syz) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    const double* s[6] = {sxx, syy, szz, sxy, sxz, syz};
    for (int i = 0; i < 6; ++i)
      if (!s[i]) {
        set_error("null stress array");
        return (int)FCM_ERR_INVALID;
      }
    if (!c->d_stress) {
      FCM_TRY(dev_alloc(&c->d_stress, 6 * (size_t)c->g.G));
      FCM_TRY(dev_alloc(&c->d_stress_c, 6 * (size_t)c->g.Gc));
      int n[3] = {c->g.nx, c->g.ny, c->g.nz};
      FCM_CUFFT(cufftPlanMany(&c->plan_r2c6, 3, n, nullptr, 1, (int)c->g.G, nullptr, 1, (int)c->g.Gc, CUFFT_D2Z, 6));
      FCM_CUFFT(cufftSetStream(c->plan_r2c6, c->stream));
    }
    for (int i = 0; i < 6; ++i) FCM_TRY(padded_to_grid(c, c->d_stress + (size_t)i * c->g.G, s[i]));
    FCM_CUFFT(cufftExecD2Z(c->plan_r2c6, c->d_stress, c->d_stress_c));
    FCM_TRY(launch_stress_divergence_project(*c, c->d_stress_c, c->g64.c, c->stream));
    FCM_CUFFT(cufftExecZ2D(c->g64.c2r, c->g64.c, c->g64.urand));
    c->urand_prec = 0;
    c->urand_ready = true;
    FCM_CUDA(cudaStreamSynchronize(c->stream));  // host stress arrays are borrowed
    return (int)FCM_OK;
  });
}

int fcm_calculate_random_blob_velocities(fcm_ctx* ctx, double* V) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede interpolation");
    return FCM_ERR_STATE;
  }
  FCM_TRY(random_velocities_dev(c, c->d_V));
  return copy_out(c, V, c->d_V, sizeof(double) * 3 * c->Nb);
}

int fcm_set_up_force_distribution(fcm_ctx* ctx, const double* F) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede spreading");
    return FCM_ERR_STATE;
  }
  FCM_TRY(copy_in(c, c->d_tmp3, F, sizeof(double) * 3 * c->Nb));
  c->det_ready = false;
  return spread_t<double>(c, c->g64.blobs, c->d_tmp3);
}

int fcm_produce_deterministic_velocity_field(fcm_ctx* ctx) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(stokes_t<double>(c));
  c->det_ready = true;
  return FCM_OK;
}

int fcm_calculate_deterministic_blob_velocities(fcm_ctx* ctx, double* V) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede interpolation");
    return FCM_ERR_STATE;
  }
  FCM_TRY(interp_t<double>(c, c->g64.blobs, c->g64.r, c->d_V));
  return copy_out(c, V, c->d_V, sizeof(double) * 3 * c->Nb);
}

int fcm_get_V(fcm_ctx* ctx, double* V) {
  CTX_CHECK(ctx);
  return copy_out(ctx->c, V, ctx->c->d_V, sizeof(double) * 3 * ctx->c->Nb);
}

int fcm_get_velocity_field(fcm_ctx* ctx, int32_t which, double* ux, double* uy, double* uz) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    double* outs[3] = {ux, uy, uz};
    const size_t G = (size_t)c->g.G;
    for (int k = 0; k < 3; ++k) {
      if (!outs[k]) continue;
      if (which == 2 && !c->shear) {
        set_error("no shear flow: call fcm_produce_shear_velocity_field first");
        return (int)FCM_ERR_STATE;
      }
      if (which == 2)
        FCM_TRY(grid_to_padded<double>(c, outs[k], c->d_ushear + k * G));
      else if (which == 1 && c->urand_prec == 1)
        FCM_TRY(grid_to_padded<float>(c, outs[k], c->g32.urand + k * G));
      else
        FCM_TRY(grid_to_padded<double>(c, outs[k], (which == 1 ? c->g64.urand : c->g64.r) + k * G));
    }
    return (int)FCM_OK;
  });
}

int fcm_apply_mobility(fcm_ctx* ctx, const double* F, double* V) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede fcm_apply_mobility");
    return FCM_ERR_STATE;
  }
  FCM_TRY(copy_in(c, c->d_tmp3, F, sizeof(double) * 3 * c->Nb));
  FCM_TRY(mobility_dev(c, c->p.precision, c->d_tmp3, c->d_V));
  return copy_out(c, V, c->d_V, sizeof(double) * 3 * c->Nb);
}

// Shear forcing (SHEARING_FORCES of the reference).
int fcm_produce_shear_velocity_field(fcm_ctx* ctx, double scale, double wavenumber) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    if (c->step_pending) {
      set_error("a step is in flight on this context: call fcm_step_wait first");
      return (int)FCM_ERR_STATE;
    }
    if (!std::isfinite(scale) || !std::isfinite(wavenumber)) {
      set_error("shear scale and wavenumber must be finite");
      return (int)FCM_ERR_INVALID;
    }
    // fx(j) of fcm_fluid_solver.cpp:727, evaluated on the host once per y index
    const double PI = 3.14159265358979323846264338327950288;
    const int ny = c->g.ny;
    std::vector<double> row(ny);
    for (int j = 0; j < ny; ++j)
      row[j] = scale * c->p.kT * std::sin(wavenumber * 2.0 * PI * double(j) / double(ny)) / c->p.blob_radius;
    if (!c->d_ushear) {
      FCM_TRY(dev_alloc(&c->d_ushear, 3 * (size_t)c->g.G));
      FCM_TRY(dev_alloc(&c->d_vshear, 3 * (size_t)(c->Nb > 0 ? c->Nb : 1)));
      FCM_CUDA(cudaMemsetAsync(c->d_vshear, 0, sizeof(double) * 3 * (size_t)(c->Nb > 0 ? c->Nb : 1), c->stream));
    }
    // the spectrum array holds the row until the forward transform overwrites it
    double* d_row = reinterpret_cast<double*>(c->g64.c);
    FCM_CUDA(cudaMemcpyAsync(d_row, row.data(), sizeof(double) * ny, cudaMemcpyHostToDevice, c->stream));
    FCM_TRY(launch_shear_forcing(*c, d_row, c->g64.r, c->stream));
    if (c->p.slip_channel) FCM_TRY(launch_slip_image<double>(*c, c->g64.r, c->stream));  // :735-760
    FCM_TRY(stokes_t<double>(c));  // :771-841, the steps of :636-701
    FCM_CUDA(cudaMemcpyAsync(c->d_ushear, c->g64.r, sizeof(double) * 3 * (size_t)c->g.G, cudaMemcpyDeviceToDevice,
                             c->stream));
    c->det_ready = true;
    c->shear = true;
    c->graph_stale = true;
    FCM_CUDA(cudaStreamSynchronize(c->stream));
    return (int)FCM_OK;
  });
}

int fcm_calculate_shear_blob_velocities(fcm_ctx* ctx, double* Vshear) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->shear) {
    set_error("no shear flow: call fcm_produce_shear_velocity_field first");
    return FCM_ERR_STATE;
  }
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede interpolation");
    return FCM_ERR_STATE;
  }
  FCM_TRY(shear_velocities_dev(c));
  return copy_out(c, Vshear, c->d_vshear, sizeof(double) * 3 * c->Nb);
}

int fcm_fluid_x_velocity_in_y(fcm_ctx* ctx, const double* F, double* profile) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    if (!profile) {
      set_error("fcm_fluid_x_velocity_in_y: null output");
      return (int)FCM_ERR_INVALID;
    }
    if (!c->gauss_ready) {
      set_error("set_up_gaussians must precede spreading");
      return (int)FCM_ERR_STATE;
    }
    FCM_TRY(copy_in(c, c->d_tmp3, F, sizeof(double) * 3 * c->Nb));
    FCM_TRY(spread_t<double>(c, c->g64.blobs, c->d_tmp3));
    FCM_TRY(stokes_t<double>(c));
    c->det_ready = true;
    // the profile (ny doubles) goes through the spectrum array, free after the solve
    double* d_prof = reinterpret_cast<double*>(c->g64.c);
    FCM_TRY(launch_x_profile(*c, c->g64.r, c->shear ? c->d_ushear : nullptr, d_prof, c->stream));
    return copy_out(c, profile, d_prof, sizeof(double) * c->g.ny);
  });
}

// Force dipoles on the FP64 deterministic grid (no reference counterpart).
int fcm_set_up_dipole_distribution(fcm_ctx* ctx, const double* F, const double* T, const double* S) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (c->p.slip_channel) {
    set_error("force dipoles have no slip-channel image system");
    return FCM_ERR_INVALID;
  }
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede spreading");
    return FCM_ERR_STATE;
  }
  const size_t Nb = (size_t)c->Nb;
  if (!c->d_dip) FCM_TRY(dev_alloc(&c->d_dip, 33 * (Nb > 0 ? Nb : 1)));
  double* dT = c->d_dip;
  double* dS = dT + 3 * Nb;
  double* dD = dS + 9 * Nb;
  if (F) {
    FCM_TRY(copy_in(c, c->d_tmp3, F, sizeof(double) * 3 * Nb));
  } else {
    FCM_CUDA(cudaMemsetAsync(c->d_tmp3, 0, sizeof(double) * 3 * Nb, c->stream));
  }
  c->det_ready = false;
  FCM_TRY(spread_t<double>(c, c->g64.blobs, c->d_tmp3));
  if (!T && !S) return FCM_OK;
  if (T) FCM_TRY(copy_in(c, dT, T, sizeof(double) * 3 * Nb));
  if (S) FCM_TRY(copy_in(c, dS, S, sizeof(double) * 9 * Nb));
  FCM_TRY(launch_blob_dipoles(T ? dT : nullptr, S ? dS : nullptr, c->Nb, dD, c->stream));
  return launch_spread_dipoles<double>(*c, c->g64.blobs, dD, c->g64.r, c->stream);
}

int fcm_calculate_deterministic_blob_rotations(fcm_ctx* ctx, double* Omega, double* E) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (c->p.slip_channel) {
    set_error("force dipoles have no slip-channel image system");
    return FCM_ERR_INVALID;
  }
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede interpolation");
    return FCM_ERR_STATE;
  }
  const size_t Nb = (size_t)c->Nb;
  if (!c->d_dip) FCM_TRY(dev_alloc(&c->d_dip, 33 * (Nb > 0 ? Nb : 1)));
  double* dOm = c->d_dip + 21 * Nb;
  double* dE = dOm + 3 * Nb;
  FCM_TRY(launch_interp_dipoles<double>(*c, c->g64.blobs, c->g64.r, dOm, dE, c->stream));
  FCM_TRY(copy_out(c, Omega, dOm, sizeof(double) * 3 * Nb));
  return copy_out(c, E, dE, sizeof(double) * 9 * Nb);
}

static int check_stage_precision(Ctx* c, int32_t precision) {
  if (precision != 0 && precision != 1) {
    set_error("precision must be 0 (FP64) or 1 (FP32)");
    return FCM_ERR_INVALID;
  }
  if (precision == 1 && c->p.precision != 1) {
    set_error("the FP32 grid needs a context created with precision 1");
    return FCM_ERR_INVALID;
  }
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede the grid stages");
    return FCM_ERR_STATE;
  }
  return FCM_OK;
}

int fcm_spread(fcm_ctx* ctx, int32_t precision, const double* F) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(check_stage_precision(c, precision));
  const double* dF = F;  // device input is read in place
  if (!is_device_ptr(F)) {
    FCM_TRY(copy_in(c, c->d_tmp3, F, sizeof(double) * 3 * c->Nb));
    dF = c->d_tmp3;
  }
  if (precision == 0) {
    c->det_ready = false;
    return spread_t<double>(c, c->g64.blobs, dF);
  }
  return spread_t<float>(c, c->g32.blobs, dF);
}

int fcm_stokes_solve(fcm_ctx* ctx, int32_t precision) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(check_stage_precision(c, precision));
  if (precision == 0) {
    FCM_TRY(stokes_t<double>(c));
    c->det_ready = true;
    return FCM_OK;
  }
  return stokes_t<float>(c);
}

int fcm_interp(fcm_ctx* ctx, int32_t precision, double* V) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(check_stage_precision(c, precision));
  double* dV = (V && is_device_ptr(V)) ? V : c->d_V;  // device output is written in place
  if (precision == 0)
    FCM_TRY(interp_t<double>(c, c->g64.blobs, c->g64.r, dV));
  else
    FCM_TRY(interp_t<float>(c, c->g32.blobs, c->g32.r, dV));
  if (dV == V) return FCM_OK;
  return copy_out(c, V, c->d_V, sizeof(double) * 3 * c->Nb);
}

int fcm_get_variants(fcm_ctx* ctx, int32_t* variants) {
  CTX_CHECK(ctx);
  if (!variants) {
    set_error("variants is NULL");
    return FCM_ERR_INVALID;
  }
  get_variants(ctx->c, variants);
  return FCM_OK;
}

int fcm_set_variants(fcm_ctx* ctx, const int32_t* variants) {
  CTX_CHECK(ctx);
  if (!variants) {
    set_error("variants is NULL");
    return FCM_ERR_INVALID;
  }
  if (ctx->c->in_batch) {
    set_error("kernel variants of a context owned by a batch are fixed");
    return FCM_ERR_STATE;
  }
  return set_variants(ctx->c, variants);
}

int fcm_autotune(fcm_ctx* ctx, int32_t reps, double* us, int32_t* variants) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (c->in_batch) {
    set_error("kernel variants of a context owned by a batch are fixed");
    return FCM_ERR_STATE;
  }
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede fcm_autotune");
    return FCM_ERR_STATE;
  }
  return guard([&]() -> int {
    const int R = reps > 0 ? reps : 5;
    double t[FCM_NUM_TUNE_TIMES];
    for (double& v : t) v = -1.0;
    FCM_TRY(ensure_grid<double>(c));
    FCM_TRY(tune_precision<double>(c, R, t));
    if (c->p.precision == 1) {
      FCM_TRY(ensure_grid<float>(c));
      FCM_TRY(tune_precision<float>(c, R, t + FCM_NUM_TUNE_TIMES / 2));
    }
    c->det_ready = false;
    c->graph_stale = true;
    if (us) std::memcpy(us, t, sizeof(t));
    if (variants) get_variants(c, variants);
    return FCM_OK;
  });
}

namespace {
int refuse_per_body(const Ctx* c, const char* what) {
  if (!c->per_body) return FCM_OK;
  set_error(std::string(what) + ": the context has per-body shapes (fcm_set_body_shapes); use "
                                "fcm_set_body_preconditioners / fcm_get_body_preconditioners");
  return FCM_ERR_STATE;
}
}  // namespace

int fcm_produce_reference_matrices(fcm_ctx* ctx) {
  CTX_CHECK(ctx);
  FCM_TRY(refuse_per_body(ctx->c, "fcm_produce_reference_matrices"));
  return guard([&] { return reference_matrices_dev(ctx->c); });
}

int fcm_get_reference_matrices(fcm_ctx* ctx, double* Minv, double* N, double* KTKinv) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(refuse_per_body(c, "fcm_get_reference_matrices"));
  const int n3 = 3 * c->nb;
  if (Minv) std::memcpy(Minv, c->h_Minv.data(), sizeof(double) * n3 * n3);
  if (N) std::memcpy(N, c->h_N.data(), sizeof(double) * 36);
  if (KTKinv) std::memcpy(KTKinv, c->h_KTKinv.data(), sizeof(double) * 36);
  return FCM_OK;
}

int fcm_set_reference_matrices(fcm_ctx* ctx, const double* Minv, const double* N) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(refuse_per_body(c, "fcm_set_reference_matrices"));
  const int n3 = 3 * c->nb;
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  if (Minv) {
    c->h_Minv.assign(Minv, Minv + (size_t)n3 * n3);
    FCM_CUDA(cudaMemcpyAsync(c->d_Minv, c->h_Minv.data(), sizeof(double) * n3 * n3, cudaMemcpyHostToDevice, c->stream));
  }
  if (N) {
    c->h_N.assign(N, N + 36);
    FCM_CUDA(cudaMemcpyAsync(c->d_N, c->h_N.data(), sizeof(double) * 36, cudaMemcpyHostToDevice, c->stream));
  }
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  c->have_ref = true;
  return FCM_OK;
}

// ------------------------------------------------------------------ per-body shapes
namespace {
// Drop every captured graph that holds the shape or preconditioner pointers.
void drop_graphs(Ctx* c) {
  for (int i = 0; i < 2; ++i)
    if (c->iter_graph[i]) {
      cudaGraphExecDestroy(c->iter_graph[i]);
      c->iter_graph[i] = nullptr;
    }
  if (c->mcmc_graph) {
    cudaGraphExecDestroy(c->mcmc_graph);
    c->mcmc_graph = nullptr;
  }
  c->graph_stale = true;
}
}  // namespace

int fcm_set_body_shapes(fcm_ctx* ctx, const double* shapes) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    if (!shapes) {
      set_error("fcm_set_body_shapes: shapes is NULL");
      return (int)FCM_ERR_INVALID;
    }
    if (c->in_batch) {
      set_error("fcm_set_body_shapes: not available to batch members");
      return (int)FCM_ERR_STATE;
    }
    if (c->step_pending) {
      set_error("fcm_set_body_shapes: a step is in flight on this context");
      return (int)FCM_ERR_STATE;
    }
    const int M = c->M, nb = c->nb, n3 = 3 * nb;
    std::vector<double> hs((size_t)n3 * M);
    FCM_CUDA(cudaStreamSynchronize(c->stream));
    FCM_CUDA(cudaMemcpy(hs.data(), shapes, sizeof(double) * hs.size(), cudaMemcpyDefault));
    for (double v : hs)
      if (!std::isfinite(v)) {
        set_error("fcm_set_body_shapes: non-finite coordinate");
        return (int)FCM_ERR_INVALID;
      }
    std::vector<double> Minv((size_t)M * n3 * n3), N(36 * (size_t)M), KTKinv(36 * (size_t)M);
    std::atomic<long long> bad{-1};
    const double a = c->p.blob_radius, eta = c->p.viscosity;
    parallel_ranges(M, [&](long long lo, long long hi) {
      for (long long n = lo; n < hi; ++n)
        if (!body_preconditioner(&hs[(size_t)n * n3], nb, a, eta, &Minv[(size_t)n * n3 * n3], &N[36 * (size_t)n],
                                 &KTKinv[36 * (size_t)n]))
          bad = n;
    });
    if (bad >= 0) {
      set_error("fcm_set_body_shapes: the preconditioner of body " + std::to_string(bad.load()) +
                " could not be formed (coincident blobs?)");
      return (int)FCM_ERR_INVALID;
    }
    double *d_ref = nullptr, *d_Minv = nullptr, *d_N = nullptr, *d_KTKinv = nullptr;
    auto release = [&] {
      cudaFree(d_ref);
      cudaFree(d_Minv);
      cudaFree(d_N);
      cudaFree(d_KTKinv);
    };
    if (dev_alloc(&d_ref, hs.size()) || dev_alloc(&d_Minv, Minv.size()) || dev_alloc(&d_N, N.size()) ||
        dev_alloc(&d_KTKinv, KTKinv.size())) {
      release();
      set_error("fcm_set_body_shapes: device allocation failed");
      return (int)FCM_ERR_NOMEM;
    }
    if (cudaMemcpy(d_ref, hs.data(), sizeof(double) * hs.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_Minv, Minv.data(), sizeof(double) * Minv.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_N, N.data(), sizeof(double) * N.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(d_KTKinv, KTKinv.data(), sizeof(double) * KTKinv.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
      release();
      set_error("fcm_set_body_shapes: copy to the device failed");
      return (int)FCM_ERR_CUDA;
    }
    drop_graphs(c);
    cudaFree(c->d_ref);
    cudaFree(c->d_Minv);
    cudaFree(c->d_N);
    cudaFree(c->d_KTKinv);
    c->d_ref = d_ref;
    c->d_Minv = d_Minv;
    c->d_N = d_N;
    c->d_KTKinv = d_KTKinv;
    c->per_body = true;
    c->ref_stride = n3;
    c->minv_stride = (long long)n3 * n3;
    c->n_stride = 36;
    // the Metropolis rotation scale: the largest |r| over every shape
    // (collection_of_rigid_bodies.cpp:110-114 over all bodies)
    c->body_radius = 0.0;
    for (size_t m = 0; m < hs.size(); m += 3)
      c->body_radius = std::max(c->body_radius, std::sqrt(hs[m] * hs[m] + hs[m + 1] * hs[m + 1] + hs[m + 2] * hs[m + 2]));
    c->have_ref = true;
    return (int)FCM_OK;
  });
}

int fcm_set_body_preconditioners(fcm_ctx* ctx, const double* Minv, const double* N) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->per_body) {
    set_error("fcm_set_body_preconditioners: call fcm_set_body_shapes first");
    return FCM_ERR_STATE;
  }
  const size_t n3 = 3 * (size_t)c->nb;
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  if (Minv) FCM_CUDA(cudaMemcpy(c->d_Minv, Minv, sizeof(double) * n3 * n3 * c->M, cudaMemcpyDefault));
  if (N) FCM_CUDA(cudaMemcpy(c->d_N, N, sizeof(double) * 36 * c->M, cudaMemcpyDefault));
  return FCM_OK;
}

int fcm_get_body_preconditioners(fcm_ctx* ctx, double* Minv, double* N, double* KTKinv) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->per_body) {
    set_error("fcm_get_body_preconditioners: call fcm_set_body_shapes first");
    return FCM_ERR_STATE;
  }
  const size_t n3 = 3 * (size_t)c->nb;
  FCM_CUDA(cudaStreamSynchronize(c->stream));
  if (Minv) FCM_CUDA(cudaMemcpy(Minv, c->d_Minv, sizeof(double) * n3 * n3 * c->M, cudaMemcpyDefault));
  if (N) FCM_CUDA(cudaMemcpy(N, c->d_N, sizeof(double) * 36 * c->M, cudaMemcpyDefault));
  if (KTKinv) FCM_CUDA(cudaMemcpy(KTKinv, c->d_KTKinv, sizeof(double) * 36 * c->M, cudaMemcpyDefault));
  return FCM_OK;
}

// ------------------------------------------------------------------ gmres_solver
int fcm_assemble_RHS(fcm_ctx* ctx) {
  CTX_CHECK(ctx);
  return assemble_rhs_dev(ctx->c);
}

int fcm_get_RHS(fcm_ctx* ctx, double* rhs) {
  CTX_CHECK(ctx);
  return copy_out(ctx->c, rhs, ctx->c->d_rhs, sizeof(double) * ctx->c->nsys);
}

int fcm_set_RHS(fcm_ctx* ctx, const double* rhs) {
  CTX_CHECK(ctx);
  return copy_in(ctx->c, ctx->c->d_rhs, rhs, sizeof(double) * ctx->c->nsys);
}

int fcm_multiply_by_Pinv(fcm_ctx* ctx, const double* in, double* out) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  FCM_TRY(copy_in(c, c->d_sys_b, in, sizeof(double) * c->nsys));
  FCM_TRY(launch_pinv(*c, c->d_qm, c->d_sys_b, c->d_sys_a, c->stream));
  return copy_out(c, out, c->d_sys_a, sizeof(double) * c->nsys);
}

int fcm_multiply_by_saddle_point_matrix(fcm_ctx* ctx, const double* in, double* out) {
  CTX_CHECK(ctx);
  Ctx* c = ctx->c;
  if (!c->gauss_ready) {
    set_error("set_up_gaussians must precede the saddle-point product");
    return FCM_ERR_STATE;
  }
  FCM_TRY(copy_in(c, c->d_sys_b, in, sizeof(double) * c->nsys));
  // as the reference's product (gmres_solver.cpp:72-83) leaves M lambda in fcm.V
  // (calculate_deterministic_blob_velocities), the context's V takes it here too
  const double* lam = c->d_sys_b;
  FCM_TRY(mobility_dev(c, 0, lam, c->d_sys_a));
  FCM_CUDA(cudaMemcpyAsync(c->d_V, c->d_sys_a, sizeof(double) * 3 * (size_t)c->Nb, cudaMemcpyDeviceToDevice,
                           c->stream));
  FCM_TRY(launch_multiply_K(*c, c->d_qm, lam + 3 * (size_t)c->Nb, c->d_sys_a, 1.0, c->stream));
  FCM_TRY(launch_multiply_KT(*c, c->d_qm, lam, c->d_sys_a + 3 * (size_t)c->Nb, -1.0, nullptr, 0.0, c->stream));
  return copy_out(c, out, c->d_sys_a, sizeof(double) * c->nsys);
}

int fcm_invert_saddle_point_system(fcm_ctx* ctx, double* soln, int32_t* iters, double* rel_residual) {
  CTX_CHECK(ctx);
  return guard([&] {
    Ctx* c = ctx->c;
    if (!c->gauss_ready) {
      set_error("set_up_gaussians must precede the saddle-point solve");
      return (int)FCM_ERR_STATE;
    }
    int it = 0, sw = 0;
    double rel = 0.0;
    double* x = c->d_soln;
    int st = solve_dev(c, c->d_rhs, x, &it, &rel, &sw);
    if (st == FCM_OK || st == FCM_ERR_NOT_CONVERGED) {
      const int s2 = copy_out(c, soln, x, sizeof(double) * c->nsys);
      if (s2 != FCM_OK) st = s2;
    }
    if (iters) *iters = it;
    if (rel_residual) *rel_residual = rel;
    return st;
  });
}

// ------------------------------------------------------------------ time step
int fcm_step(fcm_ctx* ctx, uint64_t seed, uint64_t step_index, fcm_step_info* info) {
  CTX_CHECK(ctx);
  if (ctx->c->step_pending) {
    set_error("a step issued by fcm_step_async is in flight: call fcm_step_wait first");
    return FCM_ERR_STATE;
  }
  return guard([&] { return step_host(ctx->c, seed, step_index, info); });
}

int fcm_calculate_potential(fcm_ctx* ctx, double* U) {
  CTX_CHECK(ctx);
  if (!U) {
    set_error("fcm_calculate_potential: null output");
    return FCM_ERR_INVALID;
  }
  return guard([&] {
    Ctx* c = ctx->c;
    FCM_TRY(mcmc_alloc(c));
    FCM_TRY(potential_sum_dev(c));
    double sum = 0.0;
    FCM_CUDA(cudaMemcpyAsync(&sum, c->d_usum, sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    FCM_CUDA(cudaStreamSynchronize(c->stream));
    *U = 0.5 * sum;
    return (int)FCM_OK;
  });
}

int fcm_mcmc_state_init(const fcm_ctx* ctx, fcm_mcmc_state* state) {
  CTX_CHECK(ctx);
  if (!state) return FCM_ERR_INVALID;
  std::memset(state, 0, sizeof(*state));
  state->scale = 0.1 * ctx->c->p.blob_radius;  // main.cpp:120
  state->acceptance_ratio = 0.5;              // main.cpp:121
  return FCM_OK;
}

int fcm_mcmc_run(fcm_ctx* ctx, uint64_t seed, int64_t n_steps, fcm_mcmc_state* state) {
  CTX_CHECK(ctx);
  if (!state || n_steps < 0) {
    set_error("fcm_mcmc_run: a state and n_steps >= 0 are required");
    return FCM_ERR_INVALID;
  }
  return guard([&] { return mcmc_run_dev(ctx->c, seed, n_steps, state); });
}

int fcm_batch_create(int32_t n, const fcm_params* params, const double* const* blob_ref_pos, fcm_batch** out) {
  return guard([&] {
    if (!out) return (int)FCM_ERR_INVALID;
    *out = nullptr;
    Batch* B = nullptr;
    const int st = create_batch(n, params, blob_ref_pos, &B);
    if (st != FCM_OK) return st;
    fcm_batch* h = new fcm_batch{B, {}};
    h->members.resize(n);
    for (int i = 0; i < n; ++i) h->members[i].c = B->m[i];
    *out = h;
    return (int)FCM_OK;
  });
}

int fcm_batch_destroy(fcm_batch* b) {
  if (!b) return FCM_OK;
  if (b->b) {
    cudaStreamSynchronize(b->b->stream);
    destroy_batch(b->b);
  }
  delete b;
  return FCM_OK;
}

fcm_ctx* fcm_batch_member(fcm_batch* b, int32_t i) {
  if (!b || i < 0 || i >= (int32_t)b->members.size()) {
    set_error("fcm_batch_member: index out of range");
    return nullptr;
  }
  return &b->members[i];
}

int fcm_batch_set_stream(fcm_batch* b, void* stream) {
  if (!b) {
    set_error("null batch");
    return FCM_ERR_INVALID;
  }
  b->b->stream = (cudaStream_t)stream;
  return FCM_OK;
}

int fcm_batch_last_rounds(const fcm_batch* b, int32_t* rounds) {
  if (!b || !rounds) {
    set_error("fcm_batch_last_rounds: null batch or output");
    return FCM_ERR_INVALID;
  }
  const bool graph = b->b->state == 1;
  rounds[0] = graph ? b->b->h_loop[1] : 0;
  rounds[1] = graph ? b->b->h_loop[2] : 0;
  return FCM_OK;
}

int fcm_batch_step(fcm_batch* b, const uint64_t* seeds, uint64_t step_index, fcm_step_info* infos) {
  if (!b || !seeds) {
    set_error("fcm_batch_step: null batch or seeds");
    return FCM_ERR_INVALID;
  }
  return guard([&] { return batch_step(b->b, seeds, step_index, infos); });
}

int fcm_step_async(fcm_ctx* ctx, uint64_t seed, uint64_t step_index) {
  CTX_CHECK(ctx);
  return guard([&] { return step_issue(ctx->c, seed, step_index); });
}

int fcm_step_wait(fcm_ctx* ctx, fcm_step_info* info) {
  CTX_CHECK(ctx);
  return guard([&] { return step_wait(ctx->c, info); });
}

int fcm_step_many(fcm_ctx* const* ctxs, int32_t n, const uint64_t* seeds, uint64_t step_index,
                  fcm_step_info* infos) {
  if (n < 0 || (n > 0 && (!ctxs || !seeds))) {
    set_error("fcm_step_many: n >= 0 contexts and seeds required");
    return FCM_ERR_INVALID;
  }
  for (int i = 0; i < n; ++i) CTX_CHECK(ctxs[i]);
  return guard([&] {
    int first = FCM_OK;
    std::string err;
    int issued = 0;
    for (; issued < n; ++issued) {
      const int st = step_issue(ctxs[issued]->c, seeds[issued], step_index);
      if (st != FCM_OK) {
        first = st;
        err = g_err;
        break;
      }
    }
    for (int i = 0; i < issued; ++i) {
      fcm_step_info inf;
      const int st = step_wait(ctxs[i]->c, &inf);
      if (infos) infos[i] = inf;
      if (st != FCM_OK && first == FCM_OK) {
        first = st;
        err = g_err;
      }
    }
    if (first != FCM_OK) set_error(err);
    return first;
  });
}

}  // extern "C"
