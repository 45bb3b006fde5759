// fcm_blas.cu -- FP64 vector operations of the GMRES solver
// (gmres_solver.cpp:148-306): deterministic dot products and norms, fused
// modified-Gram-Schmidt steps, scaling and the final Krylov combination.
//
// Reductions are single-launch and deterministic: a fixed grid writes one
// partial per block, and the last block to finish (ticket counter, no waiting)
// sums the partials in index order.
#include <algorithm>

#include "fcm_internal.cuh"

namespace fcm {

namespace {

constexpr int RT = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int i = 0; i < RT / 32; ++i) s += sh[i];
  return s;
}

// Finish a reduction: the last block sums `partials` in order into *out.
// mode 0: *out = total, 1: *out += total, 2: *out = sqrt(total).
// nblocks: blocks taking part (gridDim.x for a single reduction).
__device__ __forceinline__ void finish(double my_partial, double* partials, unsigned int* counter, double* out,
                                       int mode, double* sh, unsigned nblocks) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = my_partial;
    __threadfence();
    const unsigned int ticket = atomicAdd(counter, 1u);
    last = (ticket == nblocks - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  // fixed assignment of partials to threads, then a fixed-order block sum
  for (int i = threadIdx.x; i < (int)nblocks; i += RT) v += ((volatile double*)partials)[i];
  const double total = block_sum(v, sh);
  if (threadIdx.x == 0) {
    if (mode == 0) *out = total;
    else if (mode == 1) *out += total;
    else *out = sqrt(total);
    *counter = 0u;
  }
}

// *out (op)= sum a[i]*b[i]  (b == nullptr: sum a[i])
__global__ void __launch_bounds__(RT) k_dot(const double* __restrict__ a, const double* __restrict__ b, long long n,
                                            double* partials, unsigned int* counter, double* out, int mode) {
  __shared__ double sh[RT / 32];
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT)
    s += b ? a[i] * b[i] : a[i];
  const double bs = block_sum(s, sh);
  finish(bs, partials, counter, out, mode, sh, gridDim.x);
}

// One modified-Gram-Schmidt step (gmres_solver.cpp:198-206): w -= h_prev*q_prev
// (if q_prev), then *hout = dot(w, q_i) (q_i == nullptr: *hout = ||w||).
__global__ void __launch_bounds__(RT) k_mgs(double* __restrict__ w, const double* __restrict__ q_prev,
                                            const double* __restrict__ h_prev, const double* __restrict__ q_i,
                                            long long n, double* partials, unsigned int* counter, double* hout) {
  __shared__ double sh[RT / 32];
  const double h = q_prev ? *h_prev : 0.0;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)gridDim.x * RT) {
    double v = w[i];
    if (q_prev) {
      v -= h * q_prev[i];
      w[i] = v;
    }
    s += q_i ? v * q_i[i] : v * v;
  }
  const double bs = block_sum(s, sh);
  finish(bs, partials, counter, hout, q_i ? 0 : 2, sh, gridDim.x);
}

__global__ void k_scale(double* __restrict__ v, const double* __restrict__ num, int invert, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = *num;
  if (invert) {
    if (s != 0.0) v[i] = v[i] / s;
  } else {
    v[i] = v[i] * s;
  }
}

__global__ void k_copy_scaled(double* __restrict__ dst, const double* __restrict__ src, const double* __restrict__ num,
                              int invert, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double s = *num;
  dst[i] = invert ? src[i] / s : src[i] * s;
}

__global__ void k_axpby(double* __restrict__ y, const double* __restrict__ x, double a, double b, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  y[i] = a * x[i] + b * y[i];
}

// soln = sum_{i<k} y_i Q[:, i]  (gmres_solver.cpp:278-284, in column order)
__global__ void k_combine(double* __restrict__ out, const double* __restrict__ Q, const double* __restrict__ y, int k,
                          long long n) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  double s = 0.0;
  for (int i = 0; i < k; ++i) s += y[i] * Q[(size_t)i * n + t];
  out[t] = s;
}

__global__ void k_f64_to_f32(float* __restrict__ d, const double* __restrict__ s, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) d[i] = (float)s[i];
}

inline unsigned nblk(long long n, int t) { return (unsigned)((n + t - 1) / t); }

}  // namespace

int blas_dot(const Ctx& c, const double* a, const double* b, long long n, double* d_out, cudaStream_t s) {
  k_dot<<<c.red_blocks, RT, 0, s>>>(a, b, n, c.d_partials, c.d_counter, d_out, 0);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// sum of a[] accumulated into *d_out (b == nullptr, mode 1)
int blas_sum_accumulate(const Ctx& c, const double* a, long long n, double* d_out, cudaStream_t s) {
  k_dot<<<c.red_blocks, RT, 0, s>>>(a, nullptr, n, c.d_partials, c.d_counter, d_out, 1);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_norm_sq_partial(const Ctx& c, const double* a, long long n, double* d_out, cudaStream_t s) {
  k_mgs<<<c.red_blocks, RT, 0, s>>>(const_cast<double*>(a), nullptr, nullptr, nullptr, n, c.d_partials, c.d_counter,
                                    d_out);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_mgs_step(const Ctx& c, double* w, const double* q_prev, const double* h_prev, const double* q_i, long long n,
                  double* d_hout, cudaStream_t s) {
  k_mgs<<<c.red_blocks, RT, 0, s>>>(w, q_prev, h_prev, q_i, n, c.d_partials, c.d_counter, d_hout);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_scale(double* v, const double* d_num, int invert, long long n, cudaStream_t s) {
  k_scale<<<nblk(n, 256), 256, 0, s>>>(v, d_num, invert, n);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_copy_scaled(double* dst, const double* src, const double* d_num, int invert, long long n, cudaStream_t s) {
  k_copy_scaled<<<nblk(n, 256), 256, 0, s>>>(dst, src, d_num, invert, n);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t s) {
  k_axpby<<<nblk(n, 256), 256, 0, s>>>(y, x, a, b, n);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_combine(double* out, const double* Q, const double* d_y, int k, long long n, cudaStream_t s) {
  k_combine<<<nblk(n, 256), 256, 0, s>>>(out, Q, d_y, k, n);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int blas_f64_to_f32(float* dst, const double* src, long long n, cudaStream_t s) {
  k_f64_to_f32<<<nblk(n, 256), 256, 0, s>>>(dst, src, n);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

}  // namespace fcm

// ============================================================ device-side GMRES
// The Arnoldi/Givens process of gmres_solver.cpp:193-306 kept on the device, so
// one iteration is a fixed sequence of kernels (captured once in a CUDA graph):
//   z_in = Q[k]; z = P^-1 z_in; w = A z                       (caller)
//   h  = Q[0..k]^T w, w -= Q h   twice (classical Gram-Schmidt with one
//        re-orthogonalisation, the same projections as the reference's modified
//        Gram-Schmidt in exact arithmetic)
//   Q[k+1] = w / |w|; Givens rotations, residual, convergence   (one thread)
// k, the rotations, beta and the Hessenberg matrix live in device memory.
namespace fcm {
namespace {

constexpr int MDT = 256;

__global__ void k_gm_fetch(const GmState* __restrict__ st, const double* __restrict__ Q, long long n,
                           double* __restrict__ dst) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n || st->done) return;
  dst[t] = Q[(size_t)st->k * n + t];
}

// h[i] = Q[:, i] . w for i <= k; grid (nblk, maxcols); deterministic two-level sum
// (one partial per block and column, the last block of a column adds them in order).
__global__ void __launch_bounds__(MDT) k_multidot(const GmState* __restrict__ st, const double* __restrict__ Q,
                                                  const double* __restrict__ w, long long n,
                                                  double* __restrict__ partials, unsigned int* __restrict__ counters,
                                                  double* __restrict__ h) {
  __shared__ double sh[MDT / 32];
  __shared__ bool last;
  const int col = blockIdx.y;
  if (st->done || col > st->k) return;
  const double* q = Q + (size_t)col * n;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)MDT + threadIdx.x; i < n; i += (long long)gridDim.x * MDT)
    s += q[i] * w[i];
  for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int i = 0; i < MDT / 32; ++i) b += sh[i];
    partials[(size_t)col * gridDim.x + blockIdx.x] = b;
    __threadfence();
    last = (atomicAdd(counters + col, 1u) == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (threadIdx.x == 0) {
    double tot = 0.0;
    const volatile double* p = partials + (size_t)col * gridDim.x;
    for (unsigned int b = 0; b < gridDim.x; ++b) tot += p[b];
    h[col] = tot;
    counters[col] = 0u;
  }
}

// w -= sum_{i<=k} h[i] Q[:, i]
__global__ void k_gs_update(const GmState* __restrict__ st, const double* __restrict__ Q,
                            const double* __restrict__ h, long long n, double* __restrict__ w) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n || st->done) return;
  const int k = st->k;
  double v = w[t];
  for (int i = 0; i <= k; ++i) v -= h[i] * Q[(size_t)i * n + t];
  w[t] = v;
}

// Q[k+1] = w / |w| (|w| = 0: a happy breakdown, the column is left as w)
__global__ void k_gm_normalize(const GmState* __restrict__ st, const double* __restrict__ w,
                               const double* __restrict__ hnorm, long long n, double* __restrict__ Q, int hn) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n || st->done) return;
  if (!FCM_INB(st->k + 1, hn, BS_KRYLOV)) return;
  const double s = *hnorm;
  Q[(size_t)(st->k + 1) * n + t] = (s != 0.0) ? w[t] / s : w[t];
}

// gmres_solver.cpp:248-300 for column k+1 (one thread).
__device__ __forceinline__ void givens_step(GmState* st, double* __restrict__ H, int hn, double* __restrict__ beta,
                                            double* __restrict__ CS, double* __restrict__ SN,
                                            const double* __restrict__ hA, const double* __restrict__ hB,
                                            const double* __restrict__ hnorm) {
  if (st->done) return;
  const int iter = st->k + 1;
  if (!FCM_INB(iter, hn, BS_KRYLOV)) {  // no column left for Q[k+1]: end the solve
    st->done = 1;
    st->status = FCM_ERR_NOT_CONVERGED;
    return;
  }
  double* col = H + (size_t)(iter - 1) * hn;
  for (int i = 0; i < iter; ++i) col[i] = hA[i] + hB[i];
  col[iter] = *hnorm;
  for (int i = 1; i < iter; i++) {
    const double temp = CS[i - 1] * col[i - 1] + SN[i - 1] * col[i];
    col[i] = CS[i - 1] * col[i] - SN[i - 1] * col[i - 1];
    col[i - 1] = temp;
  }
  const double a = col[iter - 1], b = col[iter];
  if (b == 0.0) {
    CS[iter - 1] = 1.0;
    SN[iter - 1] = 0.0;
  } else if (fabs(b) > fabs(a)) {
    const double temp = a / b;
    SN[iter - 1] = (2.0 * double(b > 0) - 1.0) / sqrt(1.0 + temp * temp);
    CS[iter - 1] = temp * SN[iter - 1];
  } else {
    const double temp = b / a;
    CS[iter - 1] = (2.0 * double(a > 0) - 1.0) / sqrt(1.0 + temp * temp);
    SN[iter - 1] = temp * CS[iter - 1];
  }
  col[iter - 1] = CS[iter - 1] * a + SN[iter - 1] * b;
  col[iter] = 0.0;
  beta[iter] = -SN[iter - 1] * beta[iter - 1];
  beta[iter - 1] = CS[iter - 1] * beta[iter - 1];
  const double rel = fabs(beta[iter]) / st->normb;
  st->k = iter;
  st->rel = rel;
  if (!isfinite(rel)) {
    st->done = 1;
    st->status = FCM_ERR_NONFINITE;
  } else if (rel < st->tol || iter >= st->maxit) {
    st->done = 1;
    st->status = rel < st->tol ? FCM_OK : FCM_ERR_NOT_CONVERGED;
  }
}

__global__ void k_gm_givens(GmState* st, double* __restrict__ H, int hn, double* __restrict__ beta,
                            double* __restrict__ CS, double* __restrict__ SN, const double* __restrict__ hA,
                            const double* __restrict__ hB, const double* __restrict__ hnorm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  givens_step(st, H, hn, beta, CS, SN, hA, hB, hnorm);
}

// beta[0] = |b|, k = 0 (one thread); |b| == 0 or non-finite ends the solve.
__global__ void k_gm_init(GmState* st, const double* __restrict__ normb, double* __restrict__ beta, double tol,
                          const double* __restrict__ d_tol, int maxit) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double nb = *normb;
  if (d_tol) tol = *d_tol;
  st->k = 0;
  st->tol = tol;
  st->maxit = maxit;
  st->normb = nb;
  st->rel = 0.0;
  beta[0] = nb;
  if (nb > 0.0 && isfinite(nb)) {
    st->done = 0;
    st->status = FCM_OK;
  } else {
    st->done = 1;
    st->status = (nb == 0.0) ? FCM_OK : FCM_ERR_NONFINITE;
  }
}

// y = R^-1 beta (gmres_solver.cpp:302-318), one thread; k = 0 gives y = 0.
__device__ __forceinline__ void backsub_step(const GmState* __restrict__ st, const double* __restrict__ H, int hn,
                                             const double* __restrict__ beta, double* __restrict__ y) {
  const int iter = st->k;
  if (iter == 0) return;
  auto Hm = [&](int i, int j) { return H[(size_t)j * hn + i]; };
  y[iter - 1] = beta[iter - 1] / Hm(iter - 1, iter - 1);
  for (int i = iter - 2; i >= 0; i--) {
    double v = beta[i];
    for (int j = iter - 1; j > i; j--) v -= Hm(i, j) * y[j];
    y[i] = v / Hm(i, i);
  }
}

__global__ void k_gm_backsub(const GmState* __restrict__ st, const double* __restrict__ H, int hn,
                             const double* __restrict__ beta, double* __restrict__ y) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  backsub_step(st, H, hn, beta, y);
}

// soln = sum_{i<k} y_i Q[:, i] (gmres_solver.cpp:320-326), k from the state.
__global__ void k_gm_combine(const GmState* __restrict__ st, const double* __restrict__ Q,
                             const double* __restrict__ y, long long n, double* __restrict__ out) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  const int k = st->k;
  double s = 0.0;
  for (int i = 0; i < k; ++i) s += y[i] * Q[(size_t)i * n + t];
  out[t] = s;
}

}  // namespace

int gm_fetch(const Ctx& c, double* dst, cudaStream_t s) {
  const long long n = c.nsys;
  k_gm_fetch<<<nblk(n, 256), 256, 0, s>>>(c.gm, c.d_Qm, n, dst);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int gm_orthogonalize(const Ctx& c, double* w, cudaStream_t s) {
  const long long n = c.nsys;
  const dim3 grid(c.md_blocks, c.maxit_alloc + 1);
  double* hab[2] = {c.d_hA, c.d_hB};
  for (int pass = 0; pass < 2; ++pass) {
    k_multidot<<<grid, MDT, 0, s>>>(c.gm, c.d_Qm, w, n, c.d_mdpart, c.d_mdcount, hab[pass]);
    FCM_LAUNCH_CHECK();
    k_gs_update<<<nblk(n, 256), 256, 0, s>>>(c.gm, c.d_Qm, hab[pass], n, w);
    FCM_LAUNCH_CHECK();
  }
  FCM_TRY(blas_norm_sq_partial(c, w, n, c.d_hnorm, s));
  k_gm_normalize<<<nblk(n, 256), 256, 0, s>>>(c.gm, w, c.d_hnorm, n, c.d_Qm, c.maxit_alloc + 1);
  FCM_LAUNCH_CHECK();
  k_gm_givens<<<1, 32, 0, s>>>(c.gm, c.d_Hd, c.maxit_alloc + 1, c.d_beta, c.d_CS, c.d_SN, c.d_hA, c.d_hB,
                               c.d_hnorm);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int gm_init(const Ctx& c, const double* b, double tol, int maxit, cudaStream_t s, const double* d_tol) {
  const long long n = c.nsys;
  FCM_TRY(blas_norm_sq_partial(c, b, n, c.d_hnorm, s));
  k_gm_init<<<1, 32, 0, s>>>(c.gm, c.d_hnorm, c.d_beta, tol, d_tol, maxit);
  FCM_LAUNCH_CHECK();
  FCM_TRY(blas_copy_scaled(c.d_Qm, b, c.d_hnorm, 1, n, s));
  return FCM_OK;
}

int gm_finish(const Ctx& c, double* soln_pre, cudaStream_t s) {
  const long long n = c.nsys;
  k_gm_backsub<<<1, 32, 0, s>>>(c.gm, c.d_Hd, c.maxit_alloc + 1, c.d_beta, c.d_y);
  FCM_LAUNCH_CHECK();
  k_gm_combine<<<nblk(n, 256), 256, 0, s>>>(c.gm, c.d_Qm, c.d_y, n, soln_pre);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

}  // namespace fcm

// ============================================================ batched GMRES
// The same steps for every member of a batch in one launch: blockIdx.y (or .z
// for the multidot) selects the member, blockIdx.x keeps its single-member
// meaning, and each member's reductions use its own block count and ticket
// counter (the sums of its single solve).  Masks skip members whose solve is
// done (BM_GM) or whose refinement has finished (BM_REF).
namespace fcm {
namespace {

__global__ void __launch_bounds__(RT) k_b_norm(const BMember* __restrict__ mem, int vec, int out, int mask) {
  __shared__ double sh[RT / 32];
  const BMember& m = mem[blockIdx.y];
  if ((int)blockIdx.x >= m.red_blocks || bskip(m, mask)) return;
  const double* w = bvec(m, vec);
  const long long n = m.nsys;
  double s = 0.0;
  for (long long i = blockIdx.x * (long long)RT + threadIdx.x; i < n; i += (long long)m.red_blocks * RT)
    s += w[i] * w[i];
  const double bs = block_sum(s, sh);
  finish(bs, m.partials, m.counter, bout(m, out), 2, sh, (unsigned)m.red_blocks);
}

// y = a x + b y
__global__ void k_b_axpby(const BMember* __restrict__ mem, int yv, int xv, double a, double b, int mask) {
  const BMember& m = mem[blockIdx.y];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m.nsys || bskip(m, mask)) return;
  double* y = bvec(m, yv);
  const double* x = bvec(m, xv);
  y[i] = a * x[i] + b * y[i];
}

// Start of a solve (k_gm_init per member): tolerance from rs[2] when use_rs;
// members the mask excludes get an empty, finished solve.
__global__ void k_b_gm_init(const BMember* __restrict__ mem, double tol, int use_rs, int mask) {
  if (threadIdx.x != 0) return;
  const BMember& m = mem[blockIdx.x];
  GmState* st = m.gm;
  st->k = 0;
  st->maxit = m.hn - 1;
  st->rel = 0.0;
  if (mask == BM_REF && !m.sd->ref_active) {
    st->tol = tol;
    st->normb = 0.0;
    st->done = 1;
    st->status = FCM_OK;
    return;
  }
  const double nb = *m.hnorm;
  st->tol = use_rs ? m.rs[2] : tol;
  st->normb = nb;
  m.beta[0] = nb;
  if (nb > 0.0 && isfinite(nb)) {
    st->done = 0;
    st->status = FCM_OK;
  } else {
    st->done = 1;
    st->status = (nb == 0.0) ? FCM_OK : FCM_ERR_NONFINITE;
  }
}

// Q[:, 0] = b / ||b||
__global__ void k_b_first_column(const BMember* __restrict__ mem, int vec) {
  const BMember& m = mem[blockIdx.y];
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= m.nsys || m.gm->done) return;
  m.Qm[i] = bvec(m, vec)[i] / *m.hnorm;
}

__global__ void k_b_fetch(const BMember* __restrict__ mem) {
  const BMember& m = mem[blockIdx.y];
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= m.nsys || m.gm->done) return;
  m.sys_b[t] = m.Qm[(size_t)m.gm->k * m.nsys + t];
}

// Columns col = blockIdx.y, blockIdx.y + gridDim.y, ... <= k of each member:
// a fixed grid whatever k is, so few blocks exit idle.
__global__ void __launch_bounds__(MDT) k_b_multidot(const BMember* __restrict__ mem, int pass) {
  __shared__ double sh[MDT / 32];
  __shared__ bool last;
  const BMember& m = mem[blockIdx.z];
  const GmState* st = m.gm;
  const unsigned nbk = (unsigned)m.md_blocks;
  if (blockIdx.x >= nbk || st->done) return;
  const int k = st->k;
  const long long n = m.nsys;
  const double* w = m.sys_b;
  double* h = pass == 0 ? m.hA : m.hB;
  for (int col = blockIdx.y; col <= k; col += gridDim.y) {
    const double* q = m.Qm + (size_t)col * n;
    double s = 0.0;
    for (long long i = blockIdx.x * (long long)MDT + threadIdx.x; i < n; i += (long long)nbk * MDT)
      s += q[i] * w[i];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double b = 0.0;
      for (int i = 0; i < MDT / 32; ++i) b += sh[i];
      m.mdpart[(size_t)col * nbk + blockIdx.x] = b;
      __threadfence();
      last = (atomicAdd(m.mdcount + col, 1u) == nbk - 1);
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
      __threadfence();
      double tot = 0.0;
      const volatile double* p = m.mdpart + (size_t)col * nbk;
      for (unsigned int b = 0; b < nbk; ++b) tot += p[b];
      h[col] = tot;
      m.mdcount[col] = 0u;
    }
    __syncthreads();
  }
}

__global__ void k_b_gs_update(const BMember* __restrict__ mem, int pass) {
  const BMember& m = mem[blockIdx.y];
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= m.nsys || m.gm->done) return;
  const int k = m.gm->k;
  const double* h = pass == 0 ? m.hA : m.hB;
  double v = m.sys_b[t];
  for (int i = 0; i <= k; ++i) v -= h[i] * m.Qm[(size_t)i * m.nsys + t];
  m.sys_b[t] = v;
}

__global__ void k_b_normalize(const BMember* __restrict__ mem) {
  const BMember& m = mem[blockIdx.y];
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= m.nsys || m.gm->done) return;
  if (!FCM_INB(m.gm->k + 1, m.hn, BS_KRYLOV)) return;
  const double s = *m.hnorm;
  m.Qm[(size_t)(m.gm->k + 1) * m.nsys + t] = (s != 0.0) ? m.sys_b[t] / s : m.sys_b[t];
}

__global__ void k_b_givens(const BMember* __restrict__ mem) {
  if (threadIdx.x != 0) return;
  const BMember& m = mem[blockIdx.x];
  givens_step(m.gm, m.Hd, m.hn, m.beta, m.CS, m.SN, m.hA, m.hB, m.hnorm);
}

__global__ void k_b_backsub(const BMember* __restrict__ mem) {
  if (threadIdx.x != 0) return;
  const BMember& m = mem[blockIdx.x];
  backsub_step(m.gm, m.Hd, m.hn, m.beta, m.y);
}

// sys_b = sum_{i<k} y_i Q[:, i]
__global__ void k_b_combine(const BMember* __restrict__ mem) {
  const BMember& m = mem[blockIdx.y];
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= m.nsys) return;
  const int k = m.gm->k;
  double s = 0.0;
  for (int i = 0; i < k; ++i) s += m.y[i] * m.Qm[(size_t)i * m.nsys + t];
  m.sys_b[t] = s;
}

}  // namespace

int b_norm(const BatchGeom& b, int vec, int out, int mask, cudaStream_t s) {
  k_b_norm<<<dim3(b.red_blocks, b.n), RT, 0, s>>>(b.mem, vec, out, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int b_axpby(const BatchGeom& b, int y, int x, double a, double bb, int mask, cudaStream_t s) {
  k_b_axpby<<<dim3(b.max_sys_blocks, b.n), 256, 0, s>>>(b.mem, y, x, a, bb, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int b_gm_init(const BatchGeom& b, int vec, double tol, int use_rs_tol, int mask, cudaStream_t s) {
  FCM_TRY(b_norm(b, vec, BO_HNORM, mask, s));
  k_b_gm_init<<<b.n, 32, 0, s>>>(b.mem, tol, use_rs_tol, mask);
  FCM_LAUNCH_CHECK();
  k_b_first_column<<<dim3(b.max_sys_blocks, b.n), 256, 0, s>>>(b.mem, vec);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int b_gm_fetch(const BatchGeom& b, cudaStream_t s) {
  k_b_fetch<<<dim3(b.max_sys_blocks, b.n), 256, 0, s>>>(b.mem);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int b_gm_orthogonalize(const BatchGeom& b, cudaStream_t s) {
  for (int pass = 0; pass < 2; ++pass) {
    k_b_multidot<<<dim3(b.md_blocks, std::min(b.max_hn, 8), b.n), MDT, 0, s>>>(b.mem, pass);
    FCM_LAUNCH_CHECK();
    k_b_gs_update<<<dim3(b.max_sys_blocks, b.n), 256, 0, s>>>(b.mem, pass);
    FCM_LAUNCH_CHECK();
  }
  FCM_TRY(b_norm(b, BV_SYS_B, BO_HNORM, BM_GM, s));
  k_b_normalize<<<dim3(b.max_sys_blocks, b.n), 256, 0, s>>>(b.mem);
  FCM_LAUNCH_CHECK();
  k_b_givens<<<b.n, 32, 0, s>>>(b.mem);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int b_gm_finish(const BatchGeom& b, cudaStream_t s) {
  k_b_backsub<<<b.n, 32, 0, s>>>(b.mem);
  FCM_LAUNCH_CHECK();
  k_b_combine<<<dim3(b.max_sys_blocks, b.n), 256, 0, s>>>(b.mem);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

FCM_BOUNDS_READER(bounds_read_blas)

}  // namespace fcm
