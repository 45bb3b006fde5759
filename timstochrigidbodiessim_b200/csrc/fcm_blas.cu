// fcm_blas.cu -- FP64 vector operations of the GMRES solver
// (gmres_solver.cpp:148-306): deterministic dot products and norms, fused
// modified-Gram-Schmidt steps, scaling and the final Krylov combination.
//
// Reductions are single-launch and deterministic: a fixed grid writes one
// partial per block, and the last block to finish (ticket counter, no waiting)
// sums the partials in index order.
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
__device__ __forceinline__ void finish(double my_partial, double* partials, unsigned int* counter, double* out,
                                       int mode, double* sh) {
  __shared__ bool last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = my_partial;
    __threadfence();
    const unsigned int ticket = atomicAdd(counter, 1u);
    last = (ticket == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double v = 0.0;
  // fixed assignment of partials to threads, then a fixed-order block sum
  for (int i = threadIdx.x; i < (int)gridDim.x; i += RT) v += ((volatile double*)partials)[i];
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
  finish(bs, partials, counter, out, mode, sh);
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
  finish(bs, partials, counter, hout, q_i ? 0 : 2, sh);
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
