// fcm_grid.cu -- separable Gaussian stencils: set-up, spreading, interpolation.
//
// set_up_gaussians restates fcm_fluid_solver.cpp:131-165; spreading restates
// :552-600 (SLIP_CHANNEL false) and interpolation :363-424 / :426-487.
#include "fcm_internal.cuh"

namespace fcm {

namespace {

__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

// One thread per (blob, dimension): xc = int(Y/DX); stencil start
// xc - W/2 + 1; weight anorm*exp(-(xg*DX - Y)^2/anorm2), with sigma = a/sqrt(pi)
// implicit in anorm = 1/(sqrt(2) a), anorm2 = 2a^2/pi (fcm_fluid_solver.cpp:135-136).
template <typename T>
__global__ void k_set_up_gaussians(const double* __restrict__ Y, int n, int W, double dx, double anorm,
                                   double anorm2, int* __restrict__ base, T* __restrict__ w) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const double y = Y[t];
  const int xc = (int)__ddiv_rn(y, dx);
  const int b = xc - W / 2 + 1;
  base[t] = b;
  T* wt = w + (size_t)t * W;
  for (int i = 0; i < W; ++i) {
    const double xx = __dsub_rn(__dmul_rn((double)(b + i), dx), y);
    const double e = exp(__ddiv_rn(-__dmul_rn(xx, xx), anorm2));
    wt[i] = (T)(anorm * e);
  }
}

// Spreading, one CTA per blob; each thread owns stencil columns (j,k) and walks
// x.  Scatter with atomics into the zeroed grid.
template <typename T>
__global__ void k_spread_atomic(const int* __restrict__ base, const T* __restrict__ w, const double* __restrict__ F,
                                int W, int nx, int ny, int nz, long long G, T* __restrict__ grid) {
  const int np = blockIdx.x;
  const int bx = base[3 * np], by = base[3 * np + 1], bz = base[3 * np + 2];
  const T* gx = w + (size_t)(3 * np) * W;
  const T* gy = gx + W;
  const T* gz = gy + W;
  const T f0 = (T)F[3 * np], f1 = (T)F[3 * np + 1], f2 = (T)F[3 * np + 2];
  for (int jk = threadIdx.x; jk < W * W; jk += blockDim.x) {
    const int j = jk / W, k = jk - j * W;
    const int yy = wrap_index(by + j, ny), zz = wrap_index(bz + k, nz);
    const T wyz = gy[j] * gz[k];
    for (int i = 0; i < W; ++i) {
      const int xx = wrap_index(bx + i, nx);
      const T wt = gx[i] * wyz;
      const long long idx = ((long long)xx * ny + yy) * nz + zz;
      atomicAdd(grid + idx, f0 * wt);
      atomicAdd(grid + G + idx, f1 * wt);
      atomicAdd(grid + 2 * G + idx, f2 * wt);
    }
  }
}

// Interpolation, one CTA per blob, block reduction; V = DX^3 * sum u*gx*gy*gz.
template <typename T, int NT>
__global__ void __launch_bounds__(NT) k_interp_block(const int* __restrict__ base, const T* __restrict__ w,
                                                     const T* __restrict__ grid, int W, int nx, int ny, int nz,
                                                     long long G, double dx3, double* __restrict__ V) {
  const int np = blockIdx.x;
  const int bx = base[3 * np], by = base[3 * np + 1], bz = base[3 * np + 2];
  const T* gx = w + (size_t)(3 * np) * W;
  const T* gy = gx + W;
  const T* gz = gy + W;
  T s0 = 0, s1 = 0, s2 = 0;
  for (int jk = threadIdx.x; jk < W * W; jk += NT) {
    const int j = jk / W, k = jk - j * W;
    const int yy = wrap_index(by + j, ny), zz = wrap_index(bz + k, nz);
    const T wyz = gy[j] * gz[k];
    for (int i = 0; i < W; ++i) {
      const int xx = wrap_index(bx + i, nx);
      const T wt = gx[i] * wyz;
      const long long idx = ((long long)xx * ny + yy) * nz + zz;
      s0 += grid[idx] * wt;
      s1 += grid[G + idx] * wt;
      s2 += grid[2 * G + idx] * wt;
    }
  }
  __shared__ T red[3][NT / 32];
  for (int off = 16; off > 0; off >>= 1) {
    s0 += __shfl_down_sync(0xffffffffu, s0, off);
    s1 += __shfl_down_sync(0xffffffffu, s1, off);
    s2 += __shfl_down_sync(0xffffffffu, s2, off);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) { red[0][wid] = s0; red[1][wid] = s1; red[2][wid] = s2; }
  __syncthreads();
  if (threadIdx.x == 0) {
    T a0 = 0, a1 = 0, a2 = 0;
    for (int i = 0; i < NT / 32; ++i) { a0 += red[0][i]; a1 += red[1][i]; a2 += red[2][i]; }
    V[3 * np] = (double)a0 * dx3;
    V[3 * np + 1] = (double)a1 * dx3;
    V[3 * np + 2] = (double)a2 * dx3;
  }
}

}  // namespace

template <typename T>
int blob_table_alloc(BlobTable<T>& t, int n, int W, const GridDims& g) {
  if (t.n == n && t.W == W && t.base) return FCM_OK;
  blob_table_free(t);
  t.n = n;
  t.W = W;
  FCM_CUDA(cudaMalloc(&t.base, sizeof(int) * 3 * (size_t)(n > 0 ? n : 1)));
  FCM_CUDA(cudaMalloc(&t.w, sizeof(T) * 3 * (size_t)W * (n > 0 ? n : 1)));
  (void)g;
  return FCM_OK;
}

template <typename T>
void blob_table_free(BlobTable<T>& t) {
  cudaFree(t.base);
  cudaFree(t.w);
  cudaFree(t.tile_count);
  cudaFree(t.tile_blobs);
  cudaFree(t.tile_cursor);
  cudaFree(t.tile_total);
  t = BlobTable<T>();
}

template <typename T>
int launch_set_up_gaussians(const Ctx& c, BlobTable<T>& t, const double* dY, cudaStream_t s) {
  if (t.n == 0) return FCM_OK;
  const double PI = 3.14159265358979323846264338327950288;
  const double a = c.p.blob_radius;
  const double anorm = 1.0 / (sqrt(2.0) * a);
  const double anorm2 = 2.0 * a * a / PI;
  const int nt = 3 * t.n;
  k_set_up_gaussians<T><<<(nt + 127) / 128, 128, 0, s>>>(dY, t.n, t.W, c.g.dx, anorm, anorm2, t.base, t.w);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template <typename T>
int launch_spread(const Ctx& c, const BlobTable<T>& t, const double* dF, T* grid, cudaStream_t s) {
  FCM_CUDA(cudaMemsetAsync(grid, 0, sizeof(T) * 3 * (size_t)c.g.G, s));
  if (t.n == 0) return FCM_OK;
  k_spread_atomic<T><<<t.n, 128, 0, s>>>(t.base, t.w, dF, t.W, c.g.nx, c.g.ny, c.g.nz, c.g.G, grid);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template <typename T>
int launch_interp(const Ctx& c, const BlobTable<T>& t, const T* grid, double* dV, cudaStream_t s) {
  if (t.n == 0) return FCM_OK;
  const double dx3 = c.g.dx * c.g.dx * c.g.dx;
  k_interp_block<T, 256><<<t.n, 256, 0, s>>>(t.base, t.w, grid, t.W, c.g.nx, c.g.ny, c.g.nz, c.g.G, dx3, dV);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template int blob_table_alloc<double>(BlobTable<double>&, int, int, const GridDims&);
template int blob_table_alloc<float>(BlobTable<float>&, int, int, const GridDims&);
template void blob_table_free<double>(BlobTable<double>&);
template void blob_table_free<float>(BlobTable<float>&);
template int launch_set_up_gaussians<double>(const Ctx&, BlobTable<double>&, const double*, cudaStream_t);
template int launch_set_up_gaussians<float>(const Ctx&, BlobTable<float>&, const double*, cudaStream_t);
template int launch_spread<double>(const Ctx&, const BlobTable<double>&, const double*, double*, cudaStream_t);
template int launch_spread<float>(const Ctx&, const BlobTable<float>&, const double*, float*, cudaStream_t);
template int launch_interp<double>(const Ctx&, const BlobTable<double>&, const double*, double*, cudaStream_t);
template int launch_interp<float>(const Ctx&, const BlobTable<float>&, const float*, double*, cudaStream_t);

}  // namespace fcm
