// fcm_grid.cu -- separable Gaussian stencils: set-up, spreading, interpolation.
//
// set_up_gaussians restates fcm_fluid_solver.cpp:131-165; spreading restates
// :552-600 (SLIP_CHANNEL false) and interpolation :363-424 / :426-487.
//
// Tiled spreading.  The grid is cut into 8x8x8 tiles.  After set_up_gaussians
// every (blob, tile) overlap is listed per tile (count, scan, fill, then a
// per-tile sort by blob id, so every grid point sums its blobs in ascending blob
// order -- the reference's order).  One CTA per tile stages the weights of its
// blobs restricted to the tile in shared memory, accumulates its 512 points in
// registers and writes every point of the tile exactly once (the zero-fill of
// fcm_fluid_solver.cpp:556-562 is fused: tiles without blobs write zeros).  No
// atomics touch the grid.  Grids that cannot be tiled (a dimension not a
// multiple of 8, or W + 8 > n) use the per-blob atomic scatter.
#include <mutex>
#include <string>

#include "fcm_internal.cuh"

namespace fcm {

namespace {

constexpr int TE = 8;    // tile edge
constexpr int SCB = 32;  // blobs staged per chunk

__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

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

struct TileGeom {
  int ntx, nty, ntz, nx, ny, nz, W;
};

// (blob, tile) overlaps of a blob: per dimension the tiles first..first+cnt-1.
__device__ __forceinline__ void blob_tiles(const int* base, int b, const TileGeom& g, int f[3], int cnt[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int lo = base[3 * b + d];
    f[d] = floordiv(lo, TE);
    cnt[d] = floordiv(lo + g.W - 1, TE) - f[d] + 1;
  }
}

__global__ void k_tile_count(const int* __restrict__ base, int n, TileGeom g, int* __restrict__ count) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int f[3], cnt[3];
  blob_tiles(base, b, g, f, cnt);
  for (int ox = 0; ox < cnt[0]; ++ox)
    for (int oy = 0; oy < cnt[1]; ++oy)
      for (int oz = 0; oz < cnt[2]; ++oz) {
        const int tile = (wrap_index(f[0] + ox, g.ntx) * g.nty + wrap_index(f[1] + oy, g.nty)) * g.ntz +
                         wrap_index(f[2] + oz, g.ntz);
        atomicAdd(count + tile, 1);
      }
}

__global__ void k_tile_fill(const int* __restrict__ base, int n, TileGeom g, const int* __restrict__ offset,
                            int* __restrict__ cursor, unsigned* __restrict__ list) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int f[3], cnt[3];
  blob_tiles(base, b, g, f, cnt);
  for (int ox = 0; ox < cnt[0]; ++ox)
    for (int oy = 0; oy < cnt[1]; ++oy)
      for (int oz = 0; oz < cnt[2]; ++oz) {
        const int tile = (wrap_index(f[0] + ox, g.ntx) * g.nty + wrap_index(f[1] + oy, g.nty)) * g.ntz +
                         wrap_index(f[2] + oz, g.ntz);
        const unsigned j = (unsigned)((ox * cnt[1] + oy) * cnt[2] + oz);
        list[offset[tile] + atomicAdd(cursor + tile, 1)] = ((unsigned)b << 6) | j;
      }
}

// Ascending blob order within each tile (a blob meets a tile at most once).
__global__ void k_tile_sort(const int* __restrict__ offset, int ntiles, unsigned* __restrict__ list) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int b = offset[t], e = offset[t + 1];
  for (int i = b + 1; i < e; ++i) {
    const unsigned v = list[i];
    int j = i - 1;
    while (j >= b && list[j] > v) {
      list[j + 1] = list[j];
      --j;
    }
    list[j + 1] = v;
  }
}

// Stage the weights of the blobs list[c0 .. c0+nc) restricted to this tile:
// sw[k][d][i] = weight of grid coordinate O_d + i along d (zero outside the
// stencil) and sflag[k] bit h = the blob reaches y-half h of the tile.  One
// thread per (blob, dimension) copies its 8-weight window.
template <typename T>
__device__ __forceinline__ void stage_weights(const unsigned* __restrict__ list, int c0, int nc,
                                              const int* __restrict__ base, const T* __restrict__ w, const int O[3],
                                              const int N[3], int W, T (*sw)[3][TE], int* sflag) {
  for (int e = threadIdx.x; e < nc * 3; e += blockDim.x) {
    const int k = e / 3, d = e - 3 * k;
    const int b = (int)(list[c0 + k] >> 6);
    const int Od = (d == 0) ? O[0] : ((d == 1) ? O[1] : O[2]);
    const int Nd = (d == 0) ? N[0] : ((d == 1) ? N[1] : N[2]);
    int s0 = (Od - base[3 * b + d]) % Nd;
    if (s0 < 0) s0 += Nd;
    const T* wb = w + (size_t)(3 * b + d) * W;
    int fl = 0;
#pragma unroll
    for (int i = 0; i < TE; ++i) {
      int si = s0 + i;
      if (si >= Nd) si -= Nd;
      const T v = (si < W) ? wb[si] : (T)0;
      sw[k][d][i] = v;
      if (v != (T)0) fl |= 1 << (i >> 2);
    }
    if (d == 1) sflag[k] = fl;
  }
}

// Tiled spreading: one CTA (64 threads) per 8x8x8 tile.  Thread t owns the
// x-column (y, z) = (t/8, t%8) of the tile, eight points with three components
// accumulated in registers; warp h covers y-half h and skips blobs whose
// stencil misses it (a warp-uniform branch).
template <typename T>
__global__ void __launch_bounds__(64) k_spread_tiled(const int* __restrict__ base, const T* __restrict__ w,
                                                     const double* __restrict__ F, TileGeom g,
                                                     const int* __restrict__ offset,
                                                     const unsigned* __restrict__ list, long long G,
                                                     T* __restrict__ grid) {
  __shared__ T sw[SCB][3][TE];
  __shared__ T sF[SCB][3];
  __shared__ int sflag[SCB];
  const int tile = blockIdx.x;
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int O[3] = {tx * TE, ty * TE, tz * TE};
  const int N[3] = {g.nx, g.ny, g.nz};
  const int t = threadIdx.x;
  const int z = t & 7, y = t >> 3, yh = t >> 5;
  T acc[TE][3];
#pragma unroll
  for (int x = 0; x < TE; ++x)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[x][c] = 0;
  const int b0 = offset[tile], b1 = offset[tile + 1];
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncthreads();
    stage_weights<T>(list, c0, nc, base, w, O, N, g.W, sw, sflag);
    for (int e = t; e < nc * 3; e += 64) {
      const int k = e / 3, c = e - 3 * k;
      sF[k][c] = (T)F[3 * (size_t)(list[c0 + k] >> 6) + c];
    }
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
      if (!((sflag[k] >> yh) & 1)) continue;
      const T wyz = sw[k][1][y] * sw[k][2][z];
      const T f0 = sF[k][0] * wyz, f1 = sF[k][1] * wyz, f2 = sF[k][2] * wyz;
#pragma unroll
      for (int x = 0; x < TE; ++x) {
        const T wx = sw[k][0][x];
        acc[x][0] += f0 * wx;
        acc[x][1] += f1 * wx;
        acc[x][2] += f2 * wx;
      }
    }
  }
#pragma unroll
  for (int x = 0; x < TE; ++x) {
    const long long idx = ((long long)(O[0] + x) * g.ny + (O[1] + y)) * g.nz + (O[2] + z);
    grid[idx] = acc[x][0];
    grid[G + idx] = acc[x][1];
    grid[2 * G + idx] = acc[x][2];
  }
}

// Sum of v[0..31] over the 32 lanes of a warp, scattered: afterwards lane l
// holds in v[0] the warp total of value l (31 shuffles for 32 values).
template <typename T>
__device__ __forceinline__ T warp_reduce_scatter32(T v[32], int lane) {
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < off; ++i) {
      const T send = upper ? v[i] : v[i + off];
      const T keep = upper ? v[i + off] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  return v[0];
}

// Tiled interpolation: one CTA (64 threads) per 8x8x8 tile.  Thread (y, z) =
// (t/8, t%8) loads the eight points of its x-column (three components) into
// registers once.  Blobs are taken eight at a time: each thread forms
// wyz * sum_x wx * u for the blobs its warp's y-half meets, the warp reduces the
// 8x(3+1) values with one scatter-reduction, the two warps' sums are added in
// shared memory, and the per-(blob, tile) partial goes to partial[blob][j][3];
// k_interp_reduce then sums a blob's partials in j order (deterministic, no
// atomics).
template <typename T>
__global__ void __launch_bounds__(64) k_interp_tiled(const int* __restrict__ base, const T* __restrict__ w,
                                                     const T* __restrict__ grid, TileGeom g,
                                                     const int* __restrict__ offset,
                                                     const unsigned* __restrict__ list, long long G,
                                                     T* __restrict__ partial) {
  __shared__ T sw[SCB][3][TE];
  __shared__ int sflag[SCB];
  __shared__ T sred[2][32];
  const int tile = blockIdx.x;
  const int b0 = offset[tile], b1 = offset[tile + 1];
  if (b0 == b1) return;  // no blob meets this tile (uniform over the CTA)
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int O[3] = {tx * TE, ty * TE, tz * TE};
  const int N[3] = {g.nx, g.ny, g.nz};
  const int t = threadIdx.x;
  const int z = t & 7, y = t >> 3, yh = t >> 5, lane = t & 31;
  T u[TE][3];
#pragma unroll
  for (int x = 0; x < TE; ++x) {
    const long long idx = ((long long)(O[0] + x) * g.ny + (O[1] + y)) * g.nz + (O[2] + z);
    u[x][0] = grid[idx];
    u[x][1] = grid[G + idx];
    u[x][2] = grid[2 * G + idx];
  }
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncthreads();
    stage_weights<T>(list, c0, nc, base, w, O, N, g.W, sw, sflag);
    __syncthreads();
    for (int k0 = 0; k0 < nc; k0 += 8) {
      T v[32];
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int k = k0 + j;
        T p0 = 0, p1 = 0, p2 = 0;
        if (k < nc && ((sflag[k] >> yh) & 1)) {
          T s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
          for (int x = 0; x < TE; ++x) {
            const T wx = sw[k][0][x];
            s0 += wx * u[x][0];
            s1 += wx * u[x][1];
            s2 += wx * u[x][2];
          }
          const T wyz = sw[k][1][y] * sw[k][2][z];
          p0 = s0 * wyz;
          p1 = s1 * wyz;
          p2 = s2 * wyz;
        }
        v[4 * j] = p0;
        v[4 * j + 1] = p1;
        v[4 * j + 2] = p2;
        v[4 * j + 3] = 0;
      }
      const T r = warp_reduce_scatter32<T>(v, lane);
      sred[yh][lane] = r;
      __syncthreads();
      if (t < 32) {
        const int j = t >> 2, c = t & 3, k = k0 + j;
        if (c < 3 && k < nc) {
          const unsigned e = list[c0 + k];
          partial[((size_t)(e >> 6) * 64 + (e & 63u)) * 3 + c] = sred[0][t] + sred[1][t];
        }
      }
      __syncthreads();
    }
  }
}

// V = DX^3 * sum over the blob's tiles (in canonical order j) of the partials.
template <typename T>
__global__ void k_interp_reduce(const int* __restrict__ base, const T* __restrict__ partial, int n, TileGeom g,
                                double dx3, double* __restrict__ V) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int f[3], cnt[3];
  blob_tiles(base, b, g, f, cnt);
  const int nj = cnt[0] * cnt[1] * cnt[2];
  double s0 = 0, s1 = 0, s2 = 0;
  const T* p = partial + (size_t)b * 64 * 3;
  for (int j = 0; j < nj; ++j) {
    s0 += (double)p[3 * j];
    s1 += (double)p[3 * j + 1];
    s2 += (double)p[3 * j + 2];
  }
  V[3 * b] = s0 * dx3;
  V[3 * b + 1] = s1 * dx3;
  V[3 * b + 2] = s2 * dx3;
}

// Spreading of grids that cannot be tiled: one CTA per blob, each thread owns
// stencil columns (j,k) and walks x, atomics into the zeroed grid.
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
  if (lane == 0) {
    red[0][wid] = s0;
    red[1][wid] = s1;
    red[2][wid] = s2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    T a0 = 0, a1 = 0, a2 = 0;
    for (int i = 0; i < NT / 32; ++i) {
      a0 += red[0][i];
      a1 += red[1][i];
      a2 += red[2][i];
    }
    V[3 * np] = (double)a0 * dx3;
    V[3 * np + 1] = (double)a1 * dx3;
    V[3 * np + 2] = (double)a2 * dx3;
  }
}

TileGeom tile_geom(const GridDims& g, int W) {
  return TileGeom{g.nx / TE, g.ny / TE, g.nz / TE, g.nx, g.ny, g.nz, W};
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
  const bool ok = g.nx % TE == 0 && g.ny % TE == 0 && g.nz % TE == 0 && W + TE <= g.nx && W + TE <= g.ny &&
                  W + TE <= g.nz && n < (1 << 26);
  if (ok) {
    t.tiled = true;
    t.ntx = g.nx / TE;
    t.nty = g.ny / TE;
    t.ntz = g.nz / TE;
    t.ntiles = t.ntx * t.nty * t.ntz;
    const long long per = (long long)((W + TE - 2) / TE + 1);
    t.tile_cap = (long long)(n > 0 ? n : 1) * per * per * per;
    FCM_CUDA(cudaMalloc(&t.tile_count, sizeof(int) * (size_t)t.ntiles));
    FCM_CUDA(cudaMalloc(&t.tile_offset, sizeof(int) * ((size_t)t.ntiles + 1)));
    FCM_CUDA(cudaMalloc(&t.tile_cursor, sizeof(int) * (size_t)t.ntiles));
    FCM_CUDA(cudaMalloc(&t.tile_list, sizeof(unsigned) * (size_t)t.tile_cap));
    FCM_CUDA(cudaMalloc(&t.partial, sizeof(T) * 64 * 3 * (size_t)(n > 0 ? n : 1)));
  }
  return FCM_OK;
}

template <typename T>
void blob_table_free(BlobTable<T>& t) {
  cudaFree(t.base);
  cudaFree(t.w);
  cudaFree(t.tile_count);
  cudaFree(t.tile_offset);
  cudaFree(t.tile_cursor);
  cudaFree(t.tile_list);
  cudaFree(t.partial);
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
  if (t.tiled) {
    const TileGeom g = tile_geom(c.g, t.W);
    FCM_CUDA(cudaMemsetAsync(t.tile_count, 0, sizeof(int) * (size_t)t.ntiles, s));
    FCM_CUDA(cudaMemsetAsync(t.tile_cursor, 0, sizeof(int) * (size_t)t.ntiles, s));
    k_tile_count<<<(t.n + 127) / 128, 128, 0, s>>>(t.base, t.n, g, t.tile_count);
    FCM_LAUNCH_CHECK();
    FCM_TRY(launch_exclusive_scan(t.tile_count, t.tile_offset, t.ntiles, s));
    k_tile_fill<<<(t.n + 127) / 128, 128, 0, s>>>(t.base, t.n, g, t.tile_offset, t.tile_cursor, t.tile_list);
    FCM_LAUNCH_CHECK();
    k_tile_sort<<<(t.ntiles + 127) / 128, 128, 0, s>>>(t.tile_offset, t.ntiles, t.tile_list);
    FCM_LAUNCH_CHECK();
  }
  return FCM_OK;
}

template <typename T>
int launch_spread(const Ctx& c, const BlobTable<T>& t, const double* dF, T* grid, cudaStream_t s) {
  if (t.tiled) {
    k_spread_tiled<T><<<t.ntiles, 64, 0, s>>>(t.base, t.w, dF, tile_geom(c.g, t.W), t.tile_offset, t.tile_list,
                                               c.g.G, grid);
    FCM_LAUNCH_CHECK();
    return FCM_OK;
  }
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
  if (t.tiled) {
    const TileGeom g = tile_geom(c.g, t.W);
    k_interp_tiled<T><<<t.ntiles, 64, 0, s>>>(t.base, t.w, grid, g, t.tile_offset, t.tile_list, c.g.G, t.partial);
    FCM_LAUNCH_CHECK();
    k_interp_reduce<T><<<(t.n + 127) / 128, 128, 0, s>>>(t.base, t.partial, t.n, g, dx3, dV);
    FCM_LAUNCH_CHECK();
    return FCM_OK;
  }
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

// ============================================================ allocation-free interpolation
// A variant of the tiled interpolation for callers that must not allocate device
// memory: code that runs between the kernels of a time step and may not stall the
// device (cudaMalloc and cudaFree synchronise it), or applications whose device
// memory is owned entirely by their own allocator or memory pool.  Its scratch --
// Gaussian tables, tile lists and per-(blob, tile) partials -- lives in one
// file-scope device array of fixed size, held by every GPU that loads the library
// until the process exits.  Limits: at most NA_MAX_BLOBS blobs, a stencil of at
// most NA_MAX_W points and at most NA_MAX_TILES 8^3 tiles (a 256^3 grid).
namespace fcm {
namespace {

constexpr int NA_MAX_BLOBS = 8192;
constexpr int NA_MAX_W = 24;
constexpr int NA_MAX_TILES = 32768;
constexpr size_t NA_SCRATCH_BYTES = (size_t)20 << 20;  // 20 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

inline size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of g_noalloc_scratch on the current device, looked up once per
// device (the name is only a host-side stand-in in host code).
int noalloc_scratch_address(void** out) {
  static std::mutex mtx;
  static void* addr[256] = {};
  int dev = 0;
  FCM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) {
    set_error("fcm_interp_noalloc: device ordinal out of range");
    return FCM_ERR_INVALID;
  }
  std::lock_guard<std::mutex> lock(mtx);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      set_error(std::string("fcm_interp_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
      return FCM_ERR_CUDA;
    }
    addr[dev] = p;
  }
  *out = addr[dev];
  return FCM_OK;
}

bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace
}  // namespace fcm

extern "C" int fcm_interp_noalloc(int32_t nx, int32_t ny, int32_t nz, double dx, double blob_radius,
                                  int32_t ngauss, int32_t nblobs, const double* Y, const double* grid, double* V,
                                  void* stream) {
  using namespace fcm;
  const int W = ngauss, n = nblobs;
  if (n < 1 || n > NA_MAX_BLOBS) {
    set_error("fcm_interp_noalloc: nblobs must be in [1, " + std::to_string(NA_MAX_BLOBS) + "], got " +
              std::to_string(n));
    return FCM_ERR_INVALID;
  }
  if (W < 1 || W > NA_MAX_W) {
    set_error("fcm_interp_noalloc: ngauss must be in [1, " + std::to_string(NA_MAX_W) + "], got " +
              std::to_string(W));
    return FCM_ERR_INVALID;
  }
  if (nx % TE || ny % TE || nz % TE || W + TE > nx || W + TE > ny || W + TE > nz) {
    set_error("fcm_interp_noalloc: grid dimensions must be multiples of 8 and at least ngauss + 8");
    return FCM_ERR_INVALID;
  }
  const long long ntiles = (long long)(nx / TE) * (ny / TE) * (nz / TE);
  if (ntiles > NA_MAX_TILES) {
    set_error("fcm_interp_noalloc: grid has " + std::to_string(ntiles) + " 8^3 tiles, at most " +
              std::to_string(NA_MAX_TILES) + " are allowed (a 256^3 grid)");
    return FCM_ERR_INVALID;
  }
  if (!(dx > 0.0) || !(blob_radius > 0.0)) {
    set_error("fcm_interp_noalloc: dx and blob_radius must be > 0");
    return FCM_ERR_INVALID;
  }
  if (!on_device(Y) || !on_device(grid) || !on_device(V)) {
    set_error("fcm_interp_noalloc: Y, grid and V must be device pointers");
    return FCM_ERR_INVALID;
  }
  void* base_ptr = nullptr;
  FCM_TRY(noalloc_scratch_address(&base_ptr));
  // carve the scratch array
  const int per = (W + TE - 2) / TE + 1;
  const size_t cap = (size_t)n * per * per * per;
  unsigned char* p = (unsigned char*)base_ptr;
  int* s_base = (int*)p;
  p += round256(sizeof(int) * 3 * (size_t)n);
  double* s_w = (double*)p;
  p += round256(sizeof(double) * 3 * (size_t)W * n);
  int* s_count = (int*)p;
  p += round256(sizeof(int) * (size_t)ntiles);
  int* s_offset = (int*)p;
  p += round256(sizeof(int) * ((size_t)ntiles + 1));
  int* s_cursor = (int*)p;
  p += round256(sizeof(int) * (size_t)ntiles);
  unsigned* s_list = (unsigned*)p;
  p += round256(sizeof(unsigned) * cap);
  double* s_partial = (double*)p;
  p += round256(sizeof(double) * 64 * 3 * (size_t)n);
  if ((size_t)(p - (unsigned char*)base_ptr) > NA_SCRATCH_BYTES) {
    set_error("fcm_interp_noalloc: scratch layout exceeds the static array");
    return FCM_ERR_INVALID;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const double PI = 3.14159265358979323846264338327950288;
  const double anorm = 1.0 / (sqrt(2.0) * blob_radius);
  const double anorm2 = 2.0 * blob_radius * blob_radius / PI;
  const TileGeom g{nx / TE, ny / TE, nz / TE, nx, ny, nz, W};
  const long long G = (long long)nx * ny * nz;
  // the array keeps the previous call's contents: counters start at zero
  FCM_CUDA(cudaMemsetAsync(s_count, 0, sizeof(int) * (size_t)ntiles, s));
  FCM_CUDA(cudaMemsetAsync(s_cursor, 0, sizeof(int) * (size_t)ntiles, s));
  k_set_up_gaussians<double><<<(3 * n + 127) / 128, 128, 0, s>>>(Y, n, W, dx, anorm, anorm2, s_base, s_w);
  FCM_LAUNCH_CHECK();
  k_tile_count<<<(n + 127) / 128, 128, 0, s>>>(s_base, n, g, s_count);
  FCM_LAUNCH_CHECK();
  FCM_TRY(launch_exclusive_scan(s_count, s_offset, (int)ntiles, s));
  k_tile_fill<<<(n + 127) / 128, 128, 0, s>>>(s_base, n, g, s_offset, s_cursor, s_list);
  FCM_LAUNCH_CHECK();
  k_tile_sort<<<(unsigned)((ntiles + 127) / 128), 128, 0, s>>>(s_offset, (int)ntiles, s_list);
  FCM_LAUNCH_CHECK();
  k_interp_tiled<double><<<(unsigned)ntiles, 64, 0, s>>>(s_base, s_w, grid, g, s_offset, s_list, G, s_partial);
  FCM_LAUNCH_CHECK();
  k_interp_reduce<double><<<(n + 127) / 128, 128, 0, s>>>(s_base, s_partial, n, g, dx * dx * dx, V);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}
