// fcm_grid.cu -- separable Gaussian stencils: set-up, spreading, interpolation.
//
// set_up_gaussians restates fcm_fluid_solver.cpp:131-165; spreading restates
// :552-600 (SLIP_CHANNEL false) and interpolation :363-424 / :426-487.
//
// Tiled spreading.  The grid is cut into 8x8x8 tiles.  Once per position set
// (set_up_gaussians) every blob's weights are also laid out on the 8-aligned
// grid chunks its stencil meets -- per dimension four chunks of eight weights,
// zero outside the stencil -- and every (blob, tile) overlap is listed per tile
// as one 64-bit entry: blob id, the chunk index per dimension, the blob's
// canonical tile index j and which halves of the tile the stencil reaches (count,
// scan, fill, then a per-tile sort by blob id, so every grid point sums its blobs
// in ascending blob order -- the reference's order).  One CTA per tile copies the
// three 8-weight chunks of each of its blobs into shared memory with vector loads
// (no index arithmetic beyond the entry), accumulates its 512 points in registers
// and writes every point of the tile exactly once (the zero-fill of
// fcm_fluid_solver.cpp:556-562 is fused: tiles without blobs write zeros).  No
// atomics touch the grid.  Grids that cannot be tiled (a dimension not a multiple
// of 8, W + 8 > n, or W > 25) use the per-blob atomic scatter.
#include <algorithm>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "fcm_internal.cuh"

namespace fcm {

namespace {

constexpr int TE = 8;    // tile edge
constexpr int NCH = 4;   // 8-aligned chunks a stencil of at most 25 points meets per dimension
constexpr int MAXW = 25;
constexpr int SCB = 16;  // blobs staged per round (four staging lanes per blob, 64 threads)

// Entry layout (low word): bits 0-5 chunk index per dimension (2 bits each),
// 6-11 canonical tile index j of the blob, 12-13 / 14-15 / 16-17 x / y / z
// halves of the tile the stencil reaches.  The blob id is the high word.
constexpr int EJ = 6, EXM = 12, EYM = 14, EZM = 16;

__device__ __forceinline__ int wrap_index(int i, int n) {
  int r = i % n;
  return r < 0 ? r + n : r;
}

__device__ __forceinline__ int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// One thread per (blob, dimension): xc = int(Y/DX); stencil start
// xc - W/2 + 1; weight anorm*exp(-(xg*DX - Y)^2/anorm2), with sigma = a/sqrt(pi)
// implicit in anorm = 1/(sqrt(2) a), anorm2 = 2a^2/pi (fcm_fluid_solver.cpp:135-136).
// With wc given, the weights are also written on the NCH 8-aligned chunks from
// floor(base/8)*8 on (zero outside the stencil).
template <typename T>
__global__ void k_set_up_gaussians(const double* __restrict__ Y, int n, int W, double dx, double anorm,
                                   double anorm2, int* __restrict__ base, T* __restrict__ w, T* __restrict__ wc,
                                   double* __restrict__ ypos) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const double y = Y[t];
  if (ypos) ypos[t] = y;
  const int xc = (int)__ddiv_rn(y, dx);
  const int b = xc - W / 2 + 1;
  base[t] = b;
  T* wt = w + (size_t)t * W;
  for (int i = 0; i < W; ++i) {
    const double xx = __dsub_rn(__dmul_rn((double)(b + i), dx), y);
    const double e = exp(__ddiv_rn(-__dmul_rn(xx, xx), anorm2));
    wt[i] = (T)(anorm * e);
  }
  if (wc) {
    const int c0 = floordiv(b, TE) * TE;
    T* ct = wc + (size_t)t * NCH * TE;
    for (int i = 0; i < NCH * TE; ++i) {
      const int s = c0 + i - b;
      ct[i] = (s >= 0 && s < W) ? wt[s] : (T)0;
    }
  }
}

// The same tables with one warp per (blob, dimension): lane i takes grid point
// c0 + i of the blob's NCH * TE = 32-point chunk window (c0 = floor(base/8)*8),
// evaluates its weight with the arithmetic above when it lies in the stencil
// (s = c0 + i - base in [0, W)) and writes wc[i] and w[s]; every store is
// coalesced and each weight is computed once (the window holds the stencil since
// W <= 25 on tiled grids).  Without wc the lanes write w[i], i = lane, lane + 32, ...
template <typename T>
__global__ void __launch_bounds__(128) k_set_up_gaussians_warp(const double* __restrict__ Y, int n, int W, double dx,
                                                               double anorm, double anorm2, int* __restrict__ base,
                                                               T* __restrict__ w, T* __restrict__ wc,
                                                               double* __restrict__ ypos) {
  const long long t = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= 3LL * n) return;  // uniform over the warp
  const double y = Y[t];
  const int xc = (int)__ddiv_rn(y, dx);
  const int b = xc - W / 2 + 1;
  if (lane == 0) {
    base[t] = b;
    if (ypos) ypos[t] = y;
  }
  if (!wc) {
    for (int i = lane; i < W; i += 32) {
      const double xx = __dsub_rn(__dmul_rn((double)(b + i), dx), y);
      w[t * W + i] = (T)(anorm * exp(__ddiv_rn(-__dmul_rn(xx, xx), anorm2)));
    }
    return;
  }
  const int c0 = floordiv(b, TE) * TE;  // first grid point of the window
  const int g = c0 + lane, sidx = g - b;
  T val = (T)0;
  if (sidx >= 0 && sidx < W) {
    const double xx = __dsub_rn(__dmul_rn((double)g, dx), y);
    const double e = exp(__ddiv_rn(-__dmul_rn(xx, xx), anorm2));
    val = (T)(anorm * e);
    w[t * W + sidx] = val;
  }
  wc[t * NCH * TE + lane] = val;
}

// (blob, tile) overlaps of a blob: per dimension the tiles first..first+cnt-1.
__device__ __forceinline__ void blob_tiles(const int* base, int b, const TileGeom& g, int f[3], int cnt[3]) {
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int lo = base[3 * b + d];
    f[d] = floordiv(lo, TE);
    cnt[d] = floordiv(lo + g.W - 1, TE) - f[d] + 1;
  }
}

// Bit h (h = 0, 1) set when the stencil [lo, lo + W) meets half h of the chunk
// starting at s.
__device__ __forceinline__ unsigned half_mask(int lo, int W, int s) {
  return (lo < s + 4 && lo + W > s ? 1u : 0u) | (lo < s + 8 && lo + W > s + 4 ? 2u : 0u);
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
        if (FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) atomicAdd(count + tile, 1);
      }
}

__global__ void k_tile_fill(const int* __restrict__ base, int n, TileGeom g, const int* __restrict__ offset,
                            int* __restrict__ cursor, unsigned long long* __restrict__ list) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int f[3], cnt[3];
  blob_tiles(base, b, g, f, cnt);
  const int lx = base[3 * b], ly = base[3 * b + 1], lz = base[3 * b + 2];
  for (int ox = 0; ox < cnt[0]; ++ox)
    for (int oy = 0; oy < cnt[1]; ++oy)
      for (int oz = 0; oz < cnt[2]; ++oz) {
        const int tile = (wrap_index(f[0] + ox, g.ntx) * g.nty + wrap_index(f[1] + oy, g.nty)) * g.ntz +
                         wrap_index(f[2] + oz, g.ntz);
        if (!FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) continue;
        const unsigned j = (unsigned)((ox * cnt[1] + oy) * cnt[2] + oz);
        const unsigned lo = (unsigned)ox | ((unsigned)oy << 2) | ((unsigned)oz << 4) | (j << EJ) |
                            (half_mask(lx, g.W, (f[0] + ox) * TE) << EXM) |
                            (half_mask(ly, g.W, (f[1] + oy) * TE) << EYM) |
                            (half_mask(lz, g.W, (f[2] + oz) * TE) << EZM);
        const int slot = offset[tile] + atomicAdd(cursor + tile, 1);
        if (FCM_INB(slot, offset[tile + 1], BS_LIST) && FCM_INB(slot, g.list_cap, BS_LIST))
          list[slot] = ((unsigned long long)b << 32) | lo;
      }
}

// Ascending blob order within each tile (a blob meets a tile at most once).
__global__ void k_tile_sort(const int* __restrict__ offset, int ntiles, unsigned long long* __restrict__ list,
                            long long cap) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntiles) return;
  const int b = offset[t], e = offset[t + 1];
  if (!FCM_INB(b, (long long)e + 1, BS_LIST) || !FCM_INB(e, cap + 1, BS_LIST)) return;
  for (int i = b + 1; i < e; ++i) {
    const unsigned long long v = list[i];
    int j = i - 1;
    while (j >= b && list[j] > v) {
      list[j + 1] = list[j];
      --j;
    }
    list[j + 1] = v;
  }
}

// The same order, one warp per tile: the tile's entries (all distinct) are
// loaded into a shared buffer padded to a power of two with all-ones keys and
// bitonic-sorted by the warp; tiles with more than TSORT entries are sorted by
// lane 0 in place as k_tile_sort does.  128 threads = four tiles per CTA.
constexpr int TSORT = 256;
__global__ void __launch_bounds__(128) k_tile_sort_warp(const int* __restrict__ offset, int ntiles,
                                                        unsigned long long* __restrict__ list, long long cap) {
  __shared__ unsigned long long buf[4][TSORT];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int t = blockIdx.x * 4 + w;
  if (t >= ntiles) return;  // uniform over the warp
  const int b = offset[t], e = offset[t + 1], n = e - b;
  if (!FCM_INB(b, (long long)e + 1, BS_LIST) || !FCM_INB(e, cap + 1, BS_LIST)) return;  // uniform over the warp
  if (n < 2) return;
  if (n > TSORT) {
    if (lane == 0)
      for (int i = b + 1; i < e; ++i) {
        const unsigned long long v = list[i];
        int j = i - 1;
        while (j >= b && list[j] > v) {
          list[j + 1] = list[j];
          --j;
        }
        list[j + 1] = v;
      }
    return;
  }
  int P = 2;
  while (P < n) P <<= 1;
  unsigned long long* a = buf[w];
  for (int i = lane; i < P; i += 32) a[i] = i < n ? list[b + i] : ~0ull;
  __syncwarp();
  for (int k = 2; k <= P; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = lane; i < P; i += 32) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned long long x = a[i], y = a[l];
          const bool up = (i & k) == 0;
          if ((x > y) == up) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
      __syncwarp();
    }
  for (int i = lane; i < n; i += 32) list[b + i] = a[i];
}

// Eight consecutive T from global (aligned to 8*sizeof(T)) to shared memory.
__device__ __forceinline__ void copy8(double* dst, const double* __restrict__ src) {
  const double2* s = reinterpret_cast<const double2*>(src);
  double2* d = reinterpret_cast<double2*>(dst);
  const double2 a = __ldg(s), b = __ldg(s + 1), c = __ldg(s + 2), e = __ldg(s + 3);
  d[0] = a;
  d[1] = b;
  d[2] = c;
  d[3] = e;
}
__device__ __forceinline__ void copy8(float* dst, const float* __restrict__ src) {
  const float4* s = reinterpret_cast<const float4*>(src);
  float4* d = reinterpret_cast<float4*>(dst);
  const float4 a = __ldg(s), b = __ldg(s + 1);
  d[0] = a;
  d[1] = b;
}

// The tile-list entry at slot.  In the bounds-checked build a slot beyond the
// list's capacity or a blob id beyond the tables reads as entry 0, whose empty
// half masks make the spreading and interpolation skip it.
__device__ __forceinline__ unsigned long long list_entry(const unsigned long long* __restrict__ list, long long slot,
                                                         const TileGeom& g) {
  if (!FCM_INB(slot, g.list_cap, BS_LIST)) return 0ull;
  const unsigned long long e = list[slot];
  if (!FCM_INB(e >> 32, g.nblobs, BS_BLOB)) return 0ull;
  return e;
}

// A tile's entry range [b0, b1) of the list; in the bounds-checked build a range
// outside 0 <= b0 <= b1 <= capacity reads as empty.
__device__ __forceinline__ void tile_range(const int* __restrict__ offset, int tile, const TileGeom& g, int& b0,
                                           int& b1) {
  b0 = offset[tile];
  b1 = offset[tile + 1];
  if (!FCM_INB(b0, (long long)b1 + 1, BS_LIST) || !FCM_INB(b1, g.list_cap + 1, BS_LIST)) b1 = b0;
}

// Stage blobs list[c0 .. c0+nc) (nc <= SCB) of a tile: lane (k, d) = (t/4, t%4)
// copies chunk d of blob k for d < 3; lane d = 3 copies the entry's low word and,
// when F is given, the blob's force.
template <typename T>
__device__ __forceinline__ void stage_blobs(const unsigned long long* __restrict__ list, int c0, int nc,
                                            const T* __restrict__ wc, const double* __restrict__ F,
                                            T (*sw)[3][TE], T (*sF)[4], unsigned* sflag, const TileGeom& g) {
  const int k = threadIdx.x >> 2, d = threadIdx.x & 3;
  if (k >= nc) return;
  const unsigned long long e = list_entry(list, c0 + k, g);
  const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
  if (d < 3) {
    copy8(sw[k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
  } else {
    sflag[k] = lo;
    if (F) {
      sF[k][0] = (T)F[3 * (size_t)b];
      sF[k][1] = (T)F[3 * (size_t)b + 1];
      sF[k][2] = (T)F[3 * (size_t)b + 2];
    }
  }
}

// The same staging for NB blobs per round (any NB): the (blob, lane) pairs are
// dealt to the 64 threads in turn.
template <typename T, int NB>
__device__ __forceinline__ void stage_blobs_n(const unsigned long long* __restrict__ list, int c0, int nc,
                                              const T* __restrict__ wc, const double* __restrict__ F,
                                              T (*sw)[3][TE], T (*sF)[4], unsigned* sflag, const TileGeom& g) {
  for (int i = threadIdx.x; i < 4 * nc; i += 64) {
    const int k = i >> 2, d = i & 3;
    const unsigned long long e = list_entry(list, c0 + k, g);
    const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
    if (d < 3) {
      copy8(sw[k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
    } else {
      sflag[k] = lo;
      sF[k][0] = (T)F[3 * (size_t)b];
      sF[k][1] = (T)F[3 * (size_t)b + 1];
      sF[k][2] = (T)F[3 * (size_t)b + 2];
    }
  }
}

template <typename T>
struct V4 {};
template <>
struct V4<double> {
  // two doubles
  static __device__ __forceinline__ void ld(const double* p, double& a, double& b) {
    const double2 v = *reinterpret_cast<const double2*>(p);
    a = v.x;
    b = v.y;
  }
};
// x-weights xs..xs+3 (xs = 0 or 4) of a staged chunk into registers: two
// 16-byte shared loads for doubles, one for floats.
template <typename T>
__device__ __forceinline__ void load_wx4(const T* row, int xs, T wx[4]) {
  V4<T>::ld(row + xs, wx[0], wx[1]);
  V4<T>::ld(row + xs + 2, wx[2], wx[3]);
}
template <>
__device__ __forceinline__ void load_wx4<float>(const float* row, int xs, float wx[4]) {
  const float4 v = *reinterpret_cast<const float4*>(row + xs);
  wx[0] = v.x;
  wx[1] = v.y;
  wx[2] = v.z;
  wx[3] = v.w;
}

// Whether to skip an x-half the stencil misses: worth its test for FP64 (the
// FP64 pipe is the tighter limit); in FP32 the test costs about what it saves.
template <typename T>
__device__ __forceinline__ bool skip_x_half(unsigned fl, int h) {
  return sizeof(T) == 8 && !((fl >> (EXM + h)) & 1u);
}

// Tiled spreading: one CTA (64 threads) per 8x8x8 tile.  Thread t owns the
// x-column (y, z) = (t/8, t%8) of the tile, eight points with three components
// accumulated in registers.  Warp h covers y-half h and skips blobs whose
// stencil misses it; in FP64 an x-half the stencil misses is skipped by the
// whole CTA (both branches are uniform).
// NB blobs are staged per round (SCB by default); every point sums its blobs in
// ascending blob order whatever NB is, so the grids are the same bit for bit.
template <typename T, int NB = SCB>
__device__ __forceinline__ void spread_tile(const T* __restrict__ wc, const double* __restrict__ F,
                                            const TileGeom& g, const int* __restrict__ offset,
                                            const unsigned long long* __restrict__ list, long long G,
                                            T* __restrict__ grid, int tile) {
  __shared__ __align__(16) T sw[NB][3][TE];
  __shared__ __align__(16) T sF[NB][4];
  __shared__ unsigned sflag[NB];
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int t = threadIdx.x;
  const int z = t & 7, y = t >> 3, yh = t >> 5;
  if (!FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) return;  // uniform over the CTA
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  if constexpr (sizeof(T) == 4) {
    // FP32: the x-points in pairs, one packed two-lane FMA (fma.rn.f32x2) per pair
    // and component; each lane rounds as the scalar FMA does, so the sums are the
    // same bit for bit.
    float2 acc2[TE / 2][3];
#pragma unroll
    for (int x = 0; x < TE / 2; ++x)
#pragma unroll
      for (int c = 0; c < 3; ++c) acc2[x][c] = make_float2(0.f, 0.f);
    for (int c0 = b0; c0 < b1; c0 += NB) {
      const int nc = min(NB, b1 - c0);
      if (c0 != b0) __syncthreads();
      stage_blobs_n<T, NB>(list, c0, nc, wc, F, sw, sF, sflag, g);
      __syncthreads();
      for (int k = 0; k < nc; ++k) {
        const unsigned fl = sflag[k];
        if (!((fl >> (EYM + yh)) & 1u)) continue;
        const float wyz = sw[k][1][y] * sw[k][2][z];
        const float f0 = sF[k][0] * wyz, f1 = sF[k][1] * wyz, f2 = sF[k][2] * wyz;
        const float2 fc[3] = {make_float2(f0, f0), make_float2(f1, f1), make_float2(f2, f2)};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const float4 v = *reinterpret_cast<const float4*>(&sw[k][0][4 * h]);
          const float2 wa = make_float2(v.x, v.y), wb = make_float2(v.z, v.w);
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            acc2[2 * h][c] = __ffma2_rn(fc[c], wa, acc2[2 * h][c]);
            acc2[2 * h + 1][c] = __ffma2_rn(fc[c], wb, acc2[2 * h + 1][c]);
          }
        }
      }
    }
    const int ox = tx * TE, oy = ty * TE + y, oz = tz * TE + z;
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
      if (!FCM_INB(idx, G, BS_GRID)) continue;
#pragma unroll
      for (int c = 0; c < 3; ++c) grid[c * G + idx] = (x & 1) ? acc2[x >> 1][c].y : acc2[x >> 1][c].x;
    }
  } else {
    T acc[TE][3];
#pragma unroll
    for (int x = 0; x < TE; ++x)
#pragma unroll
      for (int c = 0; c < 3; ++c) acc[x][c] = 0;
    for (int c0 = b0; c0 < b1; c0 += NB) {
      const int nc = min(NB, b1 - c0);
      if (c0 != b0) __syncthreads();
      stage_blobs_n<T, NB>(list, c0, nc, wc, F, sw, sF, sflag, g);
      __syncthreads();
      for (int k = 0; k < nc; ++k) {
        const unsigned fl = sflag[k];
        if (!((fl >> (EYM + yh)) & 1u)) continue;
        const T wyz = sw[k][1][y] * sw[k][2][z];
        const T f0 = sF[k][0] * wyz, f1 = sF[k][1] * wyz, f2 = sF[k][2] * wyz;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (skip_x_half<T>(fl, h)) continue;
          T wx[4];
          load_wx4<T>(sw[k][0], 4 * h, wx);
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            acc[4 * h + i][0] += f0 * wx[i];
            acc[4 * h + i][1] += f1 * wx[i];
            acc[4 * h + i][2] += f2 * wx[i];
          }
        }
      }
    }
    const int ox = tx * TE, oy = ty * TE + y, oz = tz * TE + z;
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
      if (!FCM_INB(idx, G, BS_GRID)) continue;
      grid[idx] = acc[x][0];
      grid[G + idx] = acc[x][1];
      grid[2 * G + idx] = acc[x][2];
    }
  }
}

template <typename T, int NB = SCB>
__global__ void __launch_bounds__(64) k_spread_tiled(const T* __restrict__ wc, const double* __restrict__ F,
                                                     TileGeom g, const int* __restrict__ offset,
                                                     const unsigned long long* __restrict__ list, long long G,
                                                     T* __restrict__ grid) {
  spread_tile<T, NB>(wc, F, g, offset, list, G, grid, blockIdx.x);
}

// Tiled spreading by one warp per 8x8x8 tile: lane (yq, z) = (lane / 8, lane % 8)
// owns the x-columns of rows y = yq and yq + 4 (eight points each, three
// components, in registers) and adds each staged blob to the rows its stencil
// meets (FP32: the packed FMA over x-pairs).  The flag, x-weights and force of a
// blob are read once for both rows.  Every point sums its blobs in ascending order
// with the products of k_spread_tiled (f_c = F_c wy wz, then f_c wx), so the grid
// is the same bit for bit.
template <typename T>
__global__ void __launch_bounds__(32) k_spread_warp(const T* __restrict__ wc, const double* __restrict__ F,
                                                    TileGeom g, const int* __restrict__ offset,
                                                    const unsigned long long* __restrict__ list, long long G,
                                                    T* __restrict__ grid) {
  __shared__ __align__(16) T sw[SCB][3][TE];
  __shared__ __align__(16) T sF[SCB][4];
  __shared__ unsigned sflag[SCB];
  const int tile = blockIdx.x;
  if (!FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) return;  // uniform over the warp
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int lane = threadIdx.x, z = lane & 7, yq = lane >> 3;
  constexpr int XA = sizeof(T) == 4 ? TE / 2 : TE;  // x accumulators per row (pairs in FP32)
  using A = typename std::conditional<sizeof(T) == 4, float2, T>::type;
  A acc[2][XA][3];
#pragma unroll
  for (int r = 0; r < 2; ++r)
#pragma unroll
    for (int x = 0; x < XA; ++x)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if constexpr (sizeof(T) == 4) acc[r][x][c] = make_float2(0.f, 0.f);
        else acc[r][x][c] = 0;
      }
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncwarp();
    for (int i = lane; i < 4 * nc; i += 32) {  // staging: lane d of blob k
      const int k = i >> 2, d = i & 3;
      const unsigned long long e = list_entry(list, c0 + k, g);
      const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
      if (d < 3) {
        copy8(sw[k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
      } else {
        sflag[k] = lo;
        sF[k][0] = (T)F[3 * (size_t)b];
        sF[k][1] = (T)F[3 * (size_t)b + 1];
        sF[k][2] = (T)F[3 * (size_t)b + 2];
      }
    }
    __syncwarp();
    for (int k = 0; k < nc; ++k) {
      const unsigned fl = sflag[k];
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        if (!((fl >> (EYM + r)) & 1u)) continue;  // uniform over the warp
        const T wyz = sw[k][1][yq + 4 * r] * sw[k][2][z];
        const T f0 = sF[k][0] * wyz, f1 = sF[k][1] * wyz, f2 = sF[k][2] * wyz;
        if constexpr (sizeof(T) == 4) {
          const float2 fc[3] = {make_float2(f0, f0), make_float2(f1, f1), make_float2(f2, f2)};
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const float4 v = *reinterpret_cast<const float4*>(&sw[k][0][4 * h]);
            const float2 wa = make_float2(v.x, v.y), wb = make_float2(v.z, v.w);
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              acc[r][2 * h][c] = __ffma2_rn(fc[c], wa, acc[r][2 * h][c]);
              acc[r][2 * h + 1][c] = __ffma2_rn(fc[c], wb, acc[r][2 * h + 1][c]);
            }
          }
        } else {
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            if (skip_x_half<T>(fl, h)) continue;
            T wx[4];
            load_wx4<T>(sw[k][0], 4 * h, wx);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              acc[r][4 * h + i][0] += f0 * wx[i];
              acc[r][4 * h + i][1] += f1 * wx[i];
              acc[r][4 * h + i][2] += f2 * wx[i];
            }
          }
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int ox = tx * TE, oy = ty * TE + yq + 4 * r, oz = tz * TE + z;
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
      if (!FCM_INB(idx, G, BS_GRID)) continue;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if constexpr (sizeof(T) == 4)
          grid[c * G + idx] = (x & 1) ? acc[r][x >> 1][c].y : acc[r][x >> 1][c].x;
        else
          grid[c * G + idx] = acc[r][x][c];
      }
    }
  }
}

// ------------------------------------------------------------------ persistent pipelined tiles
// Work items of a persistent CTA: its tiles blockIdx.x, +gridDim.x, ..., each cut
// into staging rounds of SCB blobs (one empty round for a tile without blobs).
// The tile offsets are loaded two tiles ahead, so the generator never waits.
struct TileItem {
  int tile, c0, nc, last;
};

struct ItemGen {
  const int* __restrict__ offset;
  int ntiles, stride;
  int tile, c0, b1;
  int o1a, o1b, o2a, o2b;  // offsets of tile + stride and tile + 2 stride

  __device__ __forceinline__ void load_off(int tl, int& a, int& b) const {
    if (tl < ntiles) {
      a = offset[tl];
      b = offset[tl + 1];
    } else {
      a = b = 0;
    }
  }
  __device__ __forceinline__ bool first() {
    tile = blockIdx.x;
    if (tile >= ntiles) return false;
    c0 = offset[tile];
    b1 = offset[tile + 1];
    load_off(tile + stride, o1a, o1b);
    load_off(tile + 2 * stride, o2a, o2b);
    return true;
  }
  __device__ __forceinline__ bool next() {
    if (c0 + SCB < b1) {
      c0 += SCB;
      return true;
    }
    tile += stride;
    if (tile >= ntiles) return false;
    c0 = o1a;
    b1 = o1b;
    o1a = o2a;
    o1b = o2b;
    load_off(tile + 2 * stride, o2a, o2b);
    return true;
  }
  __device__ __forceinline__ TileItem item() const {
    return TileItem{tile, c0, min(SCB, b1 - c0), (c0 + SCB >= b1) ? 1 : 0};
  }
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Asynchronous copy of one 8-weight chunk (32 B float, 64 B double) to shared memory.
template <typename T>
__device__ __forceinline__ void chunk_async(T* dst, const T* __restrict__ src) {
#pragma unroll
  for (int i = 0; i < (int)(TE * sizeof(T) / 16); ++i) cp_async16(reinterpret_cast<char*>(dst) + 16 * i,
                                                                  reinterpret_cast<const char*>(src) + 16 * i);
}

// Persistent, software-pipelined tiled spreading: the arithmetic of
// k_spread_tiled (each point sums its blobs in the same order), but a CTA walks
// over many tiles and, while it accumulates one staging round, the weight
// chunks of the next round are already on their way to the other shared buffer
// (cp.async) and the list entries of the round after that are being loaded.
template <typename T>
__global__ void __launch_bounds__(64) k_spread_pipe(const T* __restrict__ wc, const double* __restrict__ F, TileGeom g,
                                                    const int* __restrict__ offset,
                                                    const unsigned long long* __restrict__ list, long long G,
                                                    T* __restrict__ grid, int ntiles) {
  __shared__ __align__(16) T sw[2][SCB][3][TE];
  __shared__ __align__(16) T sF[2][SCB][4];
  __shared__ unsigned sflag[2][SCB];
  const int t = threadIdx.x, k = t >> 2, d = t & 3;
  const int z = t & 7, y = t >> 3, yh = t >> 5;
  ItemGen gen{offset, ntiles, (int)gridDim.x, 0, 0, 0, 0, 0, 0, 0};
  if (!gen.first()) return;  // uniform over the CTA
  TileItem cur = gen.item();
  bool v1 = gen.next();
  TileItem nx1 = v1 ? gen.item() : TileItem{0, 0, 0, 0};
  bool v2 = v1 && gen.next();
  TileItem nx2 = v2 ? gen.item() : TileItem{0, 0, 0, 0};
  // prologue: the first round straight into buffer 0
  if (k < cur.nc) {
    const unsigned long long e = list_entry(list, cur.c0 + k, g);
    const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
    if (d < 3) {
      chunk_async<T>(sw[0][k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
    } else {
      sflag[0][k] = lo;
      sF[0][k][0] = (T)F[3 * (size_t)b];
      sF[0][k][1] = (T)F[3 * (size_t)b + 1];
      sF[0][k][2] = (T)F[3 * (size_t)b + 2];
    }
  }
  cp_async_commit();
  unsigned long long e1 = (v1 && k < nx1.nc) ? list_entry(list, nx1.c0 + k, g) : 0ull;
  cp_async_wait_all();
  __syncthreads();
  T acc[TE][3];
#pragma unroll
  for (int x = 0; x < TE; ++x)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[x][c] = 0;
  int buf = 0;
  while (true) {
    // the next round's weights into the other buffer, its forces into registers
    double fn0 = 0, fn1 = 0, fn2 = 0;
    unsigned fln = 0;
    if (v1 && k < nx1.nc) {
      const unsigned b = (unsigned)(e1 >> 32), lo = (unsigned)e1;
      if (d < 3) {
        chunk_async<T>(sw[buf ^ 1][k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
      } else {
        fln = lo;
        fn0 = F[3 * (size_t)b];
        fn1 = F[3 * (size_t)b + 1];
        fn2 = F[3 * (size_t)b + 2];
      }
    }
    cp_async_commit();
    // the entries of the round after
    const unsigned long long e2 = (v2 && k < nx2.nc) ? list_entry(list, nx2.c0 + k, g) : 0ull;
    // accumulate this round
    for (int kk = 0; kk < cur.nc; ++kk) {
      const unsigned fl = sflag[buf][kk];
      if (!((fl >> (EYM + yh)) & 1u)) continue;
      const T wyz = sw[buf][kk][1][y] * sw[buf][kk][2][z];
      const T f0 = sF[buf][kk][0] * wyz, f1 = sF[buf][kk][1] * wyz, f2 = sF[buf][kk][2] * wyz;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (skip_x_half<T>(fl, h)) continue;
        T wx[4];
        load_wx4<T>(sw[buf][kk][0], 4 * h, wx);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          acc[4 * h + i][0] += f0 * wx[i];
          acc[4 * h + i][1] += f1 * wx[i];
          acc[4 * h + i][2] += f2 * wx[i];
        }
      }
    }
    if (v1 && k < nx1.nc && d == 3) {
      sflag[buf ^ 1][k] = fln;
      sF[buf ^ 1][k][0] = (T)fn0;
      sF[buf ^ 1][k][1] = (T)fn1;
      sF[buf ^ 1][k][2] = (T)fn2;
    }
    if (cur.last) {  // the tile is complete: every point written once
      const int tz = cur.tile % g.ntz, ty = (cur.tile / g.ntz) % g.nty, tx = cur.tile / (g.ntz * g.nty);
      const int ox = tx * TE, oy = ty * TE + y, oz = tz * TE + z;
#pragma unroll
      for (int x = 0; x < TE; ++x) {
        const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
        if (FCM_INB(idx, G, BS_GRID)) {
          grid[idx] = acc[x][0];
          grid[G + idx] = acc[x][1];
          grid[2 * G + idx] = acc[x][2];
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[x][c] = 0;
      }
    }
    cp_async_wait_all();
    __syncthreads();
    if (!v1) break;
    cur = nx1;
    nx1 = nx2;
    v1 = v2;
    e1 = e2;
    buf ^= 1;
    v2 = v2 && gen.next();
    if (v2) nx2 = gen.item();
  }
}

// Sum of v[0..15] over the 32 lanes of a warp, scattered: afterwards lanes 2i
// and 2i+1 hold in v[0] the warp total of value i (16 shuffles for 16 values).
template <typename T>
__device__ __forceinline__ T warp_reduce_scatter16(T v[16], int lane) {
#pragma unroll
  for (int off = 16, m = 8; off >= 2; off >>= 1, m >>= 1) {
    const bool upper = (lane & off) != 0;
#pragma unroll
    for (int i = 0; i < m; ++i) {
      const T send = upper ? v[i] : v[i + m];
      const T keep = upper ? v[i + m] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
    }
  }
  return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// The x-column of one (y, z) point of a tile, three components, in registers,
// and its contraction with a blob's x-weights: s_c = sum_x wx[x] u_c[x] (x-halves
// the stencil misses skipped where skip_x_half says so).  FP64 sums the points in
// order; FP32 holds the column as x-point pairs and sums even and odd points in
// the two lanes of the packed FMA (fma.rn.f32x2), then adds the lanes.
template <typename T>
struct XColumn {
  T u[3][TE];
  __device__ __forceinline__ void set(int x, T a, T b, T c) {
    u[0][x] = a;
    u[1][x] = b;
    u[2][x] = c;
  }
  __device__ __forceinline__ void contract(const T* wrow, unsigned fl, T& s0, T& s1, T& s2) const {
    s0 = 0;
    s1 = 0;
    s2 = 0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      if (skip_x_half<T>(fl, h)) continue;
      T wx[4];
      load_wx4<T>(wrow, 4 * h, wx);
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        s0 += wx[i] * u[0][4 * h + i];
        s1 += wx[i] * u[1][4 * h + i];
        s2 += wx[i] * u[2][4 * h + i];
      }
    }
  }
};
template <>
struct XColumn<float> {
  float2 u[3][TE / 2];
  __device__ __forceinline__ void set(int x, float a, float b, float c) {
    if (x & 1) {
      u[0][x >> 1].y = a;
      u[1][x >> 1].y = b;
      u[2][x >> 1].y = c;
    } else {
      u[0][x >> 1].x = a;
      u[1][x >> 1].x = b;
      u[2][x >> 1].x = c;
    }
  }
  __device__ __forceinline__ void contract(const float* wrow, unsigned, float& s0, float& s1, float& s2) const {
    float2 a0 = make_float2(0.f, 0.f), a1 = a0, a2 = a0;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const float4 w4 = *reinterpret_cast<const float4*>(wrow + 4 * h);
      const float2 wa = make_float2(w4.x, w4.y), wb = make_float2(w4.z, w4.w);
      a0 = __ffma2_rn(wa, u[0][2 * h], a0);
      a1 = __ffma2_rn(wa, u[1][2 * h], a1);
      a2 = __ffma2_rn(wa, u[2][2 * h], a2);
      a0 = __ffma2_rn(wb, u[0][2 * h + 1], a0);
      a1 = __ffma2_rn(wb, u[1][2 * h + 1], a1);
      a2 = __ffma2_rn(wb, u[2][2 * h + 1], a2);
    }
    s0 = a0.x + a0.y;
    s1 = a1.x + a1.y;
    s2 = a2.x + a2.y;
  }
};

// Tiled interpolation: one CTA (64 threads) per 8x8x8 tile.  Thread (y, z) =
// (t/8, t%8) loads the eight points of its x-column (three components) into
// registers once.  Blobs are taken four at a time: each thread forms
// wyz * sum_x wx * u for the blobs its warp's y-half meets (x-halves the
// stencil misses are skipped), the warp reduces the 4x(3+1) values with one
// scatter-reduction, the two warps' sums are added in shared memory, and the
// per-(blob, tile) partial goes to partial[blob][j][3]; k_interp_reduce then
// sums a blob's partials in j order (deterministic, no atomics).
template <typename T>
__device__ __forceinline__ void interp_tile(const T* __restrict__ wc, const T* __restrict__ grid, const TileGeom& g,
                                            const int* __restrict__ offset,
                                            const unsigned long long* __restrict__ list, long long G,
                                            T* __restrict__ partial, int tile) {
  __shared__ __align__(16) T sw[SCB][3][TE];
  __shared__ unsigned sflag[SCB];
  __shared__ unsigned sblob[SCB];
  __shared__ T sred[SCB / 4][2][16];
  if (!FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) return;  // uniform over the CTA
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  if (b0 == b1) return;  // no blob meets this tile (uniform over the CTA)
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int t = threadIdx.x;
  const int z = t & 7, y = t >> 3, yh = t >> 5, lane = t & 31;
  XColumn<T> col;
  {
    const int ox = tx * TE, oy = ty * TE + y, oz = tz * TE + z;
    const bool live = oy < g.ycut;  // rows at or above the slip channel's upper wall read as 0
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
      const bool in = live && FCM_INB(idx, G, BS_GRID);
      col.set(x, in ? grid[idx] : (T)0, in ? grid[G + idx] : (T)0, in ? grid[2 * G + idx] : (T)0);
    }
  }
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncthreads();
    stage_blobs<T>(list, c0, nc, wc, nullptr, sw, nullptr, sflag, g);
    if ((t & 3) == 3 && (t >> 2) < nc) sblob[t >> 2] = (unsigned)(list_entry(list, c0 + (t >> 2), g) >> 32);
    __syncthreads();
    for (int k0 = 0; k0 < nc; k0 += 4) {
      T v[16];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        T p0 = 0, p1 = 0, p2 = 0;
        const unsigned fl = k < nc ? sflag[k] : 0u;
        if ((fl >> (EYM + yh)) & 1u) {
          T s0, s1, s2;
          col.contract(sw[k][0], fl, s0, s1, s2);
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
      const T r = warp_reduce_scatter16<T>(v, lane);
      if (!(lane & 1)) sred[k0 >> 2][yh][lane >> 1] = r;
    }
    __syncthreads();
    // thread t: group t/16 of four blobs, value t%16 = (blob, component)
    {
      const int grp = t >> 4, i = t & 15, c = i & 3, k = 4 * grp + (i >> 2);
      if (c < 3 && k < nc) {
        const unsigned jt = (sflag[k] >> EJ) & 63u;
        if (FCM_INB((long long)sblob[k] * 64 + jt, (long long)g.nblobs * 64, BS_PARTIAL))
          partial[((size_t)sblob[k] * 64 + jt) * 3 + c] = sred[grp][0][i] + sred[grp][1][i];
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(64) k_interp_tiled(const T* __restrict__ wc, const T* __restrict__ grid,
                                                     TileGeom g, const int* __restrict__ offset,
                                                     const unsigned long long* __restrict__ list, long long G,
                                                     T* __restrict__ partial) {
  interp_tile<T>(wc, grid, g, offset, list, G, partial, blockIdx.x);
}

// Tiled interpolation with R y-rows per thread: 64/R threads per 8x8x8 tile (one
// warp for R = 2).  Thread t = (yq, z) = (t/8, t%8) holds the x-columns of rows
// yq + r*8/R, r < R, three components each, in registers.  Per blob and row the
// thread contracts its column with the blob's x-weights (x-halves and y-halves the
// stencil misses are skipped; both tests are uniform over the CTA), scales by
// wy*wz and adds the rows.  The per-thread values of a staging round go to a
// shared buffer [3*SCB][64/R + pad] and each row (blob, component) is summed by
// one thread in lane order (the padding keeps the vector reads conflict-free).
// In FP32 the x-contraction runs on x-point pairs with the packed two-lane FMA.
// The partial per (blob, tile) goes to partial[blob][j][3] as in k_interp_tiled;
// k_interp_reduce sums them.  Fewer instructions per (blob, tile) than the
// shuffle reduction of k_interp_tiled: the three components need no padding
// slot, and with R = 2 the weight loads and flag tests are shared by two rows.
template <typename T, int R>
__global__ void __launch_bounds__(64 / R) k_interp_rows(const T* __restrict__ wc, const T* __restrict__ grid,
                                                        TileGeom g, const int* __restrict__ offset,
                                                        const unsigned long long* __restrict__ list, long long G,
                                                        T* __restrict__ partial) {
  constexpr int NT = 64 / R;                    // threads per tile
  constexpr int RS = NT + 16 / (int)sizeof(T);  // padded reduction row
  constexpr int YS = TE / R;                    // row step between a thread's rows
  __shared__ __align__(16) T sw[SCB][3][TE];
  __shared__ unsigned sflag[SCB];
  __shared__ unsigned sblob[SCB];
  __shared__ __align__(16) T sred[3 * SCB][RS];
  const int tile = blockIdx.x;
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  if (b0 == b1) return;  // no blob meets this tile (uniform over the CTA)
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int t = threadIdx.x;
  const int z = t & 7, yq = t >> 3;
  T u[R][3][TE];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int oy = ty * TE + yq + r * YS;
    const bool live = oy < g.ycut;  // rows at or above the slip channel's upper wall read as 0
    const long long base = ((long long)(tx * TE) * g.ny + oy) * g.nz + tz * TE + z;
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const bool in = FCM_INB(base + (long long)x * g.ny * g.nz, G, BS_GRID);
#pragma unroll
      for (int c = 0; c < 3; ++c)
        u[r][c][x] = (live && in) ? grid[c * G + base + (long long)x * g.ny * g.nz] : (T)0;
    }
  }
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncthreads();
    for (int i = t; i < 4 * nc; i += NT) {
      const int k = i >> 2, d = i & 3;
      const unsigned long long e = list_entry(list, c0 + k, g);
      const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
      if (d < 3) {
        copy8(sw[k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
      } else {
        sflag[k] = lo;
        sblob[k] = b;
      }
    }
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
      const unsigned fl = sflag[k];
      T p0 = 0, p1 = 0, p2 = 0;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int h = R == 2 ? r : (yq >> 2);  // y-half of this row
        if (!((fl >> (EYM + h)) & 1u)) continue;
        T s0, s1, s2;
        if constexpr (sizeof(T) == 4) {
          float2 a0 = make_float2(0.f, 0.f), a1 = a0, a2 = a0;
#pragma unroll
          for (int xh = 0; xh < 2; ++xh) {
            if (!((fl >> (EXM + xh)) & 1u)) continue;
            const float4 w4 = *reinterpret_cast<const float4*>(&sw[k][0][4 * xh]);
            const float2 wa = make_float2(w4.x, w4.y), wb = make_float2(w4.z, w4.w);
            const int x0 = 4 * xh;
            a0 = __ffma2_rn(wa, make_float2(u[r][0][x0], u[r][0][x0 + 1]), a0);
            a1 = __ffma2_rn(wa, make_float2(u[r][1][x0], u[r][1][x0 + 1]), a1);
            a2 = __ffma2_rn(wa, make_float2(u[r][2][x0], u[r][2][x0 + 1]), a2);
            a0 = __ffma2_rn(wb, make_float2(u[r][0][x0 + 2], u[r][0][x0 + 3]), a0);
            a1 = __ffma2_rn(wb, make_float2(u[r][1][x0 + 2], u[r][1][x0 + 3]), a1);
            a2 = __ffma2_rn(wb, make_float2(u[r][2][x0 + 2], u[r][2][x0 + 3]), a2);
          }
          s0 = a0.x + a0.y;
          s1 = a1.x + a1.y;
          s2 = a2.x + a2.y;
        } else {
          s0 = 0;
          s1 = 0;
          s2 = 0;
#pragma unroll
          for (int xh = 0; xh < 2; ++xh) {
            if (!((fl >> (EXM + xh)) & 1u)) continue;
            T wx[4];
            load_wx4<T>(sw[k][0], 4 * xh, wx);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              s0 += wx[i] * u[r][0][4 * xh + i];
              s1 += wx[i] * u[r][1][4 * xh + i];
              s2 += wx[i] * u[r][2][4 * xh + i];
            }
          }
        }
        const T wyz = sw[k][1][yq + r * YS] * sw[k][2][z];
        p0 += s0 * wyz;
        p1 += s1 * wyz;
        p2 += s2 * wyz;
      }
      sred[3 * k][t] = p0;
      sred[3 * k + 1][t] = p1;
      sred[3 * k + 2][t] = p2;
    }
    __syncthreads();
    for (int rr = t; rr < 3 * nc; rr += NT) {
      T sum = 0;
      if constexpr (sizeof(T) == 4) {
#pragma unroll
        for (int j = 0; j < NT; j += 4) {
          const float4 v = *reinterpret_cast<const float4*>(&sred[rr][j]);
          sum += v.x;
          sum += v.y;
          sum += v.z;
          sum += v.w;
        }
      } else {
#pragma unroll
        for (int j = 0; j < NT; j += 2) {
          const double2 v = *reinterpret_cast<const double2*>(&sred[rr][j]);
          sum += v.x;
          sum += v.y;
        }
      }
      const int k = rr / 3, c = rr - 3 * (rr / 3);
      const unsigned jt = (sflag[k] >> EJ) & 63u;
      if (FCM_INB((long long)sblob[k] * 64 + jt, (long long)g.nblobs * 64, BS_PARTIAL))
        partial[((size_t)sblob[k] * 64 + jt) * 3 + c] = sum;
    }
  }
}

// Tiled interpolation by one warp per 8x8x8 tile: lane (yq, z) = (lane / 8,
// lane % 8) holds the x-columns of rows y = yq and yq + 4 (one in each y-half),
// three components, in registers.  Per blob it contracts each row the stencil
// meets with the blob's x-weights (FP32: the packed FMA over x-pairs), scales by
// wy wz and adds the two rows, so each lane carries three values per blob; the
// warp reduces four blobs at a time with the 16-value shuffle reduce-scatter and
// lanes 2i write value i straight to partial[blob][j][c].  Against the 64-thread
// kernel this halves the reductions per (blob, tile) pair and needs no CTA
// barrier or shared-memory sum: only the staged weights pass through shared memory.
template <typename T>
__global__ void __launch_bounds__(32) k_interp_warp(const T* __restrict__ wc, const T* __restrict__ grid,
                                                    TileGeom g, const int* __restrict__ offset,
                                                    const unsigned long long* __restrict__ list, long long G,
                                                    T* __restrict__ partial) {
  __shared__ __align__(16) T sw[SCB][3][TE];
  __shared__ unsigned sflag[SCB], sblob[SCB];
  const int tile = blockIdx.x;
  if (!FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) return;  // uniform over the warp
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  if (b0 == b1) return;  // no blob meets this tile
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int lane = threadIdx.x, z = lane & 7, yq = lane >> 3;
  XColumn<T> col[2];
#pragma unroll
  for (int r = 0; r < 2; ++r) {
    const int ox = tx * TE, oy = ty * TE + yq + 4 * r, oz = tz * TE + z;
    const bool live = oy < g.ycut;  // rows at or above the slip channel's upper wall read as 0
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
      const bool in = live && FCM_INB(idx, G, BS_GRID);
      col[r].set(x, in ? grid[idx] : (T)0, in ? grid[G + idx] : (T)0, in ? grid[2 * G + idx] : (T)0);
    }
  }
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncwarp();
    for (int i = lane; i < 4 * nc; i += 32) {  // staging: lane d of blob k
      const int k = i >> 2, d = i & 3;
      const unsigned long long e = list_entry(list, c0 + k, g);
      const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
      if (d < 3) {
        copy8(sw[k][d], wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
      } else {
        sflag[k] = lo;
        sblob[k] = b;
      }
    }
    __syncwarp();
    for (int k0 = 0; k0 < nc; k0 += 4) {
      T v[16];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int k = k0 + j;
        const unsigned fl = k < nc ? sflag[k] : 0u;
        T p0 = 0, p1 = 0, p2 = 0;
#pragma unroll
        for (int r = 0; r < 2; ++r) {
          if (!((fl >> (EYM + r)) & 1u)) continue;  // uniform over the warp
          T s0, s1, s2;
          col[r].contract(sw[k][0], fl, s0, s1, s2);
          const T wyz = sw[k][1][yq + 4 * r] * sw[k][2][z];
          p0 += s0 * wyz;
          p1 += s1 * wyz;
          p2 += s2 * wyz;
        }
        v[4 * j] = p0;
        v[4 * j + 1] = p1;
        v[4 * j + 2] = p2;
        v[4 * j + 3] = 0;
      }
      const T sum = warp_reduce_scatter16<T>(v, lane);
      if (!(lane & 1)) {  // lanes 2i and 2i + 1 hold value i = 4 j + c
        const int i = lane >> 1, j = i >> 2, cc = i & 3, k = k0 + j;
        if (cc < 3 && k < nc) {
          const unsigned jt = (sflag[k] >> EJ) & 63u;
          if (FCM_INB((long long)sblob[k] * 64 + jt, (long long)g.nblobs * 64, BS_PARTIAL))
            partial[((size_t)sblob[k] * 64 + jt) * 3 + cc] = sum;
        }
      }
    }
  }
}

// ------------------------------------------------------------------ tensor-core tiles (FP32 grids)
// FP32 spreading and interpolation of one 8x8x8 tile by one warp on the tensor
// cores (mma.sync m16n8k8 with TF32 operands and FP32 accumulators).  Seen as a
// 64 x 24 matrix C[(y, z), (c, x)], a tile's grid is a sum over its blobs k of
// (wy_k[y] wz_k[z]) (F_kc wx_k[x]): the product of a 64 x K and a K x 24 matrix,
// K the tile's blobs, eight per k-step (blobs padded with zero weights).  Every
// operand is split into its TF32 rounding and the FP32 remainder, and three
// products are summed (hi*lo, lo*hi, then hi*hi; lo*lo dropped), which keeps
// each term to about 2^-22 relative, the rounding level of FP32 itself.  The
// grid agrees with the FMA kernels' to FP32 rounding, not bit for bit.
// Interpolation is the transpose: P[k, (c, x)] = sum over (y, z) of
// (wy_k[y] wz_k[z]) grid_c[x][y][z] (16 blobs x 64 (y, z) times 64 x 24, the
// tile's grid held as operand fragments in registers), then
// partial_kc = sum over x of P[k, (c, x)] wx_k[x].
//
// Fragments of m16n8k8 (g = lane / 4, t = lane % 4): A (16 x 8, row-major)
// a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4); B (8 x 8,
// column-major) b0 (t, g), b1 (t + 4, g); C (16 x 8) c0 (g, 2t), c1 (g, 2t + 1),
// c2 (g + 8, 2t), c3 (g + 8, 2t + 1).

// a = hi + lo with hi the TF32 rounding of a (low 13 mantissa bits zero; to
// nearest, ties away from zero: half of bit 13 added to the magnitude bits, then
// truncated, a carry into the exponent rounding up a binade) and lo the exact
// FP32 remainder (Sterbenz), read as TF32 by the tensor core.  Finite a only.
__device__ __forceinline__ void tf32_split(float a, unsigned& hi, unsigned& lo) {
  const unsigned h = (__float_as_uint(a) + 0x1000u) & 0xffffe000u;
  hi = h;
  lo = __float_as_uint(a - __uint_as_float(h));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
      "{%0, %1, %2, %3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += a * b in 3xTF32.
__device__ __forceinline__ void mma_3xtf32(float (&d)[4], const unsigned (&ah)[4], const unsigned (&al)[4],
                                           unsigned bh0, unsigned bh1, unsigned bl0, unsigned bl1) {
  mma_tf32(d, al, bh0, bh1);
  mma_tf32(d, ah, bl0, bl1);
  mma_tf32(d, ah, bh0, bh1);
}

// Staging of a warp's rounds of RB blobs (RB / 8 items of four parts per lane:
// part 0-2 the blob's x, y, z weight chunk, part 3 its force or nothing).  The
// kernels below keep three rounds in a pipeline: one computed from a shared
// buffer, the next one's chunks in flight to registers, the entries of the one
// after that being loaded.  Slots past a round's blobs read as entry 0, whose
// empty half masks mark padding: zero weights and forces, nothing written.
template <int RB, bool WITH_F>
struct MmaStage {
  static constexpr int NI = RB / 8;  // items per lane
  unsigned long long e[NI];          // entries of the round after the one in flight
  float4 v0[NI], v1[NI];             // chunks in flight
  double f0[NI], f1[NI], f2[NI];     // forces in flight (part 3, WITH_F)
  unsigned long long ef[NI];         // entries of the round in flight

  __device__ __forceinline__ void load_entries(const unsigned long long* __restrict__ list, const TileItem& it,
                                               const TileGeom& g) {
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const int k = 8 * i + (threadIdx.x >> 2);
      e[i] = k < it.nc ? list_entry(list, it.c0 + k, g) : 0ull;
    }
  }
  __device__ __forceinline__ void issue(const float* __restrict__ wc, const double* __restrict__ F) {
    const int d = threadIdx.x & 3;
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      ef[i] = e[i];
      const unsigned b = (unsigned)(e[i] >> 32), lo = (unsigned)e[i];
      const bool ok = ((lo >> EXM) & 63u) != 0u;
      v0[i] = v1[i] = make_float4(0.f, 0.f, 0.f, 0.f);
      f0[i] = f1[i] = f2[i] = 0.0;
      if (ok && d < 3) {
        const float4* src =
            reinterpret_cast<const float4*>(wc + ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE);
        v0[i] = __ldg(src);
        v1[i] = __ldg(src + 1);
      } else if (WITH_F && ok) {
        f0[i] = F[3 * (size_t)b];
        f1[i] = F[3 * (size_t)b + 1];
        f2[i] = F[3 * (size_t)b + 2];
      }
    }
  }
  __device__ __forceinline__ void put(float (*sw)[3][TE], float (*sF)[4], unsigned* sflag, unsigned* sblob) const {
    const int d = threadIdx.x & 3;
#pragma unroll
    for (int i = 0; i < NI; ++i) {
      const int k = 8 * i + (threadIdx.x >> 2);
      if (d < 3) {
        *reinterpret_cast<float4*>(&sw[k][d][0]) = v0[i];
        *reinterpret_cast<float4*>(&sw[k][d][4]) = v1[i];
      } else {
        if (WITH_F) *reinterpret_cast<float4*>(sF[k]) = make_float4((float)f0[i], (float)f1[i], (float)f2[i], 0.f);
        if (sflag) sflag[k] = (unsigned)ef[i];
        if (sblob) sblob[k] = (unsigned)(ef[i] >> 32);
      }
    }
  }
};

// One warp per tile in rounds of eight blobs (one k-step), the staging pipelined
// within the tile.  (A persistent form with the pipeline running on across
// tiles, like k_interp_mma's, measured 2% slower: its 168 registers leave fewer
// warps per SM.)
__global__ void __launch_bounds__(32) k_spread_mma(const float* __restrict__ wc, const double* __restrict__ F,
                                                   TileGeom g, const int* __restrict__ offset,
                                                   const unsigned long long* __restrict__ list, long long G,
                                                   float* __restrict__ grid) {
  __shared__ __align__(16) float sw[2][8][3][TE];
  __shared__ __align__(16) float sF[2][8][4];
  const int tile = blockIdx.x;
  if (!FCM_INB(tile, (long long)g.ntx * g.nty * g.ntz, BS_TILE)) return;  // uniform over the warp
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  float acc[4][3][4];  // [(y, z) row block m][component][fragment]
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[m][c][r] = 0.f;
  const int R = (b1 - b0 + 7) >> 3;  // rounds of eight blobs (one k-step)
  auto round = [&](int r) {
    const int c0 = b0 + 8 * r;
    return TileItem{tile, c0, max(0, min(8, b1 - c0)), 0};
  };
  MmaStage<8, true> st;
  if (R > 0) {
    st.load_entries(list, round(0), g);
    st.issue(wc, F);
    st.put(sw[0], sF[0], nullptr, nullptr);
    st.load_entries(list, round(1), g);
    st.issue(wc, F);
    st.load_entries(list, round(2), g);
  }
  for (int r = 0; r < R; ++r) {
    __syncwarp();
    const int cur = r & 1;
    if (r + 1 < R) {
      st.put(sw[cur ^ 1], sF[cur ^ 1], nullptr, nullptr);
      st.issue(wc, F);
      st.load_entries(list, round(r + 3), g);
    }
    const int ka = tq, kb = tq + 4;
    // B = (F_kc wx_k[x]) for blobs ka, kb and x = gq
    const float xa = sw[cur][ka][0][gq], xb = sw[cur][kb][0][gq];
    const float4 fa = *reinterpret_cast<const float4*>(sF[cur][ka]);
    const float4 fb = *reinterpret_cast<const float4*>(sF[cur][kb]);
    unsigned bh[3][2], bl[3][2];
    tf32_split(fa.x * xa, bh[0][0], bl[0][0]);
    tf32_split(fb.x * xb, bh[0][1], bl[0][1]);
    tf32_split(fa.y * xa, bh[1][0], bl[1][0]);
    tf32_split(fb.y * xb, bh[1][1], bl[1][1]);
    tf32_split(fa.z * xa, bh[2][0], bl[2][0]);
    tf32_split(fb.z * xb, bh[2][1], bl[2][1]);
    // A = (wy_k[y] wz_k[z]) for rows (y, z) = (2m, gq), (2m + 1, gq)
    const float za = sw[cur][ka][2][gq], zb = sw[cur][kb][2][gq];
    float ya[TE], yb[TE];
    *reinterpret_cast<float4*>(ya) = *reinterpret_cast<const float4*>(&sw[cur][ka][1][0]);
    *reinterpret_cast<float4*>(ya + 4) = *reinterpret_cast<const float4*>(&sw[cur][ka][1][4]);
    *reinterpret_cast<float4*>(yb) = *reinterpret_cast<const float4*>(&sw[cur][kb][1][0]);
    *reinterpret_cast<float4*>(yb + 4) = *reinterpret_cast<const float4*>(&sw[cur][kb][1][4]);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
      unsigned ah[4], al[4];
      tf32_split(ya[2 * m] * za, ah[0], al[0]);
      tf32_split(ya[2 * m + 1] * za, ah[1], al[1]);
      tf32_split(yb[2 * m] * zb, ah[2], al[2]);
      tf32_split(yb[2 * m + 1] * zb, ah[3], al[3]);
#pragma unroll
      for (int c = 0; c < 3; ++c) mma_3xtf32(acc[m][c], ah, al, bh[c][0], bh[c][1], bl[c][0], bl[c][1]);
    }
  }
  const int ox = tx * TE, oy = ty * TE, oz = tz * TE + gq;
#pragma unroll
  for (int m = 0; m < 4; ++m)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int x = 2 * tq + (r & 1), y = 2 * m + (r >> 1);
      const long long idx = ((long long)(ox + x) * g.ny + oy + y) * g.nz + oz;
      if (!FCM_INB(idx, G, BS_GRID)) continue;
#pragma unroll
      for (int c = 0; c < 3; ++c) grid[c * G + idx] = acc[m][c][r];
    }
}

// Grid tile of the interpolation in shared memory: [component][x][y][z] with each
// x-plane padded to 68 floats, so the fragment reads (eight x-planes, four z)
// fall in 32 different banks.
constexpr int SGX = TE * TE + 4;

// Asynchronous copy of a tile's three 8^3 blocks (3 x 8 x 8 rows of 32 bytes, two
// 16-byte copies each, twelve per lane) into sg; rows at or above ycut are left
// to the reader, which reads them as 0.
__device__ __forceinline__ void grid_tile_async(const float* __restrict__ grid, const TileGeom& g, long long G,
                                                int tile, float* sg) {
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
#pragma unroll
  for (int q = 0; q < 12; ++q) {
    const int i = threadIdx.x + 32 * q, row = i >> 1, half = i & 1;
    const int c = row >> 6, x = (row >> 3) & 7, y = row & 7;
    const long long idx = ((long long)(tx * TE + x) * g.ny + ty * TE + y) * g.nz + tz * TE + 4 * half;
    float* dst = sg + c * TE * SGX + x * SGX + y * TE + 4 * half;
    if (FCM_INB(idx + 3, G, BS_GRID))
      cp_async16(dst, grid + c * G + idx);
    else
      *reinterpret_cast<float4*>(dst) = make_float4(0.f, 0.f, 0.f, 0.f);
  }
  cp_async_commit();
}

// Persistent like k_spread_mma, in rounds of 16 blobs (one m-tile); the grid of
// the warp's next tile is copied to the other shared buffer while the current
// tile's rounds run, and turned into operand fragments when that tile starts.
__global__ void __launch_bounds__(32) k_interp_mma(const float* __restrict__ wc, const float* __restrict__ grid,
                                                   TileGeom g, const int* __restrict__ offset,
                                                   const unsigned long long* __restrict__ list, long long G,
                                                   float* __restrict__ partial, int ntiles) {
  __shared__ __align__(16) float sw[2][SCB][3][TE];
  __shared__ unsigned sflag[2][SCB], sblob[2][SCB];
  __shared__ __align__(16) float sg[2][3 * TE * SGX];
  ItemGen gen{offset, ntiles, (int)gridDim.x, 0, 0, 0, 0, 0, 0, 0};
  if (!gen.first()) return;  // uniform over the warp
  TileItem cur = gen.item();
  grid_tile_async(grid, g, G, cur.tile, sg[0]);
  bool v1 = gen.next();
  TileItem nx1 = v1 ? gen.item() : TileItem{0, 0, 0, 0};
  bool v2 = v1 && gen.next();
  TileItem nx2 = v2 ? gen.item() : TileItem{0, 0, 0, 0};
  const int lane = threadIdx.x, gq = lane >> 2, tq = lane & 3;
  MmaStage<SCB, false> st;
  st.load_entries(list, cur, g);
  st.issue(wc, nullptr);
  st.put(sw[0], nullptr, sflag[0], sblob[0]);
  if (v1) {
    st.load_entries(list, nx1, g);
    st.issue(wc, nullptr);
  }
  if (v2) st.load_entries(list, nx2, g);
  unsigned gh[TE][3][2], gl[TE][3][2];
  bool first = true;  // cur is the first round of its tile
  int gbuf = 0, buf = 0;
  while (true) {
    if (first) {
      // this tile's grid (copied while the previous tile ran) into fragments: k-step j
      // holds rows (y, z) = (j, tq), (j, tq + 4) and column x = gq of each component
      cp_async_wait_all();
      __syncwarp();
      const int ty = (cur.tile / g.ntz) % g.nty;
      const float* sgt = sg[gbuf];
#pragma unroll
      for (int j = 0; j < TE; ++j) {
        const bool live = ty * TE + j < g.ycut;  // rows at or above the slip channel's upper wall read as 0
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int c = 0; c < 3; ++c)
            tf32_split(live ? sgt[c * TE * SGX + gq * SGX + j * TE + tq + 4 * h] : 0.f, gh[j][c][h], gl[j][c][h]);
      }
      gbuf ^= 1;
      const int nt = cur.tile + (int)gridDim.x;
      if (nt < ntiles) grid_tile_async(grid, g, G, nt, sg[gbuf]);
    }
    __syncwarp();
    bool v3 = false;
    TileItem nx3{0, 0, 0, 0};
    if (v1) {
      st.put(sw[buf ^ 1], nullptr, sflag[buf ^ 1], sblob[buf ^ 1]);
      if (v2) {
        st.issue(wc, nullptr);
        v3 = gen.next();
        if (v3) {
          nx3 = gen.item();
          st.load_entries(list, nx3, g);
        }
      }
    }
    if (cur.nc > 0) {  // uniform over the warp
      // rows of A: blobs gq and gq + 8; columns (y, z) = (j, tq), (j, tq + 4)
      float ya[TE], yb[TE];
      *reinterpret_cast<float4*>(ya) = *reinterpret_cast<const float4*>(&sw[buf][gq][1][0]);
      *reinterpret_cast<float4*>(ya + 4) = *reinterpret_cast<const float4*>(&sw[buf][gq][1][4]);
      *reinterpret_cast<float4*>(yb) = *reinterpret_cast<const float4*>(&sw[buf][gq + 8][1][0]);
      *reinterpret_cast<float4*>(yb + 4) = *reinterpret_cast<const float4*>(&sw[buf][gq + 8][1][4]);
      const float za0 = sw[buf][gq][2][tq], za1 = sw[buf][gq][2][tq + 4];
      const float zb0 = sw[buf][gq + 8][2][tq], zb1 = sw[buf][gq + 8][2][tq + 4];
      float acc[3][4];
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[c][q] = 0.f;
#pragma unroll
      for (int j = 0; j < TE; ++j) {
        unsigned ah[4], al[4];
        tf32_split(ya[j] * za0, ah[0], al[0]);
        tf32_split(yb[j] * zb0, ah[1], al[1]);
        tf32_split(ya[j] * za1, ah[2], al[2]);
        tf32_split(yb[j] * zb1, ah[3], al[3]);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          mma_3xtf32(acc[c], ah, al, gh[j][c][0], gh[j][c][1], gl[j][c][0], gl[j][c][1]);
      }
      // contract x: lane (gq, tq) holds x = 2tq, 2tq + 1 of blobs gq (c0, c1) and gq + 8 (c2, c3)
      const float2 wa = *reinterpret_cast<const float2*>(&sw[buf][gq][0][2 * tq]);
      const float2 wb = *reinterpret_cast<const float2*>(&sw[buf][gq + 8][0][2 * tq]);
      float pa[3], pb[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        pa[c] = acc[c][0] * wa.x + acc[c][1] * wa.y;
        pb[c] = acc[c][2] * wb.x + acc[c][3] * wb.y;
        pa[c] += __shfl_xor_sync(0xffffffffu, pa[c], 1);
        pb[c] += __shfl_xor_sync(0xffffffffu, pb[c], 1);
        pa[c] += __shfl_xor_sync(0xffffffffu, pa[c], 2);
        pb[c] += __shfl_xor_sync(0xffffffffu, pb[c], 2);
      }
      if (tq < 2) {  // lane tq = 0 writes blob gq, lane tq = 1 blob gq + 8
        const int k = gq + 8 * tq;
        const unsigned fl = sflag[buf][k];
        if (k < cur.nc && ((fl >> EXM) & 63u) != 0u) {
          const unsigned jt = (fl >> EJ) & 63u;
          if (FCM_INB((long long)sblob[buf][k] * 64 + jt, (long long)g.nblobs * 64, BS_PARTIAL)) {
            float* out = partial + ((size_t)sblob[buf][k] * 64 + jt) * 3;
            out[0] = tq ? pb[0] : pa[0];
            out[1] = tq ? pb[1] : pa[1];
            out[2] = tq ? pb[2] : pa[2];
          }
        }
      }
    }
    first = cur.last != 0;
    if (!v1) break;
    cur = nx1;
    nx1 = nx2;
    v1 = v2;
    nx2 = nx3;
    v2 = v3;
    buf ^= 1;
  }
  cp_async_wait_all();  // no copy outlives the kernel
}


// V = DX^3 * sum over the blob's tiles (in canonical order j) of the partials.
template <typename T>
__device__ __forceinline__ void interp_reduce_one(const int* __restrict__ base, const T* __restrict__ partial,
                                                  const TileGeom& g, double dx3, double* __restrict__ V, int b) {
  int f[3], cnt[3];
  blob_tiles(base, b, g, f, cnt);
  int nj = cnt[0] * cnt[1] * cnt[2];
  if (!FCM_INB(nj - 1, 64, BS_PARTIAL)) nj = 0;
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

template <typename T>
__global__ void k_interp_reduce(const int* __restrict__ base, const T* __restrict__ partial, int n, TileGeom g,
                                double dx3, double* __restrict__ V) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  interp_reduce_one<T>(base, partial, g, dx3, V, b);
}

// The same sums with eight lanes per blob: lane k adds the partials j = k, k + 8,
// ... (consecutive lanes read consecutive partials, so the loads coalesce), then
// the eight lanes combine in a fixed butterfly.  Deterministic; 16 blobs per
// 128-thread CTA.
template <typename T>
__global__ void __launch_bounds__(128) k_interp_reduce8(const int* __restrict__ base, const T* __restrict__ partial,
                                                        int n, TileGeom g, double dx3, double* __restrict__ V) {
  const int b = blockIdx.x * 16 + (threadIdx.x >> 3), k = threadIdx.x & 7;
  double s0 = 0, s1 = 0, s2 = 0;
  if (b < n) {
    int f[3], cnt[3];
    blob_tiles(base, b, g, f, cnt);
    int nj = cnt[0] * cnt[1] * cnt[2];
    if (!FCM_INB(nj - 1, 64, BS_PARTIAL)) nj = 0;
    const T* p = partial + (size_t)b * 64 * 3;
    for (int j = k; j < nj; j += 8) {
      s0 += (double)p[3 * j];
      s1 += (double)p[3 * j + 1];
      s2 += (double)p[3 * j + 2];
    }
  }
#pragma unroll
  for (int off = 4; off >= 1; off >>= 1) {  // groups of eight lanes, aligned in the warp
    s0 += __shfl_xor_sync(0xffffffffu, s0, off);
    s1 += __shfl_xor_sync(0xffffffffu, s1, off);
    s2 += __shfl_xor_sync(0xffffffffu, s2, off);
  }
  if (b < n && k == 0) {
    V[3 * b] = s0 * dx3;
    V[3 * b + 1] = s1 * dx3;
    V[3 * b + 2] = s2 * dx3;
  }
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
      if (!FCM_INB(idx, G, BS_GRID)) continue;
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
                                                     long long G, double dx3, double* __restrict__ V, int ycut) {
  const int np = blockIdx.x;
  const int bx = base[3 * np], by = base[3 * np + 1], bz = base[3 * np + 2];
  const T* gx = w + (size_t)(3 * np) * W;
  const T* gy = gx + W;
  const T* gz = gy + W;
  T s0 = 0, s1 = 0, s2 = 0;
  for (int jk = threadIdx.x; jk < W * W; jk += NT) {
    const int j = jk / W, k = jk - j * W;
    const int yy = wrap_index(by + j, ny), zz = wrap_index(bz + k, nz);
    if (yy >= ycut) continue;  // Gaussians truncated at the slip channel's upper wall
    const T wyz = gy[j] * gz[k];
    for (int i = 0; i < W; ++i) {
      const int xx = wrap_index(bx + i, nx);
      const T wt = gx[i] * wyz;
      const long long idx = ((long long)xx * ny + yy) * nz + zz;
      if (!FCM_INB(idx, G, BS_GRID)) continue;
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

}  // namespace

TileGeom tile_geom(const GridDims& g, int W, int nblobs, long long list_cap) {
  return TileGeom{g.nx / TE, g.ny / TE, g.nz / TE, g.nx, g.ny, g.nz, W, g.ny, nblobs, list_cap};
}

// CTAs of a persistent kernel: as many as fit on the device at once
// (resident CTAs per SM x SMs), looked up once per kernel and device (keyed by
// the kernel's address: kernels of one signature share this instantiation).
template <typename K>
int persistent_ctas(K kernel, int threads, int device) {
  static std::mutex mtx;
  static std::map<std::pair<const void*, int>, int> cache;
  std::lock_guard<std::mutex> lock(mtx);
  const int dev = (device >= 0 && device < 64) ? device : 0;
  int& n = cache[{reinterpret_cast<const void*>(kernel), dev}];
  if (!n) {
    int per_sm = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, 0) != cudaSuccess || per_sm < 1)
      per_sm = 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
    cudaGetLastError();
    n = per_sm * sms;
  }
  return n;
}

template <typename T>
int blob_table_alloc(BlobTable<T>& t, int n, int W, const GridDims& g) {
  if (t.n == n && t.W == W && t.base) return FCM_OK;
  blob_table_free(t);
  t.n = n;
  t.W = W;
  FCM_CUDA(cudaMalloc(&t.base, sizeof(int) * 3 * (size_t)(n > 0 ? n : 1)));
  FCM_CUDA(cudaMalloc(&t.w, sizeof(T) * 3 * (size_t)W * (n > 0 ? n : 1)));
  FCM_CUDA(cudaMalloc(&t.ypos, sizeof(double) * 3 * (size_t)(n > 0 ? n : 1)));
  const bool ok = g.nx % TE == 0 && g.ny % TE == 0 && g.nz % TE == 0 && W + TE <= g.nx && W + TE <= g.ny &&
                  W + TE <= g.nz && W <= MAXW && n < (1 << 30);
  if (ok) {
    t.tiled = true;
    t.ntx = g.nx / TE;
    t.nty = g.ny / TE;
    t.ntz = g.nz / TE;
    t.ntiles = t.ntx * t.nty * t.ntz;
    const long long per = (long long)((W + TE - 2) / TE + 1);
    t.tile_cap = (long long)(n > 0 ? n : 1) * per * per * per;
    FCM_CUDA(cudaMalloc(&t.wc, sizeof(T) * 3 * NCH * TE * (size_t)(n > 0 ? n : 1)));
    FCM_CUDA(cudaMalloc(&t.tile_count, sizeof(int) * (size_t)t.ntiles));
    FCM_CUDA(cudaMalloc(&t.tile_offset, sizeof(int) * ((size_t)t.ntiles + 1)));
    FCM_CUDA(cudaMalloc(&t.tile_cursor, sizeof(int) * (size_t)t.ntiles));
    FCM_CUDA(cudaMalloc(&t.tile_list, sizeof(unsigned long long) * (size_t)t.tile_cap));
    FCM_CUDA(cudaMalloc(&t.partial, sizeof(T) * 64 * 3 * (size_t)(n > 0 ? n : 1)));
  }
  return FCM_OK;
}

template <typename T>
void blob_table_free(BlobTable<T>& t) {
  cudaFree(t.base);
  cudaFree(t.w);
  cudaFree(t.wc);
  cudaFree(t.ypos);
  cudaFree(t.wd);
  cudaFree(t.hd);
  cudaFree(t.partial9);
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
  k_set_up_gaussians_warp<T><<<(unsigned)((32LL * nt + 127) / 128), 128, 0, s>>>(dY, t.n, t.W, c.g.dx, anorm, anorm2,
                                                                               t.base, t.w,
                                                          t.tiled ? t.wc : nullptr, t.ypos);
  FCM_LAUNCH_CHECK();
  if (t.tiled) {
    const TileGeom g = tile_geom(c.g, t);
    FCM_CUDA(cudaMemsetAsync(t.tile_count, 0, sizeof(int) * (size_t)t.ntiles, s));
    FCM_CUDA(cudaMemsetAsync(t.tile_cursor, 0, sizeof(int) * (size_t)t.ntiles, s));
    k_tile_count<<<(t.n + 127) / 128, 128, 0, s>>>(t.base, t.n, g, t.tile_count);
    FCM_LAUNCH_CHECK();
    FCM_TRY(launch_exclusive_scan(t.tile_count, t.tile_offset, t.ntiles, s));
    k_tile_fill<<<(t.n + 127) / 128, 128, 0, s>>>(t.base, t.n, g, t.tile_offset, t.tile_cursor, t.tile_list);
    FCM_LAUNCH_CHECK();
    k_tile_sort_warp<<<(t.ntiles + 3) / 4, 128, 0, s>>>(t.tile_offset, t.ntiles, t.tile_list, t.tile_cap);
    FCM_LAUNCH_CHECK();
  }
  return FCM_OK;
}

template <typename T>
int launch_spread(const Ctx& c, const BlobTable<T>& t, const double* dF, T* grid, cudaStream_t s) {
  if (t.tiled) {
    // by default FP64 takes the persistent pipelined kernel (its staging latency is
    // the limit), FP32 one CTA per tile staging 16 blobs per round; fcm_autotune may
    // choose another (one CTA per tile with 8 or 32 blobs per round)
    const int v = c.spread_variant[sizeof(T) == 8 ? 0 : 1];
    const TileGeom tg = tile_geom(c.g, t);
    if (v == 0) {
      const int ctas = std::min(t.ntiles, persistent_ctas(k_spread_pipe<T>, 64, c.device));
      k_spread_pipe<T><<<ctas, 64, 0, s>>>(t.wc, dF, tg, t.tile_offset, t.tile_list, c.g.G, grid, t.ntiles);
    } else if (v == 2) {
      k_spread_tiled<T, 8><<<t.ntiles, 64, 0, s>>>(t.wc, dF, tg, t.tile_offset, t.tile_list, c.g.G, grid);
    } else if (v == 3) {
      k_spread_tiled<T, 32><<<t.ntiles, 64, 0, s>>>(t.wc, dF, tg, t.tile_offset, t.tile_list, c.g.G, grid);
    } else if (v == 4) {
      k_spread_warp<T><<<t.ntiles, 32, 0, s>>>(t.wc, dF, tg, t.tile_offset, t.tile_list, c.g.G, grid);
    } else if (v == 5 && sizeof(T) == 4) {
      if constexpr (sizeof(T) == 4)
        k_spread_mma<<<t.ntiles, 32, 0, s>>>(t.wc, dF, tg, t.tile_offset, t.tile_list, c.g.G, grid);
    } else {
      k_spread_tiled<T, 16><<<t.ntiles, 64, 0, s>>>(t.wc, dF, tg, t.tile_offset, t.tile_list, c.g.G, grid);
    }
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
  const int ycut = c.p.slip_channel ? c.g.ny / 2 : c.g.ny;  // fcm_fluid_solver.cpp:387-389
  if (t.tiled) {
    TileGeom g = tile_geom(c.g, t);
    g.ycut = ycut;
    const int v = c.interp_variant[sizeof(T) == 8 ? 0 : 1];
    if constexpr (sizeof(T) == 4) {
      // the tensor-core kernel copies 16-byte rows of the grid asynchronously
      if (v == 3 && (reinterpret_cast<uintptr_t>(grid) & 15u) == 0) {
        k_interp_mma<<<std::min(t.ntiles, persistent_ctas(k_interp_mma, 32, c.device)), 32, 0, s>>>(
            t.wc, grid, g, t.tile_offset, t.tile_list, c.g.G, t.partial, t.ntiles);
        FCM_LAUNCH_CHECK();
        k_interp_reduce8<T><<<(t.n + 15) / 16, 128, 0, s>>>(t.base, t.partial, t.n, g, dx3, dV);
        FCM_LAUNCH_CHECK();
        return FCM_OK;
      }
    }
    if (v == 2)
      k_interp_rows<T, 2><<<t.ntiles, 32, 0, s>>>(t.wc, grid, g, t.tile_offset, t.tile_list, c.g.G, t.partial);
    else if (v == 1)
      k_interp_warp<T><<<t.ntiles, 32, 0, s>>>(t.wc, grid, g, t.tile_offset, t.tile_list, c.g.G, t.partial);
    else
      k_interp_tiled<T><<<t.ntiles, 64, 0, s>>>(t.wc, grid, g, t.tile_offset, t.tile_list, c.g.G, t.partial);
    FCM_LAUNCH_CHECK();
    k_interp_reduce8<T><<<(t.n + 15) / 16, 128, 0, s>>>(t.base, t.partial, t.n, g, dx3, dV);
    FCM_LAUNCH_CHECK();
    return FCM_OK;
  }
  k_interp_block<T, 256><<<t.n, 256, 0, s>>>(t.base, t.w, grid, t.W, c.g.nx, c.g.ny, c.g.nz, c.g.G, dx3, dV, ycut);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// Slip channel (fcm_fluid_solver.cpp:602-632): fy = 0 on the wall rows 0 and ny/2;
// every row j > ny/2 becomes the mirror image of row ny - j (fx, fz copied, fy
// negated).  Rows above ny/2 read rows below it, which this kernel does not write.
template <typename T>
__global__ void k_slip_image(T* __restrict__ grid, int ny, int nz, long long G) {
  const int h = ny / 2;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < G; t += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(t % nz);
    const long long xy = t / nz;
    const int j = (int)(xy % ny);
    if (j == 0 || j == h) {
      grid[G + t] = (T)0;
    } else if (j > h) {
      const long long m = (xy - j + (ny - j)) * nz + k;
      grid[t] = grid[m];
      grid[G + t] = -grid[G + m];
      grid[2 * G + t] = grid[2 * G + m];
    }
  }
}

template <typename T>
int launch_slip_image(const Ctx& c, T* grid, cudaStream_t s) {
  const long long G = c.g.G;
  const long long nb = std::min<long long>((G + 255) / 256, 148LL * 16);
  k_slip_image<T><<<(unsigned)nb, 256, 0, s>>>(grid, c.g.ny, c.g.nz, G);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}
template int launch_slip_image<double>(const Ctx&, double*, cudaStream_t);
template int launch_slip_image<float>(const Ctx&, float*, cudaStream_t);

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

// ------------------------------------------------------------------ force dipoles
// No reference code: the FCM force-dipole terms (Lomholt & Maxey, J. Comput.
// Phys. 184 (2003) 381-405) on the grid conventions above.  Dipole envelope of
// width sigma_D = a / (6 sqrt(pi))^(1/3) on the same stencils and tiles as the
// force envelope; per (blob, dimension) the chunk tables hold
// gD = exp(-xx^2 / (2 sigma_D^2)) / (sqrt(2 pi) sigma_D) and hD = gD xx / sigma_D^2
// (xx = x - Y).  A blob dipole D_ij = S_ij - 1/2 eps_ijk T_k adds
// f_i = D_ij (x_j - Y_j) / sigma_D^2 Delta_D to the force grid; the velocity
// moments M_kj = DX^3 sum u_k (x_j - Y_j) / sigma_D^2 Delta_D give
// Omega_i = 1/2 eps_ijk M_kj and E_ij = (M_ij + M_ji) / 2.
namespace {

template <typename T>
__global__ void k_set_up_dipoles(const double* __restrict__ ypos, const int* __restrict__ base, int n, int W,
                                 double dx, double anorm, double anorm2, double inv_s2, T* __restrict__ wd,
                                 T* __restrict__ hd) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= 3 * n) return;
  const double y = ypos[t];
  const int b = base[t];
  const int c0 = floordiv(b, TE) * TE;
  T* g = wd + (size_t)t * NCH * TE;
  T* h = hd + (size_t)t * NCH * TE;
  for (int i = 0; i < NCH * TE; ++i) {
    const int s = c0 + i - b;
    if (s >= 0 && s < W) {
      const double xx = __dsub_rn(__dmul_rn((double)(c0 + i), dx), y);
      const double e = anorm * exp(__ddiv_rn(-__dmul_rn(xx, xx), anorm2));
      g[i] = (T)e;
      h[i] = (T)(e * xx * inv_s2);
    } else {
      g[i] = (T)0;
      h[i] = (T)0;
    }
  }
}

__global__ void k_blob_dipoles(const double* __restrict__ T3, const double* __restrict__ S9, int n,
                               double* __restrict__ D9) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  double D[9];
  for (int v = 0; v < 9; ++v) D[v] = S9 ? S9[9 * (size_t)b + v] : 0.0;
  if (T3) {
    const double t0 = T3[3 * (size_t)b], t1 = T3[3 * (size_t)b + 1], t2 = T3[3 * (size_t)b + 2];
    D[1] += -0.5 * t2;  // D_01
    D[3] += 0.5 * t2;   // D_10
    D[2] += 0.5 * t1;   // D_02
    D[6] += -0.5 * t1;  // D_20
    D[5] += -0.5 * t0;  // D_12
    D[7] += 0.5 * t0;   // D_21
  }
  for (int v = 0; v < 9; ++v) D9[9 * (size_t)b + v] = D[v];
}

// Stage the dipole chunks of blobs list[c0 .. c0+nc): lane (k, d) copies the
// envelope and derivative chunks of dimension d < 3; lane d = 3 the entry's
// low word, the blob id and, when D9 is given, the blob's dipole.
template <typename T>
__device__ __forceinline__ void stage_dipoles(const unsigned long long* __restrict__ list, int c0, int nc,
                                              const T* __restrict__ wd, const T* __restrict__ hd,
                                              const double* __restrict__ D9, T (*sg)[3][TE], T (*sh)[3][TE],
                                              T (*sD)[9], unsigned* sflag, unsigned* sblob, const TileGeom& g) {
  const int k = threadIdx.x >> 2, d = threadIdx.x & 3;
  if (k >= nc) return;
  const unsigned long long e = list_entry(list, c0 + k, g);
  const unsigned b = (unsigned)(e >> 32), lo = (unsigned)e;
  if (d < 3) {
    const size_t off = ((size_t)(3 * b + d) * NCH + ((lo >> (2 * d)) & 3u)) * TE;
    copy8(sg[k][d], wd + off);
    copy8(sh[k][d], hd + off);
  } else {
    sflag[k] = lo;
    sblob[k] = b;
    if (D9)
      for (int v = 0; v < 9; ++v) sD[k][v] = (T)D9[9 * (size_t)b + v];
  }
}

// Adds the dipole force density of the tile's blobs to its points (each CTA
// owns its tile, so no atomics; tiles without blobs are untouched).
template <typename T>
__global__ void __launch_bounds__(64) k_spread_dipole_tiled(const T* __restrict__ wd, const T* __restrict__ hd,
                                                            const double* __restrict__ D9, TileGeom g,
                                                            const int* __restrict__ offset,
                                                            const unsigned long long* __restrict__ list, long long G,
                                                            T* __restrict__ grid) {
  __shared__ __align__(16) T sg[SCB][3][TE];
  __shared__ __align__(16) T sh[SCB][3][TE];
  __shared__ T sD[SCB][9];
  __shared__ unsigned sflag[SCB], sblob[SCB];
  const int tile = blockIdx.x;
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  if (b0 == b1) return;
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int t = threadIdx.x;
  const int z = t & 7, y = t >> 3, yh = t >> 5;
  T acc[TE][3];
#pragma unroll
  for (int x = 0; x < TE; ++x)
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[x][c] = 0;
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncthreads();
    stage_dipoles<T>(list, c0, nc, wd, hd, D9, sg, sh, sD, sflag, sblob, g);
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
      const unsigned fl = sflag[k];
      if (!((fl >> (EYM + yh)) & 1u)) continue;
      const T gy = sg[k][1][y], hy = sh[k][1][y], gz = sg[k][2][z], hz = sh[k][2][z];
      const T gyz = gy * gz, hygz = hy * gz, gyhz = gy * hz;
      T ca[3], cb[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        ca[c] = sD[k][3 * c] * gyz;                             // times hD_x
        cb[c] = sD[k][3 * c + 1] * hygz + sD[k][3 * c + 2] * gyhz;  // times gD_x
      }
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        if (skip_x_half<T>(fl, h)) continue;
        T wg[4], wh[4];
        load_wx4<T>(sg[k][0], 4 * h, wg);
        load_wx4<T>(sh[k][0], 4 * h, wh);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int c = 0; c < 3; ++c) acc[4 * h + i][c] += ca[c] * wh[i] + cb[c] * wg[i];
      }
    }
  }
  const int ox = tx * TE, oy = ty * TE + y, oz = tz * TE + z;
#pragma unroll
  for (int x = 0; x < TE; ++x) {
    const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
    if (!FCM_INB(idx, G, BS_GRID)) continue;
    grid[idx] += acc[x][0];
    grid[G + idx] += acc[x][1];
    grid[2 * G + idx] += acc[x][2];
  }
}

// Per-(blob, tile) velocity moments M_kj (9 values) into partial9[blob][j][9].
template <typename T>
__global__ void __launch_bounds__(64) k_interp_dipole_tiled(const T* __restrict__ wd, const T* __restrict__ hd,
                                                            const T* __restrict__ grid, TileGeom g,
                                                            const int* __restrict__ offset,
                                                            const unsigned long long* __restrict__ list, long long G,
                                                            T* __restrict__ partial9) {
  __shared__ __align__(16) T sg[SCB][3][TE];
  __shared__ __align__(16) T sh[SCB][3][TE];
  __shared__ unsigned sflag[SCB], sblob[SCB];
  __shared__ T sred[SCB][2][16];
  const int tile = blockIdx.x;
  int b0, b1;
  tile_range(offset, tile, g, b0, b1);
  if (b0 == b1) return;
  const int tz = tile % g.ntz, ty = (tile / g.ntz) % g.nty, tx = tile / (g.ntz * g.nty);
  const int t = threadIdx.x;
  const int z = t & 7, y = t >> 3, yh = t >> 5, lane = t & 31;
  T u[TE][3];
  {
    const int ox = tx * TE, oy = ty * TE + y, oz = tz * TE + z;
    const bool live = oy < g.ycut;  // rows at or above the slip channel's upper wall read as 0
#pragma unroll
    for (int x = 0; x < TE; ++x) {
      const long long idx = ((long long)(ox + x) * g.ny + oy) * g.nz + oz;
      if (!FCM_INB(idx, G, BS_GRID)) {
        u[x][0] = u[x][1] = u[x][2] = (T)0;
        continue;
      }
      u[x][0] = live ? grid[idx] : (T)0;
      u[x][1] = live ? grid[G + idx] : (T)0;
      u[x][2] = live ? grid[2 * G + idx] : (T)0;
    }
  }
  for (int c0 = b0; c0 < b1; c0 += SCB) {
    const int nc = min(SCB, b1 - c0);
    if (c0 != b0) __syncthreads();
    stage_dipoles<T>(list, c0, nc, wd, hd, nullptr, sg, sh, nullptr, sflag, sblob, g);
    __syncthreads();
    for (int k = 0; k < nc; ++k) {
      const unsigned fl = sflag[k];
      T v[16];
#pragma unroll
      for (int i = 0; i < 16; ++i) v[i] = 0;
      if ((fl >> (EYM + yh)) & 1u) {
        T sx[3] = {0, 0, 0}, tx3[3] = {0, 0, 0};
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          if (skip_x_half<T>(fl, h)) continue;
          T wg[4], wh[4];
          load_wx4<T>(sg[k][0], 4 * h, wg);
          load_wx4<T>(sh[k][0], 4 * h, wh);
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              sx[c] += u[4 * h + i][c] * wh[i];
              tx3[c] += u[4 * h + i][c] * wg[i];
            }
        }
        const T gy = sg[k][1][y], hy = sh[k][1][y], gz = sg[k][2][z], hz = sh[k][2][z];
        const T gyz = gy * gz, hygz = hy * gz, gyhz = gy * hz;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          v[3 * c] = sx[c] * gyz;
          v[3 * c + 1] = tx3[c] * hygz;
          v[3 * c + 2] = tx3[c] * gyhz;
        }
      }
      const T r = warp_reduce_scatter16<T>(v, lane);
      if (!(lane & 1)) sred[k][yh][lane >> 1] = r;
    }
    __syncthreads();
    for (int e = t; e < nc * 9; e += 64) {
      const int k = e / 9, vv = e - 9 * k;
      const unsigned jt = (sflag[k] >> EJ) & 63u;
      if (FCM_INB((long long)sblob[k] * 64 + jt, (long long)g.nblobs * 64, BS_PARTIAL))
        partial9[((size_t)sblob[k] * 64 + jt) * 9 + vv] = sred[k][0][vv] + sred[k][1][vv];
    }
  }
}

template <typename T>
__global__ void k_interp_dipole_reduce(const int* __restrict__ base, const T* __restrict__ partial9, int n,
                                       TileGeom g, double dx3, double* __restrict__ Om, double* __restrict__ E) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= n) return;
  int f[3], cnt[3];
  blob_tiles(base, b, g, f, cnt);
  int nj = cnt[0] * cnt[1] * cnt[2];
  if (!FCM_INB(nj - 1, 64, BS_PARTIAL)) nj = 0;
  double M[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const T* p = partial9 + (size_t)b * 64 * 9;
  for (int j = 0; j < nj; ++j)
    for (int v = 0; v < 9; ++v) M[v] += (double)p[9 * j + v];
  for (int v = 0; v < 9; ++v) M[v] *= dx3;
  if (Om) {
    Om[3 * (size_t)b] = 0.5 * (M[7] - M[5]);
    Om[3 * (size_t)b + 1] = 0.5 * (M[2] - M[6]);
    Om[3 * (size_t)b + 2] = 0.5 * (M[3] - M[1]);
  }
  if (E)
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) E[9 * (size_t)b + 3 * a + c] = 0.5 * (M[3 * a + c] + M[3 * c + a]);
}

template <typename T>
int ensure_dipole_tables(const Ctx& c, BlobTable<T>& t, cudaStream_t s) {
  if (!t.tiled) {
    set_error("force dipoles need a grid the tiled kernels take (dimensions multiples of 8, at least ngauss + 8, "
              "ngauss <= 25)");
    return FCM_ERR_INVALID;
  }
  const size_t nn = (size_t)(t.n > 0 ? t.n : 1);
  if (!t.wd) FCM_CUDA(cudaMalloc(&t.wd, sizeof(T) * 3 * NCH * TE * nn));
  if (!t.hd) FCM_CUDA(cudaMalloc(&t.hd, sizeof(T) * 3 * NCH * TE * nn));
  if (!t.partial9) FCM_CUDA(cudaMalloc(&t.partial9, sizeof(T) * 64 * 9 * nn));
  if (t.n == 0) return FCM_OK;
  const double PI = 3.14159265358979323846264338327950288;
  const double a = c.p.blob_radius;
  const double sD = a / cbrt(6.0 * sqrt(PI));
  const double anorm = 1.0 / (sqrt(2.0 * PI) * sD);
  const double anorm2 = 2.0 * sD * sD;
  k_set_up_dipoles<T><<<(3 * t.n + 127) / 128, 128, 0, s>>>(t.ypos, t.base, t.n, t.W, c.g.dx, anorm, anorm2,
                                                          1.0 / (sD * sD), t.wd, t.hd);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

}  // namespace

int launch_blob_dipoles(const double* T3, const double* S9, int n, double* D9, cudaStream_t s) {
  if (n == 0) return FCM_OK;
  k_blob_dipoles<<<(n + 127) / 128, 128, 0, s>>>(T3, S9, n, D9);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template <typename T>
int launch_spread_dipoles(const Ctx& c, BlobTable<T>& t, const double* dD, T* grid, cudaStream_t s) {
  FCM_TRY(ensure_dipole_tables<T>(c, t, s));
  if (t.n == 0) return FCM_OK;
  k_spread_dipole_tiled<T><<<t.ntiles, 64, 0, s>>>(t.wd, t.hd, dD, tile_geom(c.g, t), t.tile_offset, t.tile_list,
                                                   c.g.G, grid);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template <typename T>
int launch_interp_dipoles(const Ctx& c, BlobTable<T>& t, const T* grid, double* dOm, double* dE, cudaStream_t s) {
  FCM_TRY(ensure_dipole_tables<T>(c, t, s));
  if (t.n == 0) return FCM_OK;
  const TileGeom g = tile_geom(c.g, t);
  k_interp_dipole_tiled<T><<<t.ntiles, 64, 0, s>>>(t.wd, t.hd, grid, g, t.tile_offset, t.tile_list, c.g.G,
                                                   t.partial9);
  FCM_LAUNCH_CHECK();
  k_interp_dipole_reduce<T><<<(t.n + 127) / 128, 128, 0, s>>>(t.base, t.partial9, t.n, g,
                                                              c.g.dx * c.g.dx * c.g.dx, dOm, dE);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template int launch_spread_dipoles<double>(const Ctx&, BlobTable<double>&, const double*, double*, cudaStream_t);
template int launch_spread_dipoles<float>(const Ctx&, BlobTable<float>&, const double*, float*, cudaStream_t);
template int launch_interp_dipoles<double>(const Ctx&, BlobTable<double>&, const double*, double*, double*,
                                           cudaStream_t);
template int launch_interp_dipoles<float>(const Ctx&, BlobTable<float>&, const float*, double*, double*,
                                          cudaStream_t);

// ------------------------------------------------------------------ batched
// One launch over the tiles of every member: tile_map[blockIdx.x] = (member,
// tile).  P selects the member's grid of that precision (0 FP64, 1 FP32).
namespace {

template <typename T, int P>
__global__ void __launch_bounds__(64) k_b_spread(const BMember* __restrict__ mem, const int2* __restrict__ tile_map,
                                                 int in, int mask) {
  const int2 mt = tile_map[blockIdx.x];
  const BMember& m = mem[mt.x];
  if (bskip(m, mask)) return;
  spread_tile<T>((const T*)m.wc[P], bvec(m, in), m.tg[P], m.toff[P], m.tlist[P],
                 (long long)m.tg[P].nx * m.tg[P].ny * m.tg[P].nz,
                 (T*)m.grid[P], mt.y);
}

template <typename T, int P>
__global__ void __launch_bounds__(64) k_b_interp(const BMember* __restrict__ mem, const int2* __restrict__ tile_map,
                                                 int mask) {
  const int2 mt = tile_map[blockIdx.x];
  const BMember& m = mem[mt.x];
  if (bskip(m, mask)) return;
  interp_tile<T>((const T*)m.wc[P], (const T*)m.grid[P], m.tg[P], m.toff[P], m.tlist[P],
                 (long long)m.tg[P].nx * m.tg[P].ny * m.tg[P].nz, (T*)m.partial[P], mt.y);
}

template <typename T, int P>
__global__ void k_b_interp_reduce(const BMember* __restrict__ mem, int out, int mask) {
  const BMember& m = mem[blockIdx.y];
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= m.Nb || bskip(m, mask)) return;
  interp_reduce_one<T>(m.base[P], (const T*)m.partial[P], m.tg[P], m.dx3, bvec(m, out), b);
}

}  // namespace

template <typename T>
int b_spread(const BatchGeom& b, int in, int mask, cudaStream_t s) {
  constexpr int P = sizeof(T) == 8 ? 0 : 1;
  k_b_spread<T, P><<<b.total_tiles, 64, 0, s>>>(b.mem, b.tile_map, in, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template <typename T>
int b_interp(const BatchGeom& b, int out, int mask, cudaStream_t s) {
  constexpr int P = sizeof(T) == 8 ? 0 : 1;
  k_b_interp<T, P><<<b.total_tiles, 64, 0, s>>>(b.mem, b.tile_map, mask);
  FCM_LAUNCH_CHECK();
  k_b_interp_reduce<T, P><<<dim3(b.max_blob_blocks, b.n), 128, 0, s>>>(b.mem, out, mask);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

template int b_spread<double>(const BatchGeom&, int, int, cudaStream_t);
template int b_spread<float>(const BatchGeom&, int, int, cudaStream_t);
template int b_interp<double>(const BatchGeom&, int, int, cudaStream_t);
template int b_interp<float>(const BatchGeom&, int, int, cudaStream_t);

FCM_BOUNDS_READER(bounds_read_grid)

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
constexpr size_t NA_SCRATCH_BYTES = (size_t)32 << 20;  // 32 MiB

static __device__ __align__(256) unsigned char g_noalloc_scratch[NA_SCRATCH_BYTES];

inline size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of g_noalloc_scratch on the current device, looked up once per
// device (the name is only a host-side stand-in in host code).  The address is
// kept for the life of the process: cudaDeviceReset unloads the library's device
// code, and the array may come back elsewhere, so the call is not to be used
// after a cudaDeviceReset in the same process.
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

// Device memory of the current device (where the kernels run) or managed memory.
// A device pointer of another GPU is refused: a kernel here would read or write
// that GPU's memory (an illegal address, or silent peer traffic).
bool on_device(const void* p) {
  cudaPointerAttributes a;
  if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (a.type == cudaMemoryTypeManaged) return true;
  int dev = -1;
  if (a.type != cudaMemoryTypeDevice || cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.device == dev;
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
    set_error("fcm_interp_noalloc: Y, grid and V must be device pointers of the current device");
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
  double* s_wc = (double*)p;
  p += round256(sizeof(double) * 3 * NCH * TE * (size_t)n);
  int* s_count = (int*)p;
  p += round256(sizeof(int) * (size_t)ntiles);
  int* s_offset = (int*)p;
  p += round256(sizeof(int) * ((size_t)ntiles + 1));
  int* s_cursor = (int*)p;
  p += round256(sizeof(int) * (size_t)ntiles);
  unsigned long long* s_list = (unsigned long long*)p;
  p += round256(sizeof(unsigned long long) * cap);
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
  const TileGeom g{nx / TE, ny / TE, nz / TE, nx, ny, nz, W, ny, n, (long long)cap};
  const long long G = (long long)nx * ny * nz;
  // the array keeps the previous call's contents: counters start at zero
  FCM_CUDA(cudaMemsetAsync(s_count, 0, sizeof(int) * (size_t)ntiles, s));
  FCM_CUDA(cudaMemsetAsync(s_cursor, 0, sizeof(int) * (size_t)ntiles, s));
  k_set_up_gaussians<double><<<(3 * n + 127) / 128, 128, 0, s>>>(Y, n, W, dx, anorm, anorm2, s_base, s_w, s_wc,
                                                                 nullptr);
  FCM_LAUNCH_CHECK();
  k_tile_count<<<(n + 127) / 128, 128, 0, s>>>(s_base, n, g, s_count);
  FCM_LAUNCH_CHECK();
  FCM_TRY(launch_exclusive_scan(s_count, s_offset, (int)ntiles, s));
  k_tile_fill<<<(n + 127) / 128, 128, 0, s>>>(s_base, n, g, s_offset, s_cursor, s_list);
  FCM_LAUNCH_CHECK();
  k_tile_sort<<<(unsigned)((ntiles + 127) / 128), 128, 0, s>>>(s_offset, (int)ntiles, s_list, (long long)cap);
  FCM_LAUNCH_CHECK();
  k_interp_tiled<double><<<(unsigned)ntiles, 64, 0, s>>>(s_wc, grid, g, s_offset, s_list, G, s_partial);
  FCM_LAUNCH_CHECK();
  k_interp_reduce<double><<<(n + 127) / 128, 128, 0, s>>>(s_base, s_partial, n, g, dx * dx * dx, V);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}
