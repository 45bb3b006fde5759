// fcm_cells.cu -- cell list and steric pair forces (linked_list.cpp).
//
// The reference keeps head/next linked lists over NUM_LINKED_LIST_CELLS_PER_DIM^3
// cells and, for each blob, visits the later blobs of its own cell and all blobs
// of 13 half-shell neighbour cells (linked_list.cpp:23-72, :192-281).  For
// ncells >= 3 those two sets together are exactly the unordered pairs of blobs
// whose cells are equal or adjacent (26-neighbourhood, periodic).  Here the list
// is a counting sort (cell start offsets + blob ids sorted within each cell) and
// each blob gathers over its 27 cells, so no atomics touch the forces and the
// pair set is the reference's.  Cell ids use the reference's arithmetic
// floor(N*(Y/L)) per dimension (linked_list.cpp:74-78) without FMA contraction.
#include "fcm_internal.cuh"

namespace fcm {

namespace {

struct CellGeom {
  int N;
  double Lx, Ly, Lz;
};

__device__ __forceinline__ int cell_coord(double y, double L, int N) {
  int c = (int)floor(__dmul_rn((double)N, __ddiv_rn(y, L)));
  // y == L can occur after the periodic wrap rounds up; the reference would
  // index one past its table there, the library wraps it to cell 0.
  if (c >= N) c -= N;
  if (c < 0) c += N;
  return c;
}

__global__ void k_cell_ids(const double* __restrict__ Y, int Nb, CellGeom g, int* __restrict__ cell,
                           int* __restrict__ count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  const int cx = cell_coord(Y[3 * i], g.Lx, g.N);
  const int cy = cell_coord(Y[3 * i + 1], g.Ly, g.N);
  const int cz = cell_coord(Y[3 * i + 2], g.Lz, g.N);
  const int id = cx + cy * g.N + cz * g.N * g.N;
  cell[i] = id;
  if (FCM_INB(id, (long long)g.N * g.N * g.N, BS_CELL)) atomicAdd(count + id, 1);
}

// Single-CTA exclusive scan of n ints (n up to a few million).
// Exclusive prefix sum of in[0..n) into out[0..n], out[n] = total, by one CTA:
// each pass covers blockDim.x * 8 entries, every thread summing eight
// consecutive ones, the thread totals scanned by warp shuffles and a second
// warp level.
__global__ void k_exclusive_scan(const int* __restrict__ in, int* __restrict__ out, int n) {
  constexpr int IPT = 8;
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int base = 0; base < n; base += blockDim.x * IPT) {
    const int i0 = base + threadIdx.x * IPT;
    int v[IPT], tot = 0;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      v[k] = (i0 + k < n) ? in[i0 + k] : 0;
      tot += v[k];
    }
    int x = tot;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, off);
      if (lane >= off) x += y;
    }
    if (lane == 31) warp_sums[wid] = x;
    __syncthreads();
    if (wid == 0) {
      int s2 = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
      for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, s2, off);
        if (lane >= off) s2 += y;
      }
      warp_sums[lane] = s2;
    }
    __syncthreads();
    int run = carry + ((wid > 0) ? warp_sums[wid - 1] : 0) + x - tot;
#pragma unroll
    for (int k = 0; k < IPT; ++k) {
      if (i0 + k < n) out[i0 + k] = run;
      run += v[k];
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry = run;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

// The same scan over many CTAs, for long inputs: chunks of SCAN_CH = 8192 entries.
// k_scan_chunk_sums writes each chunk's total to out[chunk * SCAN_CH] (the chunk's
// first output slot), k_scan_chunk_offsets turns those totals into exclusive chunk
// offsets in place (one CTA) and writes out[n], k_scan_chunks scans every chunk
// from its offset.  Integer sums: the result is that of k_exclusive_scan.
constexpr int SCAN_T = 1024, SCAN_IPT = 8, SCAN_CH = SCAN_T * SCAN_IPT;

// Block-wide exclusive scan of the thread totals `tot`; returns the thread's
// exclusive prefix within the block and writes the block total to *total.
__device__ __forceinline__ int block_exclusive(int tot, int* warp_sums, int* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = tot;
  for (int off = 1; off < 32; off <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int s2 = (lane < (int)(blockDim.x >> 5)) ? warp_sums[lane] : 0;
    for (int off = 1; off < 32; off <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s2, off);
      if (lane >= off) s2 += y;
    }
    warp_sums[lane] = s2;
  }
  __syncthreads();
  *total = warp_sums[(blockDim.x >> 5) - 1];
  return ((wid > 0) ? warp_sums[wid - 1] : 0) + x - tot;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_chunk_sums(const int* __restrict__ in, int* __restrict__ out,
                                                           int n) {
  __shared__ int warp_sums[32];
  const long long i0 = (long long)blockIdx.x * SCAN_CH + (long long)threadIdx.x * SCAN_IPT;
  int tot = 0;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) tot += (i0 + k < n) ? in[i0 + k] : 0;
  int total = 0;
  block_exclusive(tot, warp_sums, &total);
  if (threadIdx.x == 0) out[(long long)blockIdx.x * SCAN_CH] = total;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_chunk_offsets(int* __restrict__ out, int n, int nchunks) {
  __shared__ int warp_sums[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < nchunks; base += SCAN_T) {
    const int c = base + threadIdx.x;
    const int v = c < nchunks ? out[(long long)c * SCAN_CH] : 0;
    int total = 0;
    const int ex = block_exclusive(v, warp_sums, &total);
    if (c < nchunks) out[(long long)c * SCAN_CH] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += total;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[n] = carry;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_chunks(const int* __restrict__ in, int* __restrict__ out, int n) {
  __shared__ int warp_sums[32];
  __shared__ int offset;
  const long long c0 = (long long)blockIdx.x * SCAN_CH;
  if (threadIdx.x == 0) offset = out[c0];
  __syncthreads();
  const long long i0 = c0 + (long long)threadIdx.x * SCAN_IPT;
  int v[SCAN_IPT], tot = 0;
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    v[k] = (i0 + k < n) ? in[i0 + k] : 0;
    tot += v[k];
  }
  int total = 0;
  int run = offset + block_exclusive(tot, warp_sums, &total);
#pragma unroll
  for (int k = 0; k < SCAN_IPT; ++k) {
    if (i0 + k < n) out[i0 + k] = run;
    run += v[k];
  }
}

__global__ void k_cell_scatter(const int* __restrict__ cell, int Nb, int ncell, const int* __restrict__ start,
                               int* __restrict__ cursor, int* __restrict__ sorted) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  const int c = cell[i];
  if (!FCM_INB(c, ncell, BS_CELL)) return;
  const int slot = start[c] + atomicAdd(cursor + c, 1);
  if (FCM_INB(slot, start[c + 1], BS_LIST) && FCM_INB(slot, Nb, BS_LIST)) sorted[slot] = i;
}

// Ascending blob order within each cell, so every traversal is deterministic.
__global__ void k_cell_sort(const int* __restrict__ start, int ncell, int* __restrict__ sorted) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  const int b = start[c], e = start[c + 1];
  if (!FCM_INB(b, (long long)e + 1, BS_LIST) || !FCM_INB(e, (long long)start[ncell] + 1, BS_LIST)) return;
  for (int i = b + 1; i < e; ++i) {
    const int v = sorted[i];
    int j = i - 1;
    while (j >= b && sorted[j] > v) {
      sorted[j + 1] = sorted[j];
      --j;
    }
    sorted[j + 1] = v;
  }
}

// linked_list.cpp:362-497 (force magnitudes) and the polynomial potential 3.
__device__ __forceinline__ double interaction_magnitude(double r, int type, double a, double kT, double fs,
                                                        double rc) {
  if (type == 3) {
    if (r < rc) {
      const double t = (rc * rc - r * r) / (rc * rc - 4.0 * a * a);
      const double t2 = t * t;
      return fs * t2 * t2;
    }
    return 0.0;
  }
  const double U0 = 20.0 * kT, b = 0.5 * a;
  double mag = (r < 2.0 * a) ? U0 / b : U0 * exp((2.0 * a - r) / b) / b;
  if (type == 1 || type == 2) {
    const double A = 5.0 * kT, lambda = 0.5 * a;
    if (r < 2.0 * a) {
      double temp = a / lambda;
      temp = A * exp(-temp * temp);
      mag += 2.0 * a * temp / (lambda * lambda);
      if (type == 2) {
        temp = 1.5 * a / lambda;
        temp = A * exp(-temp * temp);
        mag -= 3.0 * a * temp / (lambda * lambda);
      }
    } else {
      double temp = (r - 3.0 * a) / lambda;
      mag += -2.0 * A * temp * exp(-temp * temp) / lambda;
      if (type == 2) {
        temp = (r - 3.5 * a) / lambda;
        mag += 2.0 * A * temp * exp(-temp * temp) / lambda;
      }
    }
  }
  return mag;
}

// linked_list.cpp:362-497, the MARKOV_CHAIN_MONTE_CARLO branches (pair
// energies), and for potential 3 the energy whose force is the polynomial
// F_s t^4, t = (rc^2 - r^2)/(rc^2 - 4a^2): U(r) = int_r^rc F ds (zero beyond rc).
__device__ __forceinline__ double interaction_energy(double r, int type, double a, double kT, double fs, double rc) {
  if (type == 3) {
    // the integrand is a degree-8 polynomial: 5-point Gauss-Legendre is exact,
    // and its terms are all positive (no cancellation)
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
    return fs * half * u;
  }
  const double U0 = 20.0 * kT, b = 0.5 * a;
  double e = (r < 2.0 * a) ? U0 + U0 * (2.0 * a - r) / b : U0 * exp((2.0 * a - r) / b);
  if (type == 1 || type == 2) {
    const double A = 5.0 * kT, lambda = 0.5 * a;
    if (r < 2.0 * a) {
      double temp = a / lambda;
      temp = A * exp(-temp * temp);
      e -= temp;
      e += 2.0 * a * (2.0 * a - r) * temp / (lambda * lambda);
      if (type == 2) {
        temp = 1.5 * a / lambda;
        temp = A * exp(-temp * temp);
        e += temp;
        e -= 3.0 * a * (2.0 * a - r) * temp / (lambda * lambda);
      }
    } else {
      double temp = (r - 3.0 * a) / lambda;
      e -= A * exp(-temp * temp);
      if (type == 2) {
        temp = (r - 3.5 * a) / lambda;
        e += A * exp(-temp * temp);
      }
    }
  }
  return e;
}

// Minimum image d - L trunc(2d/L) (linked_list.cpp:253-256).
__device__ __forceinline__ double min_image(double d, double L) {
  return __dsub_rn(d, __dmul_rn(L, trunc(__ddiv_rn(__dmul_rn(2.0, d), L))));
}

struct PairArgs {
  const double* Y;
  const int* cell;
  const int* start;
  const int* sorted;
  int Nb, nb;
  CellGeom g;
};

// Visit every partner j of blob i (other body, same or adjacent cell).
template <class Fn>
__device__ __forceinline__ void visit_partners(const PairArgs& a, int i, Fn fn) {
  const int N = a.g.N;
  const int id = a.cell[i];
  if (!FCM_INB(id, (long long)N * N * N, BS_CELL)) return;
  const int cx = id % N, cy = (id / N) % N, cz = id / (N * N);
  const int body = i / a.nb;
  const double x1 = a.Y[3 * i], y1 = a.Y[3 * i + 1], z1 = a.Y[3 * i + 2];
  for (int dz = -1; dz <= 1; ++dz) {
    const int zz = (cz + dz + N) % N;
    for (int dy = -1; dy <= 1; ++dy) {
      const int yy = (cy + dy + N) % N;
      for (int dx = -1; dx <= 1; ++dx) {
        const int xx = (cx + dx + N) % N;
        const int c = xx + yy * N + zz * N * N;
        const int e = a.start[c + 1];
        for (int s = a.start[c]; s < e; ++s) {
          if (!FCM_INB(s, a.Nb, BS_LIST)) break;
          const int j = a.sorted[s];
          if (!FCM_INB(j, a.Nb, BS_BLOB)) continue;
          if (j == i || j / a.nb == body) continue;
          const double xd = min_image(__dsub_rn(x1, a.Y[3 * j]), a.g.Lx);
          const double yd = min_image(__dsub_rn(y1, a.Y[3 * j + 1]), a.g.Ly);
          const double zd = min_image(__dsub_rn(z1, a.Y[3 * j + 2]), a.g.Lz);
          fn(j, xd, yd, zd);
        }
      }
    }
  }
}

// Slip-channel walls at y = 0 and y = L_y/2 (collection_of_rigid_bodies.cpp:640-662,
// :679-700): within L = 2.2a of a wall a blob feels the spring K (L - d), d its
// distance to the wall, K = 40 kT / (a L), and has the energy K (L - d)^2 / 2.
struct Walls {
  int on;
  double L, K, Ke, half_ly;  // K of the force (:643), Ke of the energy (:682)
};

__device__ __forceinline__ double wall_force_y(const Walls& w, double y) {
  if (y <= w.L) return w.K * (w.L - y);
  if ((w.half_ly - y <= w.L) && (y <= w.half_ly)) return -(w.K * (w.L - w.half_ly + y));
  return 0.0;
}

__device__ __forceinline__ double wall_energy(const Walls& w, double y) {
  if (y <= w.L) return 0.5 * w.Ke * (w.L - y) * (w.L - y);
  if ((w.half_ly - y <= w.L) && (y <= w.half_ly)) return 0.5 * w.Ke * (w.L - w.half_ly + y) * (w.L - w.half_ly + y);
  return 0.0;
}

__global__ void k_steric(PairArgs a, int type, double rad, double kT, double fs, double rc, double* __restrict__ F,
                         int accumulate, Walls w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.Nb) return;
  double f0 = 0, f1 = 0, f2 = 0;
  visit_partners(a, i, [&](int, double xd, double yd, double zd) {
    const double r = sqrt(xd * xd + yd * yd + zd * zd);
    const double mag = interaction_magnitude(r, type, rad, kT, fs, rc);
    f0 += mag * (xd / r);
    f1 += mag * (yd / r);
    f2 += mag * (zd / r);
  });
  if (w.on) f1 += wall_force_y(w, a.Y[3 * i + 1]);  // added after the barrier forces (:640)
  if (accumulate) {
    F[3 * i] += f0;
    F[3 * i + 1] += f1;
    F[3 * i + 2] += f2;
  } else {
    F[3 * i] = f0;
    F[3 * i + 1] = f1;
    F[3 * i + 2] = f2;
  }
}

// Energy of blob i with all its partners (each pair is seen from both blobs, so
// the total is half the sum over blobs; linked_list.cpp:283-360).
// A slip channel's wall energy enters twice, so that half the sum counts it once.
__global__ void k_potential_terms(PairArgs a, int type, double rad, double kT, double fs, double rc,
                                  double* __restrict__ Ui, Walls w) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.Nb) return;
  double u = 0.0;
  visit_partners(a, i, [&](int, double xd, double yd, double zd) {
    u += interaction_energy(sqrt(xd * xd + yd * yd + zd * zd), type, rad, kT, fs, rc);
  });
  if (w.on) u += 2.0 * wall_energy(w, a.Y[3 * i + 1]);
  Ui[i] = u;
}

// collection_of_rigid_bodies.cpp:207-239: a blob on the lower wall (y == 0) or at
// or beyond the upper one (y >= L_y/2).
__global__ void k_wall_overlap(const double* __restrict__ Y, int Nb, double half_ly, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= Nb) return;
  const double y = Y[3 * i + 1];
  if (y == 0.0 || y >= half_ly) atomicExch(flag, 1);
}

__global__ void k_overlap(PairArgs a, double lim, int* __restrict__ flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.Nb) return;
  bool hit = false;
  visit_partners(a, i, [&](int, double xd, double yd, double zd) {
    if (xd * xd + yd * yd + zd * zd < lim) hit = true;
  });
  if (hit) atomicExch(flag, 1);
}

__global__ void k_pairs(PairArgs a, unsigned long long* __restrict__ count, int* __restrict__ pairs,
                        long long cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.Nb) return;
  visit_partners(a, i, [&](int j, double, double, double) {
    if (j > i) {
      const unsigned long long k = atomicAdd(count, 1ull);
      if ((long long)k < cap) {
        pairs[2 * k] = i;
        pairs[2 * k + 1] = j;
      }
    }
  });
}

PairArgs pair_args(const Ctx& c) {
  PairArgs a;
  a.Y = c.d_Y;
  a.cell = c.d_cell;
  a.start = c.d_cell_start;
  a.sorted = c.d_cell_sorted;
  a.Nb = c.Nb;
  a.nb = c.nb;
  a.g.N = c.p.ncells;
  a.g.Lx = c.g.Lx;
  a.g.Ly = c.g.Ly;
  a.g.Lz = c.g.Lz;
  return a;
}

}  // namespace

int launch_exclusive_scan(const int* in, int* out, int n, cudaStream_t s) {
  if (n <= 2 * SCAN_CH) {  // one or two chunks: one CTA
    k_exclusive_scan<<<1, SCAN_T, 0, s>>>(in, out, n);
    FCM_LAUNCH_CHECK();
    return FCM_OK;
  }
  const int nchunks = (n + SCAN_CH - 1) / SCAN_CH;
  k_scan_chunk_sums<<<nchunks, SCAN_T, 0, s>>>(in, out, n);
  FCM_LAUNCH_CHECK();
  k_scan_chunk_offsets<<<1, SCAN_T, 0, s>>>(out, n, nchunks);
  FCM_LAUNCH_CHECK();
  k_scan_chunks<<<nchunks, SCAN_T, 0, s>>>(in, out, n);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

// linked_list.cpp:80-102 (populate).
int cells_build(Ctx& c, cudaStream_t s) {
  const int nc = c.ncell_total;
  FCM_CUDA(cudaMemsetAsync(c.d_cell_count, 0, sizeof(int) * nc, s));
  FCM_CUDA(cudaMemsetAsync(c.d_cell_cursor, 0, sizeof(int) * nc, s));
  if (c.Nb == 0) {
    FCM_CUDA(cudaMemsetAsync(c.d_cell_start, 0, sizeof(int) * (nc + 1), s));
    return FCM_OK;
  }
  CellGeom g{c.p.ncells, c.g.Lx, c.g.Ly, c.g.Lz};
  k_cell_ids<<<(c.Nb + 255) / 256, 256, 0, s>>>(c.d_Y, c.Nb, g, c.d_cell, c.d_cell_count);
  FCM_LAUNCH_CHECK();
  k_exclusive_scan<<<1, 1024, 0, s>>>(c.d_cell_count, c.d_cell_start, nc);
  FCM_LAUNCH_CHECK();
  k_cell_scatter<<<(c.Nb + 255) / 256, 256, 0, s>>>(c.d_cell, c.Nb, nc, c.d_cell_start, c.d_cell_cursor,
                                                    c.d_cell_sorted);
  FCM_LAUNCH_CHECK();
  k_cell_sort<<<(nc + 255) / 256, 256, 0, s>>>(c.d_cell_start, nc, c.d_cell_sorted);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

Walls walls(const Ctx& c, bool on) {
  const double L = 2.2 * c.p.blob_radius;
  return Walls{on && c.p.slip_channel ? 1 : 0, L, (40.0 * c.p.kT / c.p.blob_radius) / L,
               40.0 * c.p.kT / (L * c.p.blob_radius), 0.5 * c.g.Ly};
}

int cells_steric_forces(const Ctx& c, double* F, bool accumulate, cudaStream_t s, bool with_walls) {
  if (c.Nb == 0) return FCM_OK;
  k_steric<<<(c.Nb + 127) / 128, 128, 0, s>>>(pair_args(c), c.p.potential, c.p.blob_radius, c.p.kT, c.p.steric_fs,
                                              c.p.steric_rc, F, accumulate ? 1 : 0, walls(c, with_walls));
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int cells_potential_terms(const Ctx& c, double* Ui, cudaStream_t s) {
  if (c.Nb == 0) return FCM_OK;
  k_potential_terms<<<(c.Nb + 127) / 128, 128, 0, s>>>(pair_args(c), c.p.potential, c.p.blob_radius, c.p.kT,
                                                       c.p.steric_fs, c.p.steric_rc, Ui, walls(c, true));
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int cells_wall_overlap(const Ctx& c, int* d_flag, cudaStream_t s) {
  if (c.Nb == 0 || !c.p.slip_channel) return FCM_OK;
  k_wall_overlap<<<(c.Nb + 127) / 128, 128, 0, s>>>(c.d_Y, c.Nb, 0.5 * c.g.Ly, d_flag);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int cells_overlap(const Ctx& c, int* d_flag, cudaStream_t s) {
  FCM_CUDA(cudaMemsetAsync(d_flag, 0, sizeof(int), s));
  if (c.Nb == 0) return FCM_OK;
  const double lim = 4.0 * c.p.blob_radius * c.p.blob_radius;
  k_overlap<<<(c.Nb + 127) / 128, 128, 0, s>>>(pair_args(c), lim, d_flag);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

int cells_count_pairs(const Ctx& c, long long* d_count, int* pairs, long long cap, cudaStream_t s) {
  FCM_CUDA(cudaMemsetAsync(d_count, 0, sizeof(long long), s));
  if (c.Nb == 0) return FCM_OK;
  k_pairs<<<(c.Nb + 127) / 128, 128, 0, s>>>(pair_args(c), (unsigned long long*)d_count, pairs, cap);
  FCM_LAUNCH_CHECK();
  return FCM_OK;
}

FCM_BOUNDS_READER(bounds_read_cells)

}  // namespace fcm
