// fcm_internal.cuh -- shared declarations of the B200 FCM library (not part of
// the public C-ABI; see include/fcm_b200.h).
//
// Device data layout (one suspension, one GPU):
//   real grid    T[3][nx][ny][nz]        (component-major, z fastest, unpadded)
//   spectrum     complex T[3][nx][ny][nzh], nzh = nz/2+1 (cuFFT R2C layout)
//   blob tables  base int[Nb][3] (first stencil point per dim, unwrapped),
//                weights T[Nb][3][W], and the same weights on the four
//                8-aligned grid chunks the stencil meets, T[Nb][3][4][8]
//   system vecs  double[3Nb + 6M]       ([lambda ; U], as the reference)
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/fcm_b200.h"

namespace fcm {

// ------------------------------------------------------------------ errors
void set_error(const std::string& msg);
struct Status {
  int code;
};

#define FCM_CUDA(call)                                                          \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ::fcm::set_error(std::string(#call) + ": " + cudaGetErrorString(e_));     \
      return (int)FCM_ERR_CUDA;                                                    \
    }                                                                           \
  } while (0)

#define FCM_CUFFT(call)                                                         \
  do {                                                                          \
    cufftResult r_ = (call);                                                    \
    if (r_ != CUFFT_SUCCESS) {                                                  \
      ::fcm::set_error(std::string(#call) + ": cufft error " + std::to_string((int)r_)); \
      return (int)FCM_ERR_CUFFT;                                                \
    }                                                                           \
  } while (0)

#define FCM_TRY(expr)                 \
  do {                                \
    int s_ = (expr);                  \
    if (s_ != FCM_OK) return s_;      \
  } while (0)

void count_launch();
void count_launches(long long n);
long long launch_count();

#define FCM_LAUNCH_CHECK()                                                      \
  do {                                                                          \
    ::fcm::count_launch();                                                      \
    cudaError_t e_ = cudaGetLastError();                                        \
    if (e_ != cudaSuccess) {                                                    \
      ::fcm::set_error(std::string("kernel launch: ") + cudaGetErrorString(e_)); \
      return (int)FCM_ERR_CUDA;                                                    \
    }                                                                           \
  } while (0)

// ------------------------------------------------------------------ bounds-checked build
// Compiled with -DFCM_BOUNDS_CHECK (libfcm_b200_debug.so), FCM_INB(i, n, site) is
// true when 0 <= i < n.  Otherwise the violation is counted in this translation
// unit's device record (the first violation's site, index and limit are kept) and
// the caller skips the access.  Nothing traps: the kernel runs to its end and the
// host reads the records through fcm_debug_bounds.  In the release build FCM_INB
// is the constant true and every check compiles away.
enum BoundsSite : int {
  BS_GRID = 1,      // grid point index against the grid's 3 G values
  BS_BLOB = 2,      // blob id (from a tile list or a cell list) against the blob count
  BS_TILE = 3,      // tile index against the tile count
  BS_LIST = 4,      // tile-list or cell-list slot against its range or capacity
  BS_PARTIAL = 5,   // per-(blob, tile) partial against its table
  BS_CELL = 6,      // cell id against the cell count
  BS_SPECTRUM = 7,  // spectrum index against the spectrum's 3 Gc values
  BS_KRYLOV = 8,    // Krylov column (GMRES iteration) against the columns allocated
};
struct BoundsRecord {
  unsigned long long count;
  long long index, limit;
  int site, pad;
};
#ifdef FCM_BOUNDS_CHECK
static __device__ BoundsRecord g_fcm_bounds;
static __device__ __noinline__ void fcm_bounds_record(long long i, long long n, int site) {
  if (atomicAdd(&g_fcm_bounds.count, 1ull) == 0ull) {
    g_fcm_bounds.index = i;
    g_fcm_bounds.limit = n;
    g_fcm_bounds.site = site;
  }
}
static __device__ __forceinline__ bool fcm_inb(long long i, long long n, int site) {
  if (i >= 0 && i < n) return true;
  fcm_bounds_record(i, n, site);
  return false;
}
#define FCM_INB(i, n, site) ::fcm::fcm_inb((long long)(i), (long long)(n), (site))
#define FCM_BOUNDS_READER(fn)                                                                   \
  int fn(BoundsRecord* out, int reset) {                                                        \
    FCM_CUDA(cudaMemcpyFromSymbol(out, g_fcm_bounds, sizeof(BoundsRecord)));                    \
    if (reset) {                                                                                \
      const BoundsRecord z{};                                                                   \
      FCM_CUDA(cudaMemcpyToSymbol(g_fcm_bounds, &z, sizeof(BoundsRecord)));                     \
    }                                                                                           \
    return FCM_OK;                                                                              \
  }
#else
#define FCM_INB(i, n, site) true
#define FCM_BOUNDS_READER(fn)          \
  int fn(BoundsRecord* out, int) {     \
    *out = BoundsRecord{};             \
    return FCM_OK;                     \
  }
#endif
// The record of each translation unit with checked kernels.
int bounds_read_grid(BoundsRecord* out, int reset);
int bounds_read_cells(BoundsRecord* out, int reset);
int bounds_read_kspace(BoundsRecord* out, int reset);
int bounds_read_blas(BoundsRecord* out, int reset);

template <typename T>
struct cplx_t;
template <>
struct cplx_t<double> {
  typedef cufftDoubleComplex type;
};
template <>
struct cplx_t<float> {
  typedef cufftComplex type;
};

// ------------------------------------------------------------------ geometry
struct GridDims {
  int nx, ny, nz, nzh;
  long long G;   // nx*ny*nz
  long long Gc;  // nx*ny*nzh
  double dx, Lx, Ly, Lz;
};

// Precomputed separable Gaussian stencil of a set of blobs
// (fcm_fluid_solver.cpp:131-165 gaussx/y/z and indx/y/z).
template <typename T>
struct BlobTable {
  int n = 0;         // blobs
  int W = 0;         // stencil width
  int* base = nullptr;   // [n][3] unwrapped first grid index per dim
  T* w = nullptr;        // [n][3][W]
  // Binning of (blob, tile) overlaps for the tiled spread / interpolation.
  // Usable when every grid dimension is a multiple of the tile edge and
  // W + tile edge <= n (a stencil never meets the same tile twice).
  bool tiled = false;
  int ntx = 0, nty = 0, ntz = 0, ntiles = 0;
  T* wc = nullptr;                // [n][3][4][8] weights on the 8-aligned grid chunks a stencil meets
  int* tile_count = nullptr;      // [ntiles]
  int* tile_offset = nullptr;     // [ntiles+1] exclusive offsets
  int* tile_cursor = nullptr;     // [ntiles]
  unsigned long long* tile_list = nullptr;  // [cap] (blob << 32) | chunk indices, j and half masks
  long long tile_cap = 0;
  T* partial = nullptr;           // [n][64][3] per-(blob, tile) interpolation partials
  double* ypos = nullptr;         // [n][3] positions of the current tables
  // force dipoles (allocated on first use): dipole-envelope weights and their
  // x-derivative factors on the chunks, per-(blob, tile) velocity moments
  T* wd = nullptr;                // [n][3][4][8]
  T* hd = nullptr;                // [n][3][4][8]
  T* partial9 = nullptr;          // [n][64][9]
};

// Grid buffers and cuFFT plans of one precision.
template <typename T>
struct GridBufs {
  bool ready = false;
  bool borrowed = false;                       // r, c, urand are slices of a batch's group arrays
  T* r = nullptr;                              // 3*G real
  typename cplx_t<T>::type* c = nullptr;       // 3*Gc spectrum
  T* urand = nullptr;                          // 3*G random velocity field
  cufftHandle r2c = 0, c2r = 0;
  cufftHandle r2c2d = 0, c2r2d = 0;            // (y, z) transforms of every x-plane (fused x path)
  BlobTable<T> blobs;                          // all blobs of the suspension
  BlobTable<T> ref_blobs;                      // single body (reference matrices)
};

// Tile shape of the tiled spread / interpolation kernels.
constexpr int TILE_X = 8, TILE_Y = 8, TILE_Z = 8;

// Tile grid of the tiled spread / interpolation (fcm_grid.cu).
struct TileGeom {
  int ntx, nty, ntz, nx, ny, nz, W;
  int ycut;            // interpolation reads rows y < ycut only (ny, or ny/2 in a slip channel)
  int nblobs;          // blobs of the tables
  long long list_cap;  // capacity of the tile list (entries)
};

// k-space geometry of the projection (fcm_kspace.cu).
struct KParams {
  int nx, ny, nz, nzh;
  long long Gc;
  double fx, fy, fz;  // 2 pi / L
  double inv_etaG;    // 1 / (eta * nx*ny*nz)
  int slip;           // slip channel: image-symmetric fluctuating stress
};

// Record of one device-resident (graph) time step, written by the device.
struct StepRecord {
  int iters;     // GMRES iterations, summed over refinement sweeps
  int sweeps;    // refinement sweeps (1 for an FP64 solve)
  int status;    // FCM_OK / FCM_ERR_NOT_CONVERGED / FCM_ERR_NONFINITE
  int guard;     // iterations of the loop in progress (bounds every device loop)
  double rel;    // final relative residual
  double divU;   // GDC divergence term (0 for EM or without noise)
  double normb;  // ||RHS|| of the refinement
  double relr;   // refinement residual of the last sweep
  int ref_active;  // batched refinement: this member still sweeps
  int pad_;
};

// Device-resident state of a Metropolis run (main.cpp:113-210).
struct McmcDev {
  uint64_t seed;
  long long n_target;     // accepted + rejected steps to reach
  long long n;            // steps done (overlap retries excluded)
  long long attempt;      // proposals drawn (the random stream position)
  long long attempt_cap;  // bound on proposals in this run
  double scale, acc;      // proposal scale, running acceptance ratio
  double U_old;           // energy of the current configuration
  double body_radius, dt, kT;
  int restore;            // the last proposal is undone
  int skip_on_overlap;
};

// Device-resident state of one GMRES solve (gmres_solver.cpp:148-306).
struct GmState {
  int k;        // Arnoldi columns completed (the reference's `iter`)
  int done;     // 1 once converged, out of iterations or non-finite
  int status;   // FCM_OK / FCM_ERR_NOT_CONVERGED / FCM_ERR_NONFINITE
  int maxit;
  double normb, rel, tol;
};

// ------------------------------------------------------------------ context
struct Ctx {
  fcm_params p;
  int M = 0, nb = 0, Nb = 0, nsys = 0;
  GridDims g;
  cudaStream_t stream = 0;
  int device = 0;

  // shape: 3*nb doubles (one shape for every body, as the reference's collection
  // has), or 3*nb per body after fcm_set_body_shapes.  With per-body shapes
  // d_Minv, d_N and d_KTKinv hold one block per body as well; the strides below
  // are 0 for the shared shape and one block for per-body shapes.
  double* d_ref = nullptr;
  bool per_body = false;
  int ref_stride = 0;        // 0 or 3*nb
  long long minv_stride = 0; // 0 or (3nb)^2
  int n_stride = 0;          // 0 or 36 (ref_N and ref_KTKinv)
  // bodies (x 3M, q 4M) current / midstep / saved start of step
  double *d_x = nullptr, *d_q = nullptr, *d_xm = nullptr, *d_qm = nullptr, *d_xs = nullptr, *d_qs = nullptr;
  double *d_Y = nullptr;     // all_blob_pos Nb*3
  double *d_V = nullptr;     // fcm.V 3Nb
  double *d_F = nullptr;     // blob_forces 3Nb
  double *d_fe = nullptr;    // external body forces 6M
  double *d_U0 = nullptr;    // rigid projection of the random velocities 6M
  double *d_tmp3 = nullptr;  // 3Nb scratch
  double *d_tmp6 = nullptr;  // 6M scratch
  double *d_sys_a = nullptr, *d_sys_b = nullptr;   // system-size scratch
  double *d_rhs = nullptr;   // RHS
  double *d_soln = nullptr;  // saddle-point solution
  double *d_res = nullptr, *d_dx = nullptr;  // refinement residual / correction
  // preconditioner
  double *d_Minv = nullptr, *d_N = nullptr, *d_KTKinv = nullptr;
  std::vector<double> h_Minv, h_N, h_KTKinv;
  bool have_ref = false;
  // GMRES
  double *d_Qm = nullptr;    // nsys * (maxit+1)
  double *d_H = nullptr;     // (maxit+1) column scratch
  double *d_y = nullptr;     // maxit coefficients
  double *d_partials = nullptr;
  unsigned int* d_counter = nullptr;
  int red_blocks = 0;
  int maxit_alloc = 0;
  double* h_pinned = nullptr;  // small pinned host staging (>= 256 doubles)
  // device-side GMRES
  GmState* gm = nullptr;        // device state
  GmState* h_gm = nullptr;      // pinned host copy
  double *d_Hd = nullptr, *d_beta = nullptr, *d_CS = nullptr, *d_SN = nullptr;
  double *d_hA = nullptr, *d_hB = nullptr, *d_hnorm = nullptr;
  double* d_mdpart = nullptr;   // multidot partials [(maxit+1) * md_blocks]
  unsigned int* d_mdcount = nullptr;
  int md_blocks = 0;
  cudaStream_t cap_stream = 0;  // private stream for graph capture
  cudaGraphExec_t iter_graph[2] = {nullptr, nullptr};  // one Arnoldi iteration, per precision
  long long iter_graph_kernels[2] = {0, 0};           // kernels in each graph
  // device-resident step: the whole step as one graph with conditional loops
  StepRecord* d_step = nullptr;     // written by the step's kernels
  StepRecord* h_step = nullptr;     // pinned copy, the graph's last node
  uint64_t* d_stepargs = nullptr;   // (seed, counter) of the step in flight
  uint64_t* h_stepargs = nullptr;   // pinned staging of d_stepargs
  double* d_rs = nullptr;           // [0] ||b|| [1] ||r|| [2] inner tolerance [3] nu
  // Metropolis runs (allocated on first use)
  McmcDev* d_mcmc = nullptr;
  double* d_usum = nullptr;         // sum of the per-blob pair energies
  cudaGraphExec_t mcmc_graph = nullptr;
  long long mcmc_kernels = 0;       // kernels of one proposal in mcmc_graph
  double body_radius = 0.0;         // largest |blob_ref_pos| (collection_of_rigid_bodies.cpp:110-114)
  cudaStream_t cap_body[2] = {0, 0};  // capture streams of the loop bodies
  cudaGraphExec_t step_graph = nullptr;
  int step_graph_state = 0;         // 0 not built yet, 1 built, -1 unavailable (host-driven steps)
  long long step_kernels_top = 0, step_kernels_sweep = 0, step_kernels_iter = 0;
  bool step_pending = false;        // fcm_step_async issued, fcm_step_wait not yet called
  bool step_pending_graph = false;  // ... and it was a graph launch
  int step_pending_status = 0;      // host-driven pending step: its status and record
  fcm_step_info step_pending_info{};
  bool in_batch = false;            // owned by a batch (its step record and arguments too)
  // force dipoles (allocated on first use): T 3Nb, S 9Nb, D 9Nb, Omega 3Nb, E 9Nb
  double* d_dip = nullptr;
  // shear forcing (fcm_fluid_solver.hpp SHEARING_FORCES fields), allocated when
  // the imposed flow is produced: u_shear 3G (the grid layout of g64.r), Vshear 3Nb
  // fused x-transform of the Stokes solve, per grid precision ([0] FP64, [1] FP32):
  // on when nx is a supported length and nz is even (FP64 up to 256 points, beyond
  // which the 3D transforms are faster); twiddles exp(-2 pi i j / nx), j < nx
  bool xfft[2] = {false, false};
  // FP32 (y, z) transforms by this library's kernels instead of cuFFT's 2D plans
  // (fused FP32 grids whose ny and nz are supported lengths, nz even, nz <= 256);
  // twiddles exp(-2 pi i j / n) for n = ny, nz
  bool yz32 = false;
  // what the grids allow (fcm_autotune chooses within it): the fused x-transform per
  // precision (its (y, z) plans exist), the library's (y, z) kernels up to 512 points
  bool xfft_cap[2] = {false, false};
  bool yz32_cap = false;
  // spread kernel per precision: 0 the persistent software-pipelined one (FP64
  // default), 1 / 2 / 3 one CTA per tile staging 16 / 8 / 32 blobs per round, 4
  // one warp per tile (FP32 default); all sum every point's blobs in the same order
  int spread_variant[2] = {0, 4};
  // interpolation kernel per precision: 0 the 64-thread shuffle-reduced tile
  // kernel (k_interp_tiled), 1 one warp per tile with two y-rows per lane and the
  // shuffle reduction (k_interp_warp, the default), 2 the shared-memory reduced
  // kernel with two y-rows per thread (k_interp_rows, 32 threads per tile)
  int interp_variant[2] = {1, 1};
  void* d_ytw32 = nullptr;
  void* d_ztw32 = nullptr;
  void* d_xtw64 = nullptr;
  void* d_xtw32 = nullptr;
  double* d_ushear = nullptr;
  double* d_vshear = nullptr;
  bool shear = false;
  bool graph_stale = false;         // a captured step graph predates a change of the step's work
  // cells
  int ncell_total = 0;
  int *d_cell = nullptr, *d_cell_start = nullptr, *d_cell_count = nullptr, *d_cell_sorted = nullptr, *d_cell_cursor = nullptr;
  int *d_flag = nullptr;     // overlap flag
  long long *d_pair_count = nullptr;
  // grids
  GridBufs<double> g64;
  GridBufs<float> g32;
  // injected stress (FP64): 6*G real + 6*Gc complex
  double* d_stress = nullptr;
  cufftDoubleComplex* d_stress_c = nullptr;
  cufftHandle plan_r2c6 = 0;
  // state flags
  bool gauss_ready = false;
  bool urand_ready = false;
  bool det_ready = false;   // deterministic velocity grid holds u
  int urand_prec = 0;       // precision of the random field last produced
};

// ------------------------------------------------------------------ batches
// One member suspension of a batch as the batched kernels see it (a device
// array, one entry per member; blockIdx.y or .z selects the member).
struct BMember {
  int Nb, M, nb, nsys;
  int hn;  // columns of the member's Krylov basis (maxit_alloc + 1)
  int red_blocks, md_blocks;  // the member's own reduction grids (same sums as its single solve)
  const double *qm, *ref, *Minv, *N;
  int ref_stride, n_stride;   // per-body shape strides (0: one shared shape)
  long long minv_stride;
  double *sys_a, *sys_b, *rhs, *soln, *res, *dx;
  GmState* gm;
  double *Qm, *Hd, *beta, *CS, *SN, *hA, *hB, *hnorm, *y;
  double* partials;    // [max red blocks] batch reduction scratch
  unsigned* counter;   // [1]
  double* mdpart;      // [hn * max md blocks]
  unsigned* mdcount;   // [hn]
  StepRecord* sd;
  double* rs;          // [0] ||b|| [1] ||r|| [2] inner tolerance [3] nu
  // grid of each precision, [0] FP64 and [1] FP32
  const void* wc[2];
  const int* toff[2];
  const unsigned long long* tlist[2];
  const int* base[2];
  void* grid[2];
  void* spec[2];
  void* partial[2];
  TileGeom tg[2];  // tile geometry of each precision's tables (their stencil widths differ)
  KParams kp;
  double dx3;
  int xfft[2];  // the member's grids of each precision use the fused x-transform
};

// Which members a batched kernel works on.
enum BMask { BM_ALL = 0, BM_GM = 1, BM_REF = 2 };  // all / GMRES not done / refinement active
// Member vectors addressed by batched kernels.
enum BVec { BV_SYS_A = 0, BV_SYS_B, BV_RHS, BV_SOLN, BV_RES, BV_DX };
// Member scalars written by batched reductions.
enum BOut { BO_HNORM = 0, BO_RS0, BO_RS1 };

#ifdef __CUDACC__
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds, multipliers 0xD2511F53 / 0xCD9E8D57, Weyl key
// increments 0x9E3779B9 / 0xBB67AE85.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned int lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
    const unsigned int lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
    c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
    k.x += 0x9E3779B9u;
    k.y += 0xBB67AE85u;
  }
  return c;
}

// Uniform double in [0, 1) with 53 random bits: Philox block with counter
// (i, 0x4D434D43, attempt_lo, attempt_hi) and key (seed_lo, seed_hi); the top
// 27 bits of word 0 and the top 26 bits of word 1.
__device__ __forceinline__ double mcmc_uniform(uint64_t seed, uint64_t attempt, unsigned int i) {
  const uint4 r = philox4x32_10(make_uint4(i, 0x4D434D43u, (unsigned int)attempt, (unsigned int)(attempt >> 32)),
                                make_uint2((unsigned int)seed, (unsigned int)(seed >> 32)));
  return ((double)(r.x >> 5) * 67108864.0 + (double)(r.y >> 6)) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double* bvec(const BMember& m, int v) {
  switch (v) {
    case BV_SYS_A: return m.sys_a;
    case BV_SYS_B: return m.sys_b;
    case BV_RHS: return m.rhs;
    case BV_SOLN: return m.soln;
    case BV_RES: return m.res;
    default: return m.dx;
  }
}

__device__ __forceinline__ double* bout(const BMember& m, int o) {
  return o == BO_HNORM ? m.hnorm : (o == BO_RS0 ? m.rs : m.rs + 1);
}

__device__ __forceinline__ bool bskip(const BMember& m, int mask) {
  return (mask == BM_GM && m.gm->done) || (mask == BM_REF && !m.sd->ref_active);
}
#endif

// Launch geometry of a batch (host side).
struct BatchGeom {
  int n = 0;                   // members
  int max_sys_blocks = 1;      // ceil(max nsys / 256)
  int max_blob_blocks = 1;     // ceil(max Nb / 128)
  int max_body_blocks = 1;     // ceil(max M / 128)
  int max_pinv_blocks = 1;     // ceil(max M / 4) (4 warps per block)
  int max_nb = 1;              // blobs per body (shared memory of the preconditioner)
  int red_blocks = 1;          // reduction blocks per member (the largest)
  int md_blocks = 1;           // multidot blocks per member (the largest)
  int max_hn = 1;              // multidot columns
  int total_tiles = 0;         // sum of the members' tiles
  int total_kblocks = 0;       // sum of the members' k-space blocks (256 modes)
  const BMember* mem = nullptr;      // device array [n]
  const int2* tile_map = nullptr;    // [total_tiles] (member, tile)
  const int2* kblock_map = nullptr;  // [total_kblocks] (member, block)
};

KParams make_kparams(const Ctx& c);
// Tile geometry of a grid for tables of nblobs blobs with a tile list of
// list_cap entries.
TileGeom tile_geom(const GridDims& g, int W, int nblobs, long long list_cap);
template <typename T>
inline TileGeom tile_geom(const GridDims& g, const BlobTable<T>& t) {
  return tile_geom(g, t.W, t.n, t.tile_cap);
}

// batched kernels (fcm_blas.cu, fcm_bodies.cu, fcm_grid.cu, fcm_kspace.cu)
int b_gm_init(const BatchGeom& b, int vec, double tol, int use_rs_tol, int mask, cudaStream_t s);
int b_gm_fetch(const BatchGeom& b, cudaStream_t s);
int b_gm_orthogonalize(const BatchGeom& b, cudaStream_t s);
int b_gm_finish(const BatchGeom& b, cudaStream_t s);
int b_norm(const BatchGeom& b, int vec, int out, int mask, cudaStream_t s);
int b_axpby(const BatchGeom& b, int y, int x, double a, double bb, int mask, cudaStream_t s);
int b_pinv(const BatchGeom& b, int in, int out, int mask, cudaStream_t s);
int b_multiply_K_KT(const BatchGeom& b, int in, int out, int mask, cudaStream_t s);
template <typename T>
int b_spread(const BatchGeom& b, int in, int mask, cudaStream_t s);
template <typename T>
int b_interp(const BatchGeom& b, int out, int mask, cudaStream_t s);
template <typename T>
int b_project(const BatchGeom& b, int mask, cudaStream_t s);

// ------------------------------------------------------------------ launchers
// gaussians + binning (fcm_grid.cu)
template <typename T>
int blob_table_alloc(BlobTable<T>& t, int n, int W, const GridDims& g);
template <typename T>
void blob_table_free(BlobTable<T>& t);
template <typename T>
int launch_set_up_gaussians(const Ctx& c, BlobTable<T>& t, const double* dY, cudaStream_t s);
template <typename T>
int launch_spread(const Ctx& c, const BlobTable<T>& t, const double* dF, T* grid, cudaStream_t s);
template <typename T>
int launch_interp(const Ctx& c, const BlobTable<T>& t, const T* grid, double* dV, cudaStream_t s);
// force dipoles (fcm_grid.cu): D (9 per blob) added to the force grid; moments
// of the velocity grid into Omega (3 per blob) and E (9 per blob)
// slip channel: the image of the lower half over the upper half of a force grid
// (fcm_fluid_solver.cpp:602-632)
template <typename T>
int launch_slip_image(const Ctx& c, T* grid, cudaStream_t s);
template <typename T>
int launch_spread_dipoles(const Ctx& c, BlobTable<T>& t, const double* dD, T* grid, cudaStream_t s);
template <typename T>
int launch_interp_dipoles(const Ctx& c, BlobTable<T>& t, const T* grid, double* dOm, double* dE, cudaStream_t s);
int launch_blob_dipoles(const double* T3, const double* S9, int n, double* D9, cudaStream_t s);
// k-space (fcm_kspace.cu)
template <typename T>
int launch_project(const Ctx& c, typename cplx_t<T>::type* spec, cudaStream_t s);
// the x-transform, projection and inverse x-transform of a spectrum holding the
// (y, z) transforms of every x-plane (fcm_kspace.cu)
bool xfft_factor(int n, int* n1, int* n2);
int xfft_tables_init();
template <typename T>
int xfft_prepare(const Ctx& c);
template <typename T>
int launch_xfft_project(const Ctx& c, typename cplx_t<T>::type* spec, cudaStream_t s);
// the FP32 (y, z) transforms of `members` consecutive grids of c's shape (fcm_kspace.cu)
int launch_yz_forward(const Ctx& c, const float* r, cufftComplex* spec, int members, cudaStream_t s);
int launch_yz_inverse(const Ctx& c, cufftComplex* spec, float* r, int members, cudaStream_t s);
// the same for the members gidx[0..nm) of a batch group whose grids equal c0's
template <typename T>
int b_xfft_project(const BatchGeom& b, const Ctx& c0, const int* gidx, int nm, int mask, cudaStream_t s);
// (seed, counter) are read from d_args[0..1] instead when d_args is given.
template <typename T>
int launch_noise_kspace(const Ctx& c, typename cplx_t<T>::type* spec, uint64_t seed, uint64_t counter,
                        const uint64_t* d_args, cudaStream_t s);
int launch_stress_divergence_project(const Ctx& c, const cufftDoubleComplex* sigma6, cufftDoubleComplex* spec, cudaStream_t s);
// shear forcing (fcm_kspace.cu): grid x-component = row[j] on every (i, k),
// y and z components zero; and out[j] = mean over (i, k) of u[i][j][k] + add[i][j][k]
int launch_shear_forcing(const Ctx& c, const double* d_row, double* grid, cudaStream_t s);
int launch_x_profile(const Ctx& c, const double* u, const double* add, double* d_out, cudaStream_t s);
int launch_unpad_copy(const double* src_padded, double* dst, int nx, int ny, int nz, int pad, int ncomp_stride_dst, cudaStream_t s);
// bodies (fcm_bodies.cu)
int launch_fill_blob_pos(const Ctx& c, const double* x, const double* q, double* Y, cudaStream_t s);
int launch_multiply_K(const Ctx& c, const double* qm, const double* in6, double* out3, double scale_acc, cudaStream_t s);
int launch_multiply_KT(const Ctx& c, const double* qm, const double* in3, double* out6, double scale, const double* add6, double add_scale, cudaStream_t s);
int launch_pinv(const Ctx& c, const double* qm, const double* in, double* out, cudaStream_t s);
int launch_rigid_projection(const Ctx& c, const double* q, const double* V, double* U6, cudaStream_t s);
// U scaled by `scale`, times *d_nu when d_nu is given.
int launch_body_update(const Ctx& c, double* x, double* q, const double* U6, double scale, cudaStream_t s,
                       const double* d_nu = nullptr);
int launch_body_update_uniform(const Ctx& c, double* x, double* q, const double* e6, cudaStream_t s);
// Metropolis proposal for every body (bodies saved to xs, qs first) and the
// undo of a rejected proposal (main.cpp:126-160, :170-185).
int launch_mcmc_propose(const Ctx& c, const McmcDev* st, cudaStream_t s);
int launch_mcmc_restore(const Ctx& c, const McmcDev* st, cudaStream_t s);
int launch_divU_accumulate(const Ctx& c, const double* U6, const double* U0, int component, double delta, double* acc, cudaStream_t s);
int launch_exclusive_scan(const int* in, int* out, int n, cudaStream_t s);
// cells (fcm_cells.cu)
int cells_build(Ctx& c, cudaStream_t s);
// with_walls adds a slip channel's wall forces (collection_of_rigid_bodies.cpp:640-662)
int cells_steric_forces(const Ctx& c, double* F, bool accumulate, cudaStream_t s, bool with_walls = false);
// OR-s a slip channel's wall contacts of all_blob_pos into *d_flag (no-op otherwise)
int cells_wall_overlap(const Ctx& c, int* d_flag, cudaStream_t s);
int cells_overlap(const Ctx& c, int* d_flag, cudaStream_t s);
// per-blob pair energies (half their sum is the potential of linked_list.cpp:283-360)
int cells_potential_terms(const Ctx& c, double* Ui, cudaStream_t s);
int cells_count_pairs(const Ctx& c, long long* d_count, int* pairs, long long cap, cudaStream_t s);
// vector ops (fcm_blas.cu)
int blas_dot(const Ctx& c, const double* a, const double* b, long long n, double* d_out, cudaStream_t s);
int blas_mgs_step(const Ctx& c, double* w, const double* q_prev, const double* h_prev, const double* q_i, long long n, double* d_hout, cudaStream_t s);
int blas_scale(double* v, const double* d_num, int invert, long long n, cudaStream_t s);
int blas_axpby(double* y, const double* x, double a, double b, long long n, cudaStream_t s);
int blas_combine(double* out, const double* Q, const double* d_y, int k, long long n, cudaStream_t s);
int blas_copy_scaled(double* dst, const double* src, const double* d_num, int invert, long long n, cudaStream_t s);
int blas_norm_sq_partial(const Ctx& c, const double* a, long long n, double* d_out, cudaStream_t s);
int blas_f64_to_f32(float* dst, const double* src, long long n, cudaStream_t s);
int blas_sum_accumulate(const Ctx& c, const double* a, long long n, double* d_out, cudaStream_t s);
// device-side GMRES pieces (fcm_blas.cu)
// tol is read from *d_tol instead when d_tol is given.
int gm_init(const Ctx& c, const double* b, double tol, int maxit, cudaStream_t s, const double* d_tol = nullptr);
int gm_fetch(const Ctx& c, double* dst, cudaStream_t s);
int gm_orthogonalize(const Ctx& c, double* w, cudaStream_t s);
int gm_finish(const Ctx& c, double* soln_pre, cudaStream_t s);

// symmetric inverse: inv() when well conditioned, otherwise the pseudo-inverse
// (fcm_linalg.cpp)
bool sym_inv_or_pinv(const std::vector<double>& A, int n, std::vector<double>& out, bool* used_pinv);

}  // namespace fcm
