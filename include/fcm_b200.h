/*
 * fcm_b200.h -- C-ABI of the B200-native fluctuating force-coupling-method (FCM)
 * mobility solve for Brownian suspensions of rigid multi-blob bodies.
 *
 * Every entry point is `extern "C"`, takes plain pointers and sizes, and returns an
 * int status (FCM_OK == 0).  Array arguments may be HOST or DEVICE pointers: the
 * library inspects each pointer (cudaPointerGetAttributes) and copies as needed.
 * Host arrays are borrowed for the duration of the call only.  Device buffers are
 * owned by the context.  A context is not thread-safe; separate contexts may run on
 * separate streams.  All work is issued on the context's stream (fcm_set_stream);
 * calls that return data to a host pointer synchronise that stream.
 *
 * The functions replace the public methods of the reference's five C++ classes
 * (fft_solver, fcm_fluid_solver, collection_of_rigid_bodies, linked_list,
 * gmres_solver).  Each declaration cites the reference method it replaces as
 * file:line within the reference project.  The reference's MPI domain
 * decomposition is collapsed to one rank on one GPU: every MPI_Allreduce in the
 * replaced methods becomes a local sum.
 *
 * Array layouts (all FP64 at the boundary):
 *   blob_ref_pos : 3*nb, blob-major (x,y,z of blob m at 3m..3m+2); the columns of
 *                  the reference's `blob_ref_pos` (3 x nb) matrix.
 *   Y            : Nb*3, blob-major xyz (row np of the reference's `all_blob_pos`).
 *   F, V, lambda : 3*Nb, index 3*np+c (the reference's `vec` layout).
 *   body x, q    : 3*M and 4*M (q = scalar part then vector part).
 *   U (bodies)   : 6*M, (Ux,Uy,Uz,Wx,Wy,Wz) per body.
 *   system vec   : 3*Nb + 6*M = [lambda ; U] (gmres_solver.cpp:60).
 *   grid arrays  : the reference's FFTW layout: real [x][y][pad] with
 *                  pad = 2*(nz/2+1); after a forward transform the complex
 *                  result is in FFTW_TRANSPOSED_ORDER [y][x][kz] (re,im).
 */
#ifndef FCM_B200_H
#define FCM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
enum fcm_status {
  FCM_OK = 0,
  FCM_ERR_INVALID = 1,       /* bad argument or parameter                        */
  FCM_ERR_CUDA = 2,          /* CUDA runtime error (message in fcm_last_error)    */
  FCM_ERR_CUFFT = 3,         /* cuFFT error                                       */
  FCM_ERR_STATE = 4,         /* call out of order (e.g. interpolation before
                                fcm_set_up_gaussians)                             */
  FCM_ERR_NOT_CONVERGED = 5, /* GMRES reached max_iter above tol; the iterate is
                                still returned, as gmres_solver.cpp:294-300 does  */
  FCM_ERR_NONFINITE = 6,     /* a NaN/Inf appeared (residual, forces, velocities) */
  FCM_ERR_OVERLAP = 7,       /* prohibited overlap after a step; bodies restored  */
  FCM_ERR_NOMEM = 8,         /* device allocation failed                          */
  FCM_ERR_CAPACITY = 9       /* caller-provided output buffer too small           */
};

/* ------------------------------------------------------------------ parameters
 * Runtime replacements for the compile-time macros of config.hpp.  Defaults
 * (fcm_default_params) follow config.hpp with SLIP_CHANNEL false and
 * SIMULATION_ALGORITHM 2 (Euler-Maruyama); set slip_channel = 1 for the
 * reference's default geometry. */
typedef struct fcm_params {
  int32_t nx, ny, nz;        /* NUM_FFT_GRID_POINTS_{X,Y,Z} (config.hpp:65-67)     */
  int32_t ngauss;            /* NUM_FCM_GAUSSIAN_POINTS, stencil width W (:69)     */
  double dx;                 /* DX, grid spacing; box side L_d = dx*n_d (:88-91)   */
  double blob_radius;        /* BLOB_RADIUS a (:48)                                */
  double viscosity;          /* FLUID_VISCOSITY eta (:49)                          */
  double kT;                 /* ENERGY_SCALE (:50)                                 */
  double dt;                 /* DT (:84)                                           */
  int32_t num_bodies;        /* NUM_BODIES M (:47)                                 */
  int32_t blobs_per_body;    /* nb (collection_of_rigid_bodies.cpp:21-32)          */
  int32_t ncells;            /* NUM_LINKED_LIST_CELLS_PER_DIM (:71), must be >= 3  */
  int32_t potential;         /* INTERACTION_POTENTIAL_TYPE (:20): 0 soft sphere,
                                1 hydrophobic, 2 hydrophilic (linked_list.cpp:362-497);
                                3 = polynomial repulsion F_s((rc^2-r^2)/(rc^2-4a^2))^4
                                for r < rc (no counterpart in the reference)       */
  double steric_fs;          /* potential 3: force scale F_s                       */
  double steric_rc;          /* potential 3: cutoff r_c                            */
  int32_t gmres_max_iter;    /* GMRES_MAX_ITER (:63)                               */
  double gmres_tol;          /* GMRES_TOL (:62), relative residual                 */
  double fd_delta;           /* FINITE_DIFFERENCE_DELTA_FACTOR (:73)               */
  int32_t algorithm;         /* SIMULATION_ALGORITHM (:26): 1 = GDC, 2 = EM        */
  int32_t precision;         /* 0 = FP64 throughout; 1 = FP32 grid work (spread,
                                FFT, projection, interpolation) inside FP64
                                iterative refinement                               */
  int32_t noise;             /* 1 = fluctuating stress on (main.cpp:231),
                                0 = noise off (deterministic runs)                  */
  int32_t skip_on_overlap;   /* SKIP_ON_OVERLAP (:35)                              */
  int32_t slip_channel;      /* SLIP_CHANNEL (:33): free-slip walls at y = 0 and
                                y = L_y/2 by the image system in y (the bodies live
                                in 0 < y < L_y/2): mirrored force grids and stress,
                                Gaussians truncated at ny/2, wall forces and
                                potential, steps rejected on wall contact.  Not
                                with batches, force dipoles or skip-free graph steps
                                (slip-channel steps are host-driven).             */
} fcm_params;

/* Per-step diagnostics returned by fcm_step. */
typedef struct fcm_step_info {
  int32_t gmres_iters;       /* Krylov iterations (sum over refinement sweeps)     */
  int32_t refinement_sweeps; /* outer FP64 sweeps (1 for precision 0)              */
  double gmres_rel_residual; /* final relative residual of the saddle-point system */
  double divU;               /* GDC drift divergence (0 for EM)                    */
  int32_t overlap;           /* 1 if the step was rejected and bodies restored     */
  int32_t status;            /* status of the GMRES solve                          */
} fcm_step_info;

/* State of a Metropolis Monte Carlo run (main.cpp:113-210), carried across calls. */
typedef struct fcm_mcmc_state {
  double scale;             /* proposal scale (main.cpp:120 starts at 0.1 a)           */
  double acceptance_ratio;  /* running acceptance ratio (main.cpp:121 starts at 0.5)   */
  double potential;         /* energy of the current configuration (output)            */
  int64_t steps;            /* Metropolis steps done (n of main.cpp; overlap retries
                               excluded)                                               */
  int64_t attempts;         /* proposals drawn: the position in the random stream      */
} fcm_mcmc_state;

typedef struct fcm_ctx fcm_ctx;   /* opaque solver context: one suspension */
typedef struct fcm_fft fcm_fft;   /* opaque standalone 3-D real FFT        */

/* Fill *p with config.hpp's defaults (single body type, 256^3 grid ...). */
void fcm_default_params(fcm_params* p);

/* Text of the last error recorded on this thread (never NULL). */
const char* fcm_last_error(void);

/* Library version string. */
const char* fcm_version(void);

/* Number of this library's own kernel launches so far in the process (cuFFT's
 * kernels are not included); a diagnostic counter. */
int64_t fcm_kernel_launch_count(void);

/* ================================================================ fft_solver
 * fft_solver.hpp:10-31.  In-place 3-D real transforms on an array of
 * total_local_size = nx*ny*pad doubles, unnormalised, forward sign e^{-iqx},
 * k-space result in FFTW_TRANSPOSED_ORDER [y][x][kz].  The inverse treats its
 * input as FFTW 2.x's rfftwnd does: complex inverse transforms along x and y,
 * then a half-complex-to-real transform along z that ignores the imaginary parts
 * of the kz = 0 and kz = nz/2 terms. */
int fcm_fft_create(int32_t nx, int32_t ny, int32_t nz, fcm_fft** out);   /* fft_solver.cpp:17-28 initialise */
int fcm_fft_destroy(fcm_fft* f);                                           /* fft_solver.cpp:8-15 ~fft_solver */
int fcm_fft_local_sizes(const fcm_fft* f, int32_t* local_nx, int32_t* local_x_start,
                        int32_t* local_ny_after_transpose,
                        int32_t* local_y_start_after_transpose,
                        int64_t* total_local_size, int32_t* pad);          /* fft_solver.cpp:24-26 */
int fcm_fft_transform(fcm_fft* f, double* in);                             /* fft_solver.cpp:32-36 */
int fcm_fft_inverse_transform(fcm_fft* f, double* in);                     /* fft_solver.cpp:38-42 */

/* ================================================================ context */
/* Create a context for one suspension.  blob_ref_pos: 3*nb reference blob
 * positions of the (single) body shape.  Replaces
 * collection_of_rigid_bodies::initialise (collection_of_rigid_bodies.cpp:15-153),
 * fcm_fluid_solver::initialise (fcm_fluid_solver.cpp:29-129),
 * gmres_solver::initialise (gmres_solver.cpp:14-34) and
 * linked_list::initialise (linked_list.cpp:23-72). */
int fcm_create(const fcm_params* p, const double* blob_ref_pos, fcm_ctx** out);
int fcm_destroy(fcm_ctx* ctx);
/* Issue all further work of this context on `stream` (a cudaStream_t). */
int fcm_set_stream(fcm_ctx* ctx, void* stream);
int fcm_get_params(const fcm_ctx* ctx, fcm_params* p);

/* ================================================================ collection_of_rigid_bodies */
/* Body state (particle x and quaternion q, particle.hpp:21-22). */
int fcm_set_bodies(fcm_ctx* ctx, const double* x, const double* q);
int fcm_get_bodies(fcm_ctx* ctx, double* x, double* q);
int fcm_get_midstep_bodies(fcm_ctx* ctx, double* x, double* q);
/* External force and torque per body (6*M), added to -K^T F in the RHS.  The
 * reference has none (only steric and wall forces); NULL clears it. */
int fcm_set_external_forces(fcm_ctx* ctx, const double* fe);
/* collection_of_rigid_bodies.cpp:155-174 (midstep=0) and :176-193 (midstep=1). */
int fcm_fill_all_blob_pos(fcm_ctx* ctx, int32_t at_midstep);
/* Overwrite / read all_blob_pos directly (Nb*3). */
int fcm_set_all_blob_pos(fcm_ctx* ctx, const double* Y);
int fcm_get_all_blob_pos(fcm_ctx* ctx, double* Y);
/* collection_of_rigid_bodies.cpp:707-731: out(3Nb) = K*in(6M) at the midstep. */
int fcm_multiply_by_K_at_midstep(fcm_ctx* ctx, const double* in, double* out);
/* collection_of_rigid_bodies.cpp:733-757: out(6M) = K^T*in(3Nb) at the midstep. */
int fcm_multiply_by_KT_at_midstep(fcm_ctx* ctx, const double* in, double* out);
/* collection_of_rigid_bodies.cpp:623-664: populate the cell list from
 * all_blob_pos and set blob_forces = steric forces (EM also sets the midstep
 * bodies to the current bodies, :625-629). */
int fcm_calculate_forces(fcm_ctx* ctx);
int fcm_get_blob_forces(fcm_ctx* ctx, double* F);
int fcm_set_blob_forces(fcm_ctx* ctx, const double* F);
/* collection_of_rigid_bodies.cpp:566-621: rigid projection of V (3Nb; NULL =
 * the context's last interpolated velocities) with ref_KTKinv, half step to the
 * midstep.  *overlap as the reference's return value. */
int fcm_advance_to_midstep(fcm_ctx* ctx, const double* V, int32_t* overlap);
/* collection_of_rigid_bodies.cpp:869-953: finite-difference div(U) of the random
 * velocity field over six body perturbations. */
int fcm_calculate_divU(fcm_ctx* ctx, double* divU);
/* collection_of_rigid_bodies.cpp:759-790: bodies += nu*dt*U (6M). */
int fcm_end_of_step_update(fcm_ctx* ctx, const double* U, double nu, int32_t* overlap);
/* collection_of_rigid_bodies.cpp:792-796. */
int fcm_reset_to_start_of_step(fcm_ctx* ctx);
/* collection_of_rigid_bodies.cpp:195-205 on the current all_blob_pos. */
int fcm_check_for_overlap(fcm_ctx* ctx, int32_t* overlap);
/* collection_of_rigid_bodies.cpp:207-239 on the current all_blob_pos: a blob with
 * y == 0 or y >= L_y/2 (always 0 without a slip channel).  With slip_channel,
 * fcm_advance_to_midstep and fcm_end_of_step_update report such contacts whatever
 * skip_on_overlap is (:611-617, :780-786). */
int fcm_check_for_channel_wall_overlap(fcm_ctx* ctx, int32_t* overlap);

/* ================================================================ linked_list */
/* linked_list.cpp:74-102: cell of every blob from all_blob_pos. */
int fcm_list_populate(fcm_ctx* ctx);
/* Cell id of every blob (Nb ints), linked_list.cpp:74-78. */
int fcm_list_get_cells(fcm_ctx* ctx, int32_t* cell_of_blob);
/* Inter-body pair set visited by linked_list.cpp:192-281 as (i<j) int pairs,
 * sorted lexicographically.  *npairs receives the total; FCM_ERR_CAPACITY if it
 * exceeds cap (then nothing is written). */
int fcm_list_get_pairs(fcm_ctx* ctx, int32_t* pairs, int64_t cap, int64_t* npairs);
/* linked_list.cpp:192-281: blob_forces(3Nb) += steric forces. */
int fcm_apply_barrier_forces(fcm_ctx* ctx, double* blob_forces);

/* ================================================================ fcm_fluid_solver */
/* fcm_fluid_solver.cpp:131-165 on Y (Nb*3; NULL = all_blob_pos). */
int fcm_set_up_gaussians(fcm_ctx* ctx, const double* Y);
/* The tables of the last fcm_set_up_gaussians (fcm_fluid_solver.cpp:131-165) on
 * the grid of one precision (0 = FP64; 1 = FP32, in a context of precision 1,
 * whose stencil may be narrower): ind (Nb*3*W, may be NULL) the periodic grid
 * indices indx/indy/indz of every blob, dimension and stencil point, w (Nb*3*W,
 * may be NULL) the weights gaussx/y/z; W is the stencil width of that grid
 * (ngauss for FP64). */
int fcm_get_gaussians(fcm_ctx* ctx, int32_t precision, int32_t* ind, double* w);
/* fcm_fluid_solver.cpp:167-361 with the stress drawn from a counter-based
 * Philox4x32-10 stream keyed by (seed, counter). */
int fcm_produce_random_velocity_field(fcm_ctx* ctx, uint64_t seed, uint64_t counter);
/* fcm_fluid_solver.cpp:167-361 with the six stress arrays supplied by the caller
 * (the reference's sxx..syz after the fill at :174-234, each nx*ny*pad doubles). */
int fcm_inject_random_stress(fcm_ctx* ctx, const double* sxx, const double* syy,
                             const double* szz, const double* sxy,
                             const double* sxz, const double* syz);
/* fcm_fluid_solver.cpp:426-487: V(3Nb) = J u_rand (NULL keeps it in the context). */
int fcm_calculate_random_blob_velocities(fcm_ctx* ctx, double* V);
/* fcm_fluid_solver.cpp:552-634: spread F (3Nb) onto the force grids. */
int fcm_set_up_force_distribution(fcm_ctx* ctx, const double* F);
/* fcm_fluid_solver.cpp:636-701: Stokes solve of the force grids. */
int fcm_produce_deterministic_velocity_field(fcm_ctx* ctx);
/* fcm_fluid_solver.cpp:363-424: V(3Nb) = J u (NULL keeps it in the context). */
int fcm_calculate_deterministic_blob_velocities(fcm_ctx* ctx, double* V);
/* The context's last interpolated velocities (fcm.V) to V (3Nb). */
int fcm_get_V(fcm_ctx* ctx, double* V);
/* Velocity grids u{x,y,z} (deterministic: which=0, random: which=1, imposed shear
 * flow: which=2) in the reference's padded [x][y][pad] layout, 3 arrays of
 * nx*ny*pad doubles. */
int fcm_get_velocity_field(fcm_ctx* ctx, int32_t which, double* ux, double* uy, double* uz);
/* M*F in one call: spread, Stokes solve, interpolation (V = 3Nb). */
int fcm_apply_mobility(fcm_ctx* ctx, const double* F, double* V);
/* Force dipoles -- no reference counterpart (the reference spreads forces only).
 * The FCM dipole terms (Lomholt & Maxey, J. Comput. Phys. 184 (2003)) on the FP64
 * deterministic grid: blob forces F (3Nb), torques T (3Nb) and stresslets S
 * (9Nb, row-major, symmetric) -- each may be NULL for zero -- spread with the force
 * envelope (F) and the dipole envelope sigma_D = a / (6 sqrt(pi))^(1/3) (the
 * dipole D = S - 1/2 eps.T as f_i = D_ij (x_j - Y_j)/sigma_D^2 Delta_D).  After
 * fcm_produce_deterministic_velocity_field, V comes from
 * fcm_calculate_deterministic_blob_velocities and the blob rotation rates Omega
 * (3Nb) and strain rates E (9Nb, row-major) from
 * fcm_calculate_deterministic_blob_rotations (either output may be NULL).
 * Positions are those of the last fcm_set_up_gaussians; the grid must be one the
 * tiled kernels take (dimensions multiples of 8, ngauss + 8 <= n, ngauss <= 25).
 * The dipole envelope is narrower than the force envelope: resolve it with
 * dx <= a/2 or finer for accurate rotation rates. */
int fcm_set_up_dipole_distribution(fcm_ctx* ctx, const double* F, const double* T, const double* S);
int fcm_calculate_deterministic_blob_rotations(fcm_ctx* ctx, double* Omega, double* E);

/* Shear forcing (SHEARING_FORCES, config.hpp:32, :52-56).
 * fcm_produce_shear_velocity_field replaces fcm_fluid_solver.cpp:703-842: the
 * Stokes flow u_shear driven by the body force
 * fx = scale * kT * sin(wavenumber * 2 pi j / ny) / a (fy = fz = 0) on every grid
 * point -- scale and wavenumber are SHEAR_FORCE_SCALE and SHEAR_WAVENUMBER -- solved
 * once, as main.cpp:98-100 does at start-up.  From then on every RHS subtracts
 * Vshear (gmres_solver.cpp:62-64), and a GDC step interpolates u_shear at the
 * midstep (main.cpp:270-272) before its solve; an EM step, like the reference's,
 * never does, so it uses the Vshear last computed (zero until
 * fcm_calculate_shear_blob_velocities is called).  The deterministic grids are
 * left holding the shear solve.
 * fcm_calculate_shear_blob_velocities replaces fcm_fluid_solver.cpp:489-550:
 * Vshear (3Nb, may be NULL) = J u_shear on the current Gaussians; fcm.V is kept.
 * fcm_fluid_x_velocity_in_y replaces main.cpp:371-433: spread F (3Nb) on the
 * current Gaussians, solve, and write profile[j] (ny doubles) = the mean over x
 * and z of ux + ux_shear at y index j (ux alone without a shear flow). */
int fcm_produce_shear_velocity_field(fcm_ctx* ctx, double scale, double wavenumber);
int fcm_calculate_shear_blob_velocities(fcm_ctx* ctx, double* Vshear);
int fcm_fluid_x_velocity_in_y(fcm_ctx* ctx, const double* F, double* profile);

/* The three stages of M*F one at a time on the working grid of one precision
 * (0 = FP64, 1 = FP32, which needs a context of precision 1): spread F (3Nb),
 * Stokes solve of that grid in place, interpolation of it into V (3Nb).  The
 * FP64 stages are those of fcm_set_up_force_distribution,
 * fcm_produce_deterministic_velocity_field and
 * fcm_calculate_deterministic_blob_velocities; no reference counterpart for FP32. */
int fcm_spread(fcm_ctx* ctx, int32_t precision, const double* F);
int fcm_stokes_solve(fcm_ctx* ctx, int32_t precision);
int fcm_interp(fcm_ctx* ctx, int32_t precision, double* V);

/* Kernel variants of the grid stages (no reference counterpart).
 * variants[FCM_NUM_VARIANTS]:
 *   [0] FP64 spread, [2] FP32 spread: 0 = the persistent software-pipelined tile
 *       kernel, 1 / 2 / 3 = one CTA per 8^3 tile staging 16 / 8 / 32 blobs per
 *       round, 4 = one warp per tile staging 16 blobs per round, two y-rows per
 *       lane.  All sum every grid point's blobs in the same order with the same
 *       products, so the grids are the same bit for bit.  FP32 only: 5 = one warp
 *       per tile on the tensor cores (mma.sync with TF32 operands split in two,
 *       3xTF32, FP32 accumulators), equal to the others to FP32 rounding.
 *   [1] FP64 Stokes solve, [3] FP32 Stokes solve: 0 = cuFFT 3D transforms and the
 *       projection kernel, 1 = cuFFT (y, z) transforms around the fused x-transform
 *       + projection kernel, 2 = the library's own (y, z) transforms around it
 *       (FP32 only).  FP64 defaults to 0 beyond 256 points along x.  The solves
 *       agree within rounding.
 *   [4] FP64 interpolation, [5] FP32 interpolation: 0 = 64 threads per 8^3 tile
 *       with a warp shuffle reduction, 1 = one warp per tile (two y-rows per
 *       lane, added in the lane) with the shuffle reduction, 2 = one warp per tile
 *       (two y-rows per thread) with a shared-memory reduction; FP32 only: 3 = one
 *       warp per tile on the tensor cores (3xTF32).  They agree within rounding.
 * Defaults: spread 0 (FP64) and 4 (FP32), solve 1 (FP64 up to 256 points along
 * x, else 0) and 2 (FP32, where the grid allows, else 1 or 0), interpolation 1.
 * A variant the grid does not allow (solve 1 and 2 need supported lengths, 2 also
 * nz <= 512) or out of range is refused with FCM_ERR_INVALID; the spread and
 * interpolation entries have no effect where the grid is not tiled, the FP32
 * entries none in a context without an FP32 grid (they are still range-checked).
 * Step graphs are rebuilt on the next step.  Refused for a context owned by a
 * batch. */
#define FCM_NUM_VARIANTS 6
int fcm_get_variants(fcm_ctx* ctx, int32_t* variants);
int fcm_set_variants(fcm_ctx* ctx, const int32_t* variants);
/* Times every variant the grids allow on this context (reps timed calls of each,
 * 5 when reps <= 0, after one untimed call; zero forces, zeroed grids) and keeps
 * the fastest per stage and precision.  us (may be NULL) receives
 * FCM_NUM_TUNE_TIMES doubles, [16 P + v] for precision P (0 FP64, 1 FP32): v = 0..5
 * the spread variants, v = 6, 7, 8 the solve variants 0, 1, 2, v = 9..12 the
 * interpolation variants 0..3, in microseconds per call, -1 where not available
 * (FP64 v = 5 and 12, v = 13..15 always); variants (may be NULL) receives the
 * choice as fcm_get_variants does.
 * Needs set_up_gaussians first; overwrites the grid work arrays, so call it
 * between steps. */
#define FCM_NUM_TUNE_TIMES 32
int fcm_autotune(fcm_ctx* ctx, int32_t reps, double* us, int32_t* variants);
/* fcm_fluid_solver.cpp:842-881: single-body mobility at the box centre,
 * ref_Minv = inv_sympd(M_body) ((3nb)^2), ref_N = inv(K^T ref_Minv K) (6x6). */
int fcm_produce_reference_matrices(fcm_ctx* ctx);
/* Column-major ref_Minv ((3nb)^2), ref_N (36), ref_KTKinv (36); any may be NULL. */
int fcm_get_reference_matrices(fcm_ctx* ctx, double* ref_Minv, double* ref_N, double* ref_KTKinv);
int fcm_set_reference_matrices(fcm_ctx* ctx, const double* ref_Minv, const double* ref_N);

/* Per-body shapes.  No counterpart in the reference: its collection has one
 * blob_ref_pos for every body (collection_of_rigid_bodies.hpp:24) and one probed
 * preconditioner reference (fcm_fluid_solver.cpp:842-881).  shapes (3*nb*M)
 * holds body n's reference blob positions at 3*nb*n (the same blob-major layout
 * as blob_ref_pos); every body keeps nb blobs, so blob i still belongs to body
 * i/nb (linked_list.cpp:106,118).  From then on blob positions, K, K^T, the
 * preconditioner and the GDC rigid projection use each body's own shape, each
 * body gets its own ref_KTKinv = inv(K^T K) (collection_of_rigid_bodies.cpp:
 * 117-130 per body), and the Metropolis rotation scale is the largest blob
 * distance over all shapes.  Probing 3*nb FCM solves per shape
 * (fcm_produce_reference_matrices) is out of reach for thousands of shapes, so
 * each body's ref_Minv is the inverse of its blob-blob mobility computed with the
 * free-space FCM pair mobility of two Gaussian envelopes (sigma = a/sqrt(pi)):
 *   M(r) = [A I + B rr/r^2] / (8 pi eta r), s^2 = 2 sigma^2,
 *   A = (1 + s^2/r^2) erf(r/(sqrt2 s)) - sqrt(2/pi)(s/r) exp(-r^2/2s^2),
 *   B = (1 - 3s^2/r^2) erf(r/(sqrt2 s)) + 3 sqrt(2/pi)(s/r) exp(-r^2/2s^2),
 *   M(0) = I/(6 pi eta a),
 * and ref_N = inv(K^T ref_Minv K) (pseudo-inverse for collinear blobs).  The
 * preconditioner changes GMRES's iteration count, never its solution.
 * fcm_set_body_preconditioners replaces ref_Minv (M*(3nb)^2, body-major,
 * column-major blocks) and/or ref_N (36*M); fcm_get_body_preconditioners reads
 * them and the per-body ref_KTKinv (36*M).  After fcm_set_body_shapes the
 * single-shape calls fcm_produce/get/set_reference_matrices are refused
 * (FCM_ERR_STATE); not available to batch members. */
int fcm_set_body_shapes(fcm_ctx* ctx, const double* shapes);
int fcm_set_body_preconditioners(fcm_ctx* ctx, const double* Minv, const double* N);
int fcm_get_body_preconditioners(fcm_ctx* ctx, double* Minv, double* N, double* KTKinv);

/* ================================================================ gmres_solver */
/* gmres_solver.cpp:58-70: RHS = [-V ; -K^T blob_forces - external]. */
int fcm_assemble_RHS(fcm_ctx* ctx);
int fcm_get_RHS(fcm_ctx* ctx, double* rhs);
int fcm_set_RHS(fcm_ctx* ctx, const double* rhs);
/* gmres_solver.cpp:85-146 (system vectors, 3Nb+6M). */
int fcm_multiply_by_Pinv(fcm_ctx* ctx, const double* in, double* out);
/* gmres_solver.cpp:72-83. */
int fcm_multiply_by_saddle_point_matrix(fcm_ctx* ctx, const double* in, double* out);
/* gmres_solver.cpp:148-306: right-preconditioned GMRES(max_iter) on the stored
 * RHS; soln (3Nb+6M, may be NULL) receives P^{-1} sum y_i q_i.  Returns FCM_OK,
 * FCM_ERR_NOT_CONVERGED (solution still written) or an error. */
int fcm_invert_saddle_point_system(fcm_ctx* ctx, double* soln, int32_t* iters,
                                   double* rel_residual);

/* ================================================================ time step */
/* One accepted-or-rejected time step of main.cpp:222-451 for the configured
 * algorithm (EM or GDC), noise from Philox (seed, counter=step index) when
 * params.noise is 1.  Returns FCM_OK or FCM_ERR_OVERLAP (state restored). */
int fcm_step(fcm_ctx* ctx, uint64_t seed, uint64_t step_index, fcm_step_info* info);

/* Asynchronous steps.  fcm_step_async issues the step of fcm_step without
 * waiting for it; fcm_step_wait waits and returns its status and record (one step
 * in flight per context; fcm_step refuses while one is).  The first step issued
 * on a context runs host-driven, after which the whole step is captured in one
 * CUDA graph whose GMRES iterations and refinement sweeps are device-side
 * conditional loops (at most gmres_max_iter iterations per solve and 8 sweeps),
 * and later steps launch that graph on the context's stream: no host round trip
 * inside a step.  Contexts with skip_on_overlap = 1 keep host-driven steps.  A
 * step whose solve fails (non-finite residual) leaves the bodies as they were,
 * as fcm_step does.  No reference counterpart (main.cpp:222-451 steps
 * synchronously). */
int fcm_step_async(fcm_ctx* ctx, uint64_t seed, uint64_t step_index);
int fcm_step_wait(fcm_ctx* ctx, fcm_step_info* info);
/* collection_of_rigid_bodies.cpp:666-705 with linked_list.cpp:283-360: the
 * pair potential of the current bodies (blob positions and cells refreshed),
 * using the MARKOV_CHAIN_MONTE_CARLO energy forms of linked_list.cpp:362-497 for
 * potentials 0-2 and, for potential 3, the energy whose force is that potential's
 * polynomial.  Each pair of blobs of different bodies in adjacent cells counts once. */
int fcm_calculate_potential(fcm_ctx* ctx, double* U);
/* main.cpp:113-210: n_steps Metropolis steps of global rigid-body moves, on the
 * device (one CUDA graph, the loop conditional on the device).  Each step moves
 * every body by dt * scale * (2u - 1) per component (rotations divided by the
 * body radius), accepts with probability min(1, exp((U_old - U)/kT)), updates the
 * running acceptance ratio over 20 steps and scales `scale` by 1.02 above a
 * ratio of 0.5 and 0.98 otherwise.  With skip_on_overlap a proposal that
 * overlaps is undone and drawn again without counting.  The uniforms are
 * Philox4x32-10 (seed, state->attempts), so runs continue exactly across calls.
 * fcm_mcmc_state_init sets the reference's starting scale and ratio. */
int fcm_mcmc_state_init(const fcm_ctx* ctx, fcm_mcmc_state* state);
int fcm_mcmc_run(fcm_ctx* ctx, uint64_t seed, int64_t n_steps, fcm_mcmc_state* state);

/* Batches: n independent suspensions (members, each with its own params and
 * blob_ref_pos; body counts and grids may differ, precision and gmres_tol are
 * common, skip_on_overlap must be 0) stepped together.  Per-member work runs
 * concurrently; the saddle-point solves run in lockstep as batched kernels
 * (one spread, projection and interpolation launch over every member, one
 * cuFFT plan per group of members with equal grids, the GMRES vector work of
 * all members per launch), members whose solve is done being skipped, and a
 * step is one CUDA graph whose GMRES iterations and refinement sweeps loop on
 * the device until every member is done.  The first fcm_batch_step runs the
 * members host-driven and captures that graph.  Each member's solve and
 * trajectory are those of fcm_step on the same member.  No reference
 * counterpart. */
typedef struct fcm_batch fcm_batch;
int fcm_batch_create(int32_t n, const fcm_params* params, const double* const* blob_ref_pos, fcm_batch** out);
int fcm_batch_destroy(fcm_batch* b);
/* Member i as a context (owned by the batch: set bodies, forces, reference
 * matrices, read results through it; fcm_destroy refuses it). NULL if out of range. */
fcm_ctx* fcm_batch_member(fcm_batch* b, int32_t i);
/* Stream of the batch's graph launches (a cudaStream_t, 0 = legacy). */
int fcm_batch_set_stream(fcm_batch* b, void* stream);
/* One step of every member: seeds[i] for member i, the same step_index; infos
 * (n records) may be NULL.  Returns FCM_OK or the first failing status (a member
 * whose solve failed keeps its bodies). */
int fcm_batch_step(fcm_batch* b, const uint64_t* seeds, uint64_t step_index, fcm_step_info* infos);
/* Lockstep rounds of the last graph step: rounds[0] GMRES iterations (summed
 * over sweeps), rounds[1] refinement sweeps (0 for FP64 batches); both 0 before
 * the first graph step.  A member's own counts are in its fcm_step_info. */
int fcm_batch_last_rounds(const fcm_batch* b, int32_t* rounds);

/* One step of each of n independent suspensions (seeds[i] for context i, the
 * same step_index): all issued, then all awaited, so contexts on different
 * streams run concurrently.  infos (n records) may be NULL.  Returns FCM_OK or
 * the first failing status. */
int fcm_step_many(fcm_ctx* const* ctxs, int32_t n, const uint64_t* seeds, uint64_t step_index,
                  fcm_step_info* infos);

/* ================================================================ allocation-free interpolation
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory -- a time-step loop that must not stall the device (cudaMalloc and
 * cudaFree synchronise it), or an application whose device memory all belongs to
 * its own allocator or pool -- this interpolates a caller-owned velocity grid
 * onto blobs without allocating anything:
 *   V_c(blob) = DX^3 * sum over the blob's W^3 stencil points of
 *               u_c(point) * gx(point) * gy(point) * gz(point),
 * with the separable Gaussian weights g(x) = exp(-pi (x - Y)^2 / (2 a^2)) /
 * (sqrt(2) a) on the W grid points nearest each blob coordinate Y.  The grid is
 * fully periodic: there is no slip-channel truncation of the Gaussians, so the
 * result equals a context's interpolation only for a periodic box (slip_channel
 * 0).  Y (nblobs*3), grid (3*nx*ny*nz, component-major [3][nx][ny][nz],
 * unpadded) and V must be DEVICE pointers of the current device (or managed
 * memory); work is issued on `stream` (a cudaStream_t, 0 = legacy).
 * Limits: nblobs <= 8192, ngauss <= 24, nx, ny, nz multiples of 8 with
 * ngauss + 8 <= n, and at most 32768 8^3 tiles (a 256^3 grid); larger inputs are
 * rejected with FCM_ERR_INVALID.  Scratch is a fixed 32 MiB device array inside the
 * library, held by every GPU that loads it until exit.  The first call on a device
 * looks up that array's device address (once per device), so make the first call
 * before any stream capture; the address is kept for the process's lifetime, so
 * do not use this call after cudaDeviceReset in the same process.  Every call
 * shares the array: calls that may overlap on the GPU (different streams, no
 * ordering between them) race. */
int fcm_interp_noalloc(int32_t nx, int32_t ny, int32_t nz, double dx, double blob_radius, int32_t ngauss,
                       int32_t nblobs, const double* Y, const double* grid, double* V, void* stream);

/* ================================================================ bounds-checked build
 * No counterpart in the reference (which has no device code).  The library is
 * also built with every device index checked (libfcm_b200_debug.so, same entry
 * points): grid point indices against the grid, blob ids read from the tile and
 * cell lists against the blob count, tile and cell ids, tile-list and cell-list
 * slots against their ranges and capacities, per-(blob, tile) partials, spectrum
 * indices of the fused x-transform and projection, and Krylov columns against the
 * columns allocated.  A kernel that meets an index outside its range counts it,
 * keeps the first one's site, index and limit, skips the access and runs on: no
 * trap, no assert.  This call waits for the current device, then writes
 * *checked = 1 in the checked build (0 in the release build, whose counts are
 * always zero), the number of violations on the current device since the last
 * reset, and the first one's site (1 grid point, 2 blob id, 3 tile id, 4 list
 * slot, 5 partial, 6 cell id, 7 spectrum index, 8 Krylov column; 0 none), index
 * and limit; reset != 0 then clears the counts.  Any output pointer may be NULL.
 * Returns FCM_OK or FCM_ERR_CUDA. */
#define FCM_BOUNDS_SITES 8
int fcm_debug_bounds(int32_t* checked, int64_t* count, int32_t* site, int64_t* index, int64_t* limit,
                     int32_t reset);

#ifdef __cplusplus
}
#endif

#endif /* FCM_B200_H */
