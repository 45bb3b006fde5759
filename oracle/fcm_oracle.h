/*
 * fcm_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * C API of the CPU FP64 restatement of the reference's FCM mobility path
 * (fcm_fluid_solver.cpp, fft_solver.cpp, gmres_solver.cpp, linked_list.cpp,
 * collection_of_rigid_bodies.cpp, particle.cpp, quaternion.cpp, rcross.cpp and
 * the main.cpp time loop), with the MPI decomposition collapsed to one rank.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load
 * it, and only as the checker / the reported CPU baseline.  The product path
 * (timstochrigidbodiessim_b200) never calls it.
 *
 * Parity status: the reference cannot be built here (it needs MPI, Armadillo,
 * FFTW 2.x MPI and SPRNG, none of which are present) and it ships no tests,
 * fixtures or golden vectors.  This restatement is therefore pinned by
 * known-answer checks instead (numpy FFTs for the FFTW 2.x transform semantics,
 * the Hasimoto periodic self-mobility, operator identities), see tests/.
 * Against the reference's own outputs it is "parity unpinned".
 *
 * The array layouts are those of include/fcm_b200.h.
 */
#ifndef FCM_ORACLE_H
#define FCM_ORACLE_H

#include <stdint.h>
#include "../include/fcm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc orc;

/* Threads used by the FFT / grid loops (default: 1, as one reference MPI rank
 * with OPENBLAS_NUM_THREADS=1). */
void orc_set_threads(int n);
int orc_get_threads(void);

/* fft_solver with FFTW 2.x rfftwnd_mpi semantics on one rank. */
int orc_fft_transform(int nx, int ny, int nz, double* in);          /* fft_solver.cpp:32-36 */
int orc_fft_inverse_transform(int nx, int ny, int nz, double* in);  /* fft_solver.cpp:38-42 */

orc* orc_create(const fcm_params* p, const double* blob_ref_pos);
void orc_destroy(orc* o);

void orc_set_bodies(orc* o, const double* x, const double* q);
void orc_get_bodies(orc* o, double* x, double* q);
void orc_get_midstep_bodies(orc* o, double* x, double* q);
void orc_set_external_forces(orc* o, const double* fe);
void orc_fill_all_blob_pos(orc* o, int at_midstep);
void orc_set_all_blob_pos(orc* o, const double* Y);
void orc_get_all_blob_pos(orc* o, double* Y);
void orc_multiply_by_K_at_midstep(orc* o, const double* in, double* out);
void orc_multiply_by_KT_at_midstep(orc* o, const double* in, double* out);
void orc_calculate_forces(orc* o);
void orc_get_blob_forces(orc* o, double* F);
void orc_set_blob_forces(orc* o, const double* F);
int orc_advance_to_midstep(orc* o, const double* V);
double orc_calculate_divU(orc* o);
int orc_end_of_step_update(orc* o, const double* U, double nu);
void orc_reset_to_start_of_step(orc* o);
int orc_check_for_overlap(orc* o);

void orc_list_populate(orc* o);
void orc_list_get_cells(orc* o, int32_t* cell_of_blob);
int64_t orc_list_get_pairs(orc* o, int32_t* pairs, int64_t cap);
void orc_apply_barrier_forces(orc* o, double* blob_forces);

void orc_set_up_gaussians(orc* o, const double* Y);
void orc_get_gaussians(orc* o, int32_t* ind, double* w);   /* each Nb*3*W: [np][dim][i] */
void orc_inject_random_stress(orc* o, const double* sxx, const double* syy, const double* szz,
                              const double* sxy, const double* sxz, const double* syz);
/* Real-space stress from Philox normals (polar method), as the reference fills
 * it at fcm_fluid_solver.cpp:174-234, then the same solve as inject. */
void orc_produce_random_velocity_field(orc* o, uint64_t seed, uint64_t counter);
void orc_calculate_random_blob_velocities(orc* o, double* V);
void orc_set_up_force_distribution(orc* o, const double* F);
void orc_produce_deterministic_velocity_field(orc* o);
void orc_calculate_deterministic_blob_velocities(orc* o, double* V);
/* Force dipoles (no reference code): forces F (3Nb or NULL), torques T (3Nb or
 * NULL) and stresslets S (9Nb row-major, or NULL) spread with the dipole envelope;
 * then Omega (3Nb) and E (9Nb) of the deterministic field. */
void orc_set_up_dipole_distribution(orc* o, const double* F, const double* T, const double* S);
void orc_calculate_deterministic_blob_rotations(orc* o, double* Om, double* E);
/* Shear forcing (fcm_fluid_solver.cpp:703-842, :489-550; main.cpp:371-433):
 * produce the imposed flow once; afterwards GDC steps interpolate it at the
 * midstep and every RHS subtracts Vshear. */
void orc_produce_shear_velocity_field(orc* o, double scale, double wavenumber);
void orc_calculate_shear_blob_velocities(orc* o, double* Vshear);
void orc_fluid_x_velocity_in_y(orc* o, const double* F, double* profile);
/* Pair potential of the current bodies, and Metropolis runs (main.cpp:113-210)
 * with the same Philox uniforms as the GPU library. */
double orc_calculate_potential(orc* o);
int orc_mcmc_run(orc* o, uint64_t seed, int64_t n_steps, fcm_mcmc_state* st);
void orc_get_V(orc* o, double* V);
void orc_get_grid(orc* o, int which, double* out);  /* 0..2 fx,fy,fz 3..5 ux,uy,uz 6..8 u*_rand */
void orc_produce_reference_matrices(orc* o);
void orc_get_reference_matrices(orc* o, double* ref_Minv, double* ref_N, double* ref_KTKinv);
void orc_set_reference_matrices(orc* o, const double* ref_Minv, const double* ref_N);
/* Per-body shapes (3*nb per body) with per-body ref_KTKinv and preconditioner
 * blocks; no counterpart in the reference. */
void orc_set_body_shapes(orc* o, const double* shapes);
void orc_set_body_preconditioners(orc* o, const double* Minv, const double* N);
void orc_get_body_preconditioners(orc* o, double* Minv, double* N, double* KTKinv);
void orc_produce_body_preconditioners(orc* o);
/* Noise from one stream continued across calls (on = 1): the stress of every
 * plane drawn in plane order from UniformStream(seed, stream), as one reference
 * rank draws from its SPRNG stream; produce_random_velocity_field's own seed and
 * counter are then not used.  on = 0 returns to per-plane streams. */
void orc_set_sequential_noise(orc* o, int on, uint64_t seed, uint64_t stream);

void orc_assemble_RHS(orc* o);
void orc_get_RHS(orc* o, double* rhs);
void orc_set_RHS(orc* o, const double* rhs);
void orc_multiply_by_Pinv(orc* o, const double* in, double* out);
void orc_multiply_by_saddle_point_matrix(orc* o, const double* in, double* out);
int orc_invert_saddle_point_system(orc* o, double* soln, int* iters, double* rel_residual);

/* main.cpp:222-451, one step; noise from orc_produce_random_velocity_field
 * (seed, step_index) when params.noise is 1.  Returns 0, or 7 on overlap. */
int orc_step(orc* o, uint64_t seed, uint64_t step_index, fcm_step_info* info);
/* Same step with the stress injected (six arrays as orc_inject_random_stress);
 * GDC reuses the injected field for every interpolation of the step. */
int orc_step_injected(orc* o, const double* s6, fcm_step_info* info);

#ifdef __cplusplus
}
#endif
#endif
