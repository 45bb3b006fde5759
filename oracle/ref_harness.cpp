// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY.  C entry points over the
// reference's own classes (collection_of_rigid_bodies, fcm_fluid_solver,
// gmres_solver, linked_list), compiled unchanged from the reference's sources
// with the stand-in headers of oracle/ref_shim and one of its config.hpp files
// (recipe: oracle/Makefile, target `ref`; output oracle/_ref/libref_<config>.so).
// The functions only call the reference's methods, in the order main.cpp calls
// them; every number they return is computed by the reference's code.  The
// fixtures made from them (tests/golden/make_ref_golden.py) pin the oracle.
#include <armadillo>
#include <cstring>

#include "collection_of_rigid_bodies.hpp"
#include "config.hpp"
#include "fcm_fluid_solver.hpp"
#include "gmres_solver.hpp"
#include "sprng.h"

namespace {
collection_of_rigid_bodies* C = nullptr;
fcm_fluid_solver* F = nullptr;
gmres_solver* G = nullptr;

void copy_out(const arma::mat& a, double* out) { std::memcpy(out, a.memptr(), sizeof(double) * a.n_elem); }
}  // namespace

extern "C" {

// collection_of_rigid_bodies::initialise, fcm_fluid_solver::initialise and
// gmres_solver::initialise (main.cpp:73-107); returns blobs per body.
int rh_init(void) {
  if (!C) {
    C = new collection_of_rigid_bodies();
    C->initialise(0, 1);
    F = new fcm_fluid_solver();
    F->initialise(C->total_num_blobs);
    G = new gmres_solver();
    G->initialise(C->total_num_blobs);
  }
  return C->blobs_per_body;
}

// The compile-time parameters of this build.
void rh_config(double* o) {
  o[0] = NUM_BODIES;
  o[1] = C->blobs_per_body;
  o[2] = NUM_FFT_GRID_POINTS_X;
  o[3] = NUM_FFT_GRID_POINTS_Y;
  o[4] = NUM_FFT_GRID_POINTS_Z;
  o[5] = DX;
  o[6] = BLOB_RADIUS;
  o[7] = FLUID_VISCOSITY;
  o[8] = ENERGY_SCALE;
  o[9] = DT;
  o[10] = GMRES_TOL;
  o[11] = GMRES_MAX_ITER;
  o[12] = NUM_FCM_GAUSSIAN_POINTS;
  o[13] = NUM_LINKED_LIST_CELLS_PER_DIM;
  o[14] = SLIP_CHANNEL ? 1 : 0;
  o[15] = SIMULATION_ALGORITHM;
  o[16] = INTERACTION_POTENTIAL_TYPE;
  o[17] = FINITE_DIFFERENCE_DELTA_FACTOR;
  o[18] = SKIP_ON_OVERLAP ? 1 : 0;
}

// blob_ref_pos (3 x nb) as 3*nb values, blob after blob.
void rh_blob_ref_pos(double* out) { copy_out(C->blob_ref_pos, out); }

// Set the bodies and populate the cell list from their blobs, as seed_the_bodies
// does (collection_of_rigid_bodies.cpp:428-429).  The reference populates the
// list only there, at the midstep and at the end of a step (:609, :778), so an
// Euler-Maruyama run started from a state file reaches calculate_forces with a
// never-populated list (all-zero head and next arrays) and its traversal loops
// forever; the harness populates it here.
void rh_set_bodies(const double* x, const double* q) {
  for (int n = 0; n < NUM_BODIES; ++n) {
    C->bodies[n].x = {x[3 * n], x[3 * n + 1], x[3 * n + 2]};
    C->bodies[n].q = quaternion(q[4 * n], q[4 * n + 1], q[4 * n + 2], q[4 * n + 3]);
  }
  C->midstep_bodies = C->bodies;
  C->fill_all_blob_pos();
  C->list.populate(C->all_blob_pos);
}

void rh_get_bodies(double* x, double* q) {
  for (int n = 0; n < NUM_BODIES; ++n) {
    for (int d = 0; d < 3; ++d) x[3 * n + d] = C->bodies[n].x(d);
    q[4 * n] = C->bodies[n].q.scalar_part;
    for (int d = 0; d < 3; ++d) q[4 * n + 1 + d] = C->bodies[n].q.vector_part(d);
  }
}

// fcm_fluid_solver.cpp:842-881; matrices column-major.
void rh_produce_reference_matrices(void) { F->produce_reference_matrices(*C); }
void rh_get_reference_matrices(double* Minv, double* N, double* KTKinv) {
  if (Minv) copy_out(F->ref_Minv, Minv);
  if (N) copy_out(F->ref_N, N);
  if (KTKinv) copy_out(C->ref_KTKinv, KTKinv);
}
void rh_set_reference_matrices(const double* Minv, const double* N) {
  const int n3 = 3 * C->blobs_per_body;
  F->ref_Minv = arma::mat(n3, n3);
  std::memcpy(F->ref_Minv.memptr(), Minv, sizeof(double) * n3 * n3);
  F->ref_N = arma::mat(6, 6);
  std::memcpy(F->ref_N.memptr(), N, sizeof(double) * 36);
}

void rh_sprng_reset(uint64_t seed, uint64_t stream) { ref_sprng_reset(seed, stream); }

// all_blob_pos (collection_of_rigid_bodies.cpp:155-174), blob after blob.
void rh_blob_positions(double* Y) {
  C->fill_all_blob_pos();
  for (int i = 0; i < C->total_num_blobs; ++i)
    for (int d = 0; d < 3; ++d) Y[3 * i + d] = C->all_blob_pos(i, d);
}

// fcm_fluid_solver.cpp:131-165 at all_blob_pos: ind and w as [blob][dim][W].
void rh_gaussians(int* ind, double* w) {
  C->fill_all_blob_pos();
  F->set_up_gaussians(C->all_blob_pos);
  const int W = NUM_FCM_GAUSSIAN_POINTS;
  for (int b = 0; b < C->total_num_blobs; ++b)
    for (int i = 0; i < W; ++i) {
      ind[(3 * b + 0) * W + i] = F->indx(b, i);
      ind[(3 * b + 1) * W + i] = F->indy(b, i);
      ind[(3 * b + 2) * W + i] = F->indz(b, i);
      w[(3 * b + 0) * W + i] = F->gaussx(b, i);
      w[(3 * b + 1) * W + i] = F->gaussy(b, i);
      w[(3 * b + 2) * W + i] = F->gaussz(b, i);
    }
}

// M F at all_blob_pos: spread, Stokes solve, interpolation (fcm_fluid_solver.cpp:
// 552-701, :363-424).
void rh_mobility(const double* Fin, double* Vout) {
  C->fill_all_blob_pos();
  F->set_up_gaussians(C->all_blob_pos);
  arma::vec f(3 * C->total_num_blobs);
  std::memcpy(f.memptr(), Fin, sizeof(double) * f.n_elem);
  F->set_up_force_distribution(f);
  F->produce_deterministic_velocity_field();
  F->calculate_deterministic_blob_velocities();
  copy_out(F->V, Vout);
}

// The random velocity field from the SPRNG stream as it stands
// (fcm_fluid_solver.cpp:167-361) and its interpolation (:426-487).
void rh_random_velocities(double* Vout) {
  C->fill_all_blob_pos();
  F->produce_random_velocity_field();
  F->set_up_gaussians(C->all_blob_pos);
  F->calculate_random_blob_velocities();
  copy_out(F->V, Vout);
}

// collection_of_rigid_bodies.cpp:623-664 at time t: the blob forces.
void rh_forces(double t, double* Fout) {
  C->fill_all_blob_pos();
  C->calculate_forces(t);
  copy_out(C->blob_forces, Fout);
}

double rh_potential(void) {
  C->fill_all_blob_pos();
  return C->calculate_potential();
}

// The cell of every blob (linked_list.cpp:74-78) at all_blob_pos.
void rh_cells(int* cells) {
  C->fill_all_blob_pos();
  for (int i = 0; i < C->total_num_blobs; ++i) cells[i] = C->list.find_containing_cell(C->all_blob_pos.row(i));
}

// K and K^T at the midstep bodies (collection_of_rigid_bodies.cpp:707-757).
void rh_multiply_K(const double* in, double* out) {
  arma::vec v(6 * NUM_BODIES);
  std::memcpy(v.memptr(), in, sizeof(double) * v.n_elem);
  copy_out(C->multiply_by_K_at_midstep(v), out);
}
void rh_multiply_KT(const double* in, double* out) {
  arma::vec v(3 * C->total_num_blobs);
  std::memcpy(v.memptr(), in, sizeof(double) * v.n_elem);
  copy_out(C->multiply_by_KT_at_midstep(v), out);
}

// gmres_solver.cpp:85-146 and :72-83 on a system vector (the saddle-point
// product at all_blob_pos's Gaussians).
void rh_multiply_by_Pinv(const double* in, double* out) {
  arma::vec v(3 * C->total_num_blobs + 6 * NUM_BODIES);
  std::memcpy(v.memptr(), in, sizeof(double) * v.n_elem);
  copy_out(G->multiply_by_Pinv(v, *C, *F), out);
}
void rh_multiply_by_saddle_point_matrix(const double* in, double* out) {
  C->fill_all_blob_pos();
  F->set_up_gaussians(C->all_blob_pos);
  arma::vec v(3 * C->total_num_blobs + 6 * NUM_BODIES);
  std::memcpy(v.memptr(), in, sizeof(double) * v.n_elem);
  copy_out(G->multiply_by_saddle_point_matrix(v, *C, *F), out);
}

// One time step in main.cpp:222-340's order of calls (rigid bodies, no shear
// forcing), the noise drawn from the SPRNG stream as it stands.  soln receives
// the saddle-point solution (3Nb + 6M); *nu_out the GDC factor nu (1 for EM).
// Returns 0, or 1 / 2 when the step was restarted at the midstep / at its end
// (the bodies are then as main.cpp leaves them before its `continue`).
int rh_step(double t, double* soln_out, double* nu_out) {
  C->fill_all_blob_pos();
  F->produce_random_velocity_field();
  F->set_up_gaussians(C->all_blob_pos);
  F->calculate_random_blob_velocities();
  double nu = 1.0;
#if GEN_DRIFTER_CORRECTOR
  if (C->advance_to_midstep(F->V)) return 1;
  const double divU = C->calculate_divU(*F);
  nu = 1.0 + 0.5 * DT * divU;
  C->fill_all_blob_pos_at_midstep();
  F->set_up_gaussians(C->all_blob_pos);
  F->calculate_random_blob_velocities();
#endif
  C->calculate_forces(t);
  G->assemble_RHS(*C, *F);
  arma::vec soln = G->invert_saddle_point_system(*C, *F, 0, t);
  if (soln_out) copy_out(soln, soln_out);
  if (nu_out) *nu_out = nu;
  const bool overlap =
      C->end_of_step_update(soln.subvec(3 * C->total_num_blobs, 3 * C->total_num_blobs + 6 * NUM_BODIES - 1), nu);
  if (overlap) {
    C->reset_to_start_of_step();
    return 2;
  }
  C->accept_configuration_from_master_process(0);
  return 0;
}

}  // extern "C"
