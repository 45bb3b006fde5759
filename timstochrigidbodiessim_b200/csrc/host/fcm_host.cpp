// fcm_host.cpp -- reference-named C++ classes over the C-ABI (see fcm_host.hpp).
#include "fcm_host.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iomanip>

namespace fcm_host {

// ------------------------------------------------------------------ fft_solver
fft_solver::~fft_solver() {
  if (f_) fcm_fft_destroy(f_);
}

void fft_solver::initialise(int nx, int ny, int nz) {
  check(fcm_fft_create(nx, ny, nz, &f_), "fft_solver::initialise");
  int64_t tot = 0;
  check(fcm_fft_local_sizes(f_, &local_nx, &local_x_start, &local_ny_after_transpose,
                            &local_y_start_after_transpose, &tot, &pad),
        "fft_solver::initialise");
  total_local_size = tot;
}

void fft_solver::transform(double* in) { check(fcm_fft_transform(f_, in), "fft_solver::transform"); }
void fft_solver::inverse_transform(double* in) {
  check(fcm_fft_inverse_transform(f_, in), "fft_solver::inverse_transform");
}

// ------------------------------------------------------------------ collection
collection_of_rigid_bodies::~collection_of_rigid_bodies() {
  if (ctx_) fcm_destroy(ctx_);
}

void collection_of_rigid_bodies::initialise(const fcm_params& p, const std::vector<double>& ref) {
  params = p;
  blobs_per_body = p.blobs_per_body;
  total_num_blobs = p.num_bodies * p.blobs_per_body;
  if ((int)ref.size() != 3 * blobs_per_body) throw std::invalid_argument("blob_ref_pos size");
  blob_ref_pos = mat(3, blobs_per_body);
  for (int m = 0; m < blobs_per_body; ++m)
    for (int d = 0; d < 3; ++d) blob_ref_pos(d, m) = ref[3 * m + d];
  check(fcm_create(&p, ref.data(), &ctx_), "collection_of_rigid_bodies::initialise");
  all_blob_pos = mat(total_num_blobs, 3);
  blob_forces = vec(3 * total_num_blobs);
  bodies.assign(p.num_bodies, particle());
  midstep_bodies = bodies;
}

void collection_of_rigid_bodies::set_bodies(const std::vector<particle>& b) {
  const int M = params.num_bodies;
  std::vector<double> x(3 * M), q(4 * M);
  for (int n = 0; n < M; ++n) {
    for (int d = 0; d < 3; ++d) x[3 * n + d] = b[n].x[d];
    q[4 * n] = b[n].q.scalar_part;
    for (int d = 0; d < 3; ++d) q[4 * n + 1 + d] = b[n].q.vector_part[d];
  }
  check(fcm_set_bodies(ctx_, x.data(), q.data()), "set_bodies");
  bodies = b;
  midstep_bodies = b;
}

void collection_of_rigid_bodies::set_external_forces(const vec& fe) {
  check(fcm_set_external_forces(ctx_, fe.memptr()), "set_external_forces");
}

void collection_of_rigid_bodies::pull_bodies() {
  const int M = params.num_bodies;
  std::vector<double> x(3 * M), q(4 * M), xm(3 * M), qm(4 * M);
  check(fcm_get_bodies(ctx_, x.data(), q.data()), "get_bodies");
  check(fcm_get_midstep_bodies(ctx_, xm.data(), qm.data()), "get_midstep_bodies");
  for (int n = 0; n < M; ++n) {
    for (int d = 0; d < 3; ++d) {
      bodies[n].x[d] = x[3 * n + d];
      midstep_bodies[n].x[d] = xm[3 * n + d];
    }
    bodies[n].q = quaternion(q[4 * n], q[4 * n + 1], q[4 * n + 2], q[4 * n + 3]);
    midstep_bodies[n].q = quaternion(qm[4 * n], qm[4 * n + 1], qm[4 * n + 2], qm[4 * n + 3]);
  }
}

void collection_of_rigid_bodies::pull_blob_pos() {
  std::vector<double> Y(3 * (size_t)total_num_blobs);
  check(fcm_get_all_blob_pos(ctx_, Y.data()), "get_all_blob_pos");
  for (int i = 0; i < total_num_blobs; ++i)
    for (int d = 0; d < 3; ++d) all_blob_pos(i, d) = Y[3 * i + d];
}

static std::vector<double> rows_of(const mat& Y) {
  std::vector<double> out(3 * Y.n_rows);
  for (size_t i = 0; i < Y.n_rows; ++i)
    for (int d = 0; d < 3; ++d) out[3 * i + d] = Y(i, d);
  return out;
}

void collection_of_rigid_bodies::fill_all_blob_pos() {
  check(fcm_fill_all_blob_pos(ctx_, 0), "fill_all_blob_pos");
  pull_blob_pos();
}

void collection_of_rigid_bodies::fill_all_blob_pos_at_midstep() {
  check(fcm_fill_all_blob_pos(ctx_, 1), "fill_all_blob_pos_at_midstep");
  pull_blob_pos();
}

bool collection_of_rigid_bodies::advance_to_midstep(const vec& V) {
  int32_t ov = 0;
  check(fcm_advance_to_midstep(ctx_, V.memptr(), &ov), "advance_to_midstep");
  pull_bodies();
  pull_blob_pos();
  return ov != 0;
}

void collection_of_rigid_bodies::calculate_forces(double) {
  check(fcm_calculate_forces(ctx_), "calculate_forces");
  check(fcm_get_blob_forces(ctx_, blob_forces.memptr()), "calculate_forces");
  pull_bodies();
}

vec collection_of_rigid_bodies::multiply_by_K_at_midstep(const vec& in) const {
  vec out(3 * (size_t)total_num_blobs);
  check(fcm_multiply_by_K_at_midstep(ctx_, in.memptr(), out.memptr()), "multiply_by_K_at_midstep");
  return out;
}

vec collection_of_rigid_bodies::multiply_by_KT_at_midstep(const vec& in) const {
  vec out(6 * (size_t)params.num_bodies);
  check(fcm_multiply_by_KT_at_midstep(ctx_, in.memptr(), out.memptr()), "multiply_by_KT_at_midstep");
  return out;
}

bool collection_of_rigid_bodies::end_of_step_update(const vec& V, double nu) {
  int32_t ov = 0;
  check(fcm_end_of_step_update(ctx_, V.memptr(), nu, &ov), "end_of_step_update");
  pull_bodies();
  pull_blob_pos();
  return ov != 0;
}

void collection_of_rigid_bodies::reset_to_start_of_step() {
  check(fcm_reset_to_start_of_step(ctx_), "reset_to_start_of_step");
  pull_bodies();
}

double collection_of_rigid_bodies::calculate_divU(fcm_fluid_solver& fcm) {
  double d = 0.0;
  check(fcm_calculate_divU(ctx_, &d), "calculate_divU");
  check(fcm_get_V(ctx_, fcm.V.memptr()), "calculate_divU");
  pull_blob_pos();
  return d;
}

bool collection_of_rigid_bodies::check_for_overlap() {
  int32_t ov = 0;
  check(fcm_check_for_overlap(ctx_, &ov), "check_for_overlap");
  return ov != 0;
}

bool collection_of_rigid_bodies::check_for_channel_wall_overlap() {
  int32_t ov = 0;
  check(fcm_check_for_channel_wall_overlap(ctx_, &ov), "check_for_channel_wall_overlap");
  return ov != 0;
}

// collection_of_rigid_bodies.cpp:798-814: "t x y z q0 q1 q2 q3 ..." per line.
void collection_of_rigid_bodies::write_data_to_file(double t, const std::string& name, int digits) const {
  std::ofstream f(name, std::ios::app);
  f << std::scientific << std::setprecision(digits) << t << " ";
  for (const particle& b : bodies) {
    f << b.x[0] << " " << b.x[1] << " " << b.x[2] << " ";
    f << b.q.scalar_part << " " << b.q.vector_part[0] << " " << b.q.vector_part[1] << " " << b.q.vector_part[2]
      << " ";
  }
  f << std::endl;
}

void collection_of_rigid_bodies::write_blob_forces_to_file(double t, const std::string& name, int digits) const {
  std::ofstream f(name, std::ios::app);
  f << std::scientific << std::setprecision(digits) << t << " ";
  for (size_t i = 0; i < blob_forces.n_elem(); ++i) f << blob_forces(i) << " ";
  f << std::endl;
}

double collection_of_rigid_bodies::calculate_potential() {
  double U = 0.0;
  check(fcm_calculate_potential(ctx_, &U), "calculate_potential");
  pull_blob_pos();
  return U;
}

// ------------------------------------------------------------------ linked_list
void linked_list::initialise(int, int, int) {}  // the cell map is built with the context

void linked_list::populate(const mat& Y) {
  const std::vector<double> y = rows_of(Y);
  check(fcm_set_all_blob_pos(owner_->ctx(), y.data()), "linked_list::populate");
  check(fcm_list_populate(owner_->ctx()), "linked_list::populate");
}

bool linked_list::check_for_overlap(const mat& Y) const {
  const std::vector<double> y = rows_of(Y);
  check(fcm_set_all_blob_pos(owner_->ctx(), y.data()), "linked_list::check_for_overlap");
  int32_t ov = 0;
  check(fcm_check_for_overlap(owner_->ctx(), &ov), "linked_list::check_for_overlap");
  return ov != 0;
}

void linked_list::apply_barrier_forces(vec& F, const mat& Y) const {
  const std::vector<double> y = rows_of(Y);
  check(fcm_set_all_blob_pos(owner_->ctx(), y.data()), "linked_list::apply_barrier_forces");
  check(fcm_list_populate(owner_->ctx()), "linked_list::apply_barrier_forces");
  check(fcm_apply_barrier_forces(owner_->ctx(), F.memptr()), "linked_list::apply_barrier_forces");
}

std::vector<int> linked_list::cells() const {
  std::vector<int> c(owner_->total_num_blobs);
  check(fcm_list_get_cells(owner_->ctx(), c.data()), "linked_list::cells");
  return c;
}

// ------------------------------------------------------------------ fcm_fluid_solver
fcm_ctx* fcm_fluid_solver::ctx() const { return bodies_->ctx(); }

void fcm_fluid_solver::initialise(collection_of_rigid_bodies& c) {
  bodies_ = &c;
  V = vec(3 * (size_t)c.total_num_blobs);
  ref_Minv = mat(3 * c.blobs_per_body, 3 * c.blobs_per_body);
  ref_N = mat(6, 6);
}

void fcm_fluid_solver::set_up_gaussians(const mat& Y) {
  const std::vector<double> y = rows_of(Y);
  check(fcm_set_up_gaussians(ctx(), y.data()), "set_up_gaussians");
}

void fcm_fluid_solver::produce_random_velocity_field(unsigned long long seed, unsigned long long counter) {
  check(fcm_produce_random_velocity_field(ctx(), seed, counter), "produce_random_velocity_field");
}

void fcm_fluid_solver::inject_random_stress(const std::vector<const double*>& s) {
  if (s.size() != 6) throw std::invalid_argument("six stress arrays expected");
  check(fcm_inject_random_stress(ctx(), s[0], s[1], s[2], s[3], s[4], s[5]), "inject_random_stress");
}

void fcm_fluid_solver::calculate_random_blob_velocities() {
  check(fcm_calculate_random_blob_velocities(ctx(), V.memptr()), "calculate_random_blob_velocities");
}

void fcm_fluid_solver::set_up_force_distribution(const vec& F) {
  check(fcm_set_up_force_distribution(ctx(), F.memptr()), "set_up_force_distribution");
}

void fcm_fluid_solver::produce_deterministic_velocity_field() {
  check(fcm_produce_deterministic_velocity_field(ctx()), "produce_deterministic_velocity_field");
}

void fcm_fluid_solver::calculate_deterministic_blob_velocities() {
  check(fcm_calculate_deterministic_blob_velocities(ctx(), V.memptr()), "calculate_deterministic_blob_velocities");
}

void fcm_fluid_solver::produce_shear_velocity_field(double scale, double wavenumber) {
  check(fcm_produce_shear_velocity_field(ctx(), scale, wavenumber), "produce_shear_velocity_field");
  Vshear = vec(3 * (size_t)bodies_->total_num_blobs);
}

void fcm_fluid_solver::calculate_shear_blob_velocities() {
  Vshear = vec(3 * (size_t)bodies_->total_num_blobs);
  check(fcm_calculate_shear_blob_velocities(ctx(), Vshear.memptr()), "calculate_shear_blob_velocities");
}

std::vector<double> fcm_fluid_solver::fluid_x_velocity_in_y(const vec& F) {
  std::vector<double> prof((size_t)bodies_->params.ny, 0.0);
  check(fcm_fluid_x_velocity_in_y(ctx(), F.memptr(), prof.data()), "fluid_x_velocity_in_y");
  return prof;
}

void fcm_fluid_solver::produce_reference_matrices(collection_of_rigid_bodies& c) {
  bodies_ = &c;
  check(fcm_produce_reference_matrices(ctx()), "produce_reference_matrices");
  check(fcm_get_reference_matrices(ctx(), ref_Minv.memptr(), ref_N.memptr(), nullptr), "produce_reference_matrices");
}

void fcm_fluid_solver::fetch_velocity_field(int which) {
  const fcm_params& p = bodies_->params;
  const size_t P = (size_t)p.nx * p.ny * 2 * (p.nz / 2 + 1);
  ux.assign(P, 0.0);
  uy.assign(P, 0.0);
  uz.assign(P, 0.0);
  check(fcm_get_velocity_field(ctx(), which, ux.data(), uy.data(), uz.data()), "fetch_velocity_field");
}

// ------------------------------------------------------------------ gmres_solver
void gmres_solver::initialise(const collection_of_rigid_bodies& c) {
  num_blobs = c.total_num_blobs;
  system_size = 3 * num_blobs + 6 * c.params.num_bodies;
  RHS = vec(system_size);
}

void gmres_solver::assemble_RHS(const collection_of_rigid_bodies& c, const fcm_fluid_solver& fcm) {
  check(fcm_set_blob_forces(c.ctx(), c.blob_forces.memptr()), "assemble_RHS");
  check(fcm_assemble_RHS(c.ctx()), "assemble_RHS");
  check(fcm_get_RHS(c.ctx(), RHS.memptr()), "assemble_RHS");
  (void)fcm;
}

vec gmres_solver::multiply_by_Pinv(const vec& in, const collection_of_rigid_bodies& c, const fcm_fluid_solver&) {
  vec out(system_size);
  check(fcm_multiply_by_Pinv(c.ctx(), in.memptr(), out.memptr()), "multiply_by_Pinv");
  return out;
}

vec gmres_solver::multiply_by_saddle_point_matrix(const vec& in, const collection_of_rigid_bodies& c,
                                                  fcm_fluid_solver&) {
  vec out(system_size);
  check(fcm_multiply_by_saddle_point_matrix(c.ctx(), in.memptr(), out.memptr()), "multiply_by_saddle_point_matrix");
  return out;
}

vec gmres_solver::invert_saddle_point_system(const collection_of_rigid_bodies& c, fcm_fluid_solver&, int myrank,
                                             double t) {
  vec soln(system_size);
  check(fcm_set_RHS(c.ctx(), RHS.memptr()), "invert_saddle_point_system");
  int32_t it = 0;
  double rel = 0.0;
  const int st = fcm_invert_saddle_point_system(c.ctx(), soln.memptr(), &it, &rel);
  if (st != FCM_OK && st != FCM_ERR_NOT_CONVERGED) throw error(st, "invert_saddle_point_system");
  last_iterations = it;
  last_relative_error = rel;
  last_status = st;
  // gmres_solver.cpp:328-340: progress message on rank 0
  if (myrank == 0 && std::getenv("FCM_VERBOSE")) {
    if (st == FCM_OK)
      std::printf("[t = %g] GMRES converged to a relative error of %g in %d iterations...\n", t, rel, it);
    else
      std::printf("[t = %g] GMRES failed to converge in %d iterations. The relative error is %g\n", t, it, rel);
  }
  return soln;
}

}  // namespace fcm_host
