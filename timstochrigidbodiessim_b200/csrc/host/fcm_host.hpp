// fcm_host.hpp -- C++ classes with the names, methods and public members of the
// reference's fft_solver, fcm_fluid_solver, collection_of_rigid_bodies,
// linked_list, gmres_solver, particle and quaternion (their .hpp files), built on
// the C-ABI of include/fcm_b200.h.  All state lives in one device context owned
// by collection_of_rigid_bodies; the other classes reference it.  Public members
// that the reference reads directly (fcm.V, all_bodies.all_blob_pos, blob_forces,
// bodies, ref_Minv, ref_N) are host mirrors refreshed by the methods that produce
// them.  Errors throw fcm_host::error carrying the library status.
//
// Differences from the reference, which has compile-time configuration and
// Armadillo: parameters come from an fcm_params (config.hpp's macros), and
// vec/mat are the small column-major containers below.
#pragma once

#include <cmath>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../../include/fcm_b200.h"

namespace fcm_host {

struct error : std::runtime_error {
  int status;
  error(int s, const std::string& where) : std::runtime_error(where + ": " + fcm_last_error()), status(s) {}
};

inline void check(int s, const char* where) {
  if (s != FCM_OK) throw error(s, where);
}

// Column vector (Armadillo's vec subset).
struct vec {
  std::vector<double> d;
  vec() {}
  explicit vec(size_t n, double v = 0.0) : d(n, v) {}
  size_t n_elem() const { return d.size(); }
  double& operator()(size_t i) { return d[i]; }
  double operator()(size_t i) const { return d[i]; }
  double* memptr() { return d.data(); }
  const double* memptr() const { return d.data(); }
  void zeros() { std::fill(d.begin(), d.end(), 0.0); }
  vec subvec(size_t a, size_t b) const {
    vec o(b - a + 1);
    for (size_t i = a; i <= b; ++i) o.d[i - a] = d[i];
    return o;
  }
};

// Column-major matrix (Armadillo's mat subset).
struct mat {
  size_t n_rows = 0, n_cols = 0;
  std::vector<double> d;
  mat() {}
  mat(size_t r, size_t c) : n_rows(r), n_cols(c), d(r * c, 0.0) {}
  double& operator()(size_t i, size_t j) { return d[j * n_rows + i]; }
  double operator()(size_t i, size_t j) const { return d[j * n_rows + i]; }
  double* memptr() { return d.data(); }
  const double* memptr() const { return d.data(); }
};

// quaternion.hpp:17-104 (the parts the driver uses).
struct quaternion {
  double scalar_part = 1.0;
  double vector_part[3] = {0.0, 0.0, 0.0};
  quaternion() {}
  quaternion(double q0, double q1, double q2, double q3) : scalar_part(q0) {
    vector_part[0] = q1;
    vector_part[1] = q2;
    vector_part[2] = q3;
  }
  double norm() const {
    return std::sqrt(scalar_part * scalar_part + vector_part[0] * vector_part[0] + vector_part[1] * vector_part[1] +
                     vector_part[2] * vector_part[2]);
  }
};

// particle.hpp:17-33 (position and orientation).
struct particle {
  double x[3] = {0.0, 0.0, 0.0};
  quaternion q;
};

class collection_of_rigid_bodies;
class fcm_fluid_solver;

// fft_solver.hpp:10-31 on the GPU.
class fft_solver {
 public:
  int local_nx = 0, local_x_start = 0, local_ny_after_transpose = 0, local_y_start_after_transpose = 0;
  long long total_local_size = 0;
  int pad = 0;
  ~fft_solver();
  fft_solver() {}
  void initialise(int nx, int ny, int nz);  // fft_solver.cpp:17-28 (sizes from NUM_FFT_GRID_POINTS_*)
  void transform(double* in);               // fft_solver.cpp:32-36
  void inverse_transform(double* in);       // fft_solver.cpp:38-42

 private:
  fcm_fft* f_ = nullptr;
};

// linked_list.hpp:15-37.
class linked_list {
 public:
  explicit linked_list(collection_of_rigid_bodies* owner = nullptr) : owner_(owner) {}
  void initialise(int total_num_blobs, int myrank, int totalnodes);  // linked_list.cpp:23-72
  void populate(const mat& Y);                                       // linked_list.cpp:80-102
  bool check_for_overlap(const mat& Y) const;                        // linked_list.cpp:104-190
  void apply_barrier_forces(vec& blob_forces, const mat& Y) const;   // linked_list.cpp:192-281
  std::vector<int> cells() const;                                    // cell of every blob
  collection_of_rigid_bodies* owner_;
};

// collection_of_rigid_bodies.hpp:21-59.
class collection_of_rigid_bodies {
 public:
  int blobs_per_body = 0;
  int total_num_blobs = 0;
  mat blob_ref_pos;                 // 3 x nb
  mat all_blob_pos;                 // Nb x 3 (host mirror)
  std::vector<particle> bodies, midstep_bodies;
  vec blob_forces;                  // host mirror
  linked_list list;
  fcm_params params;

  collection_of_rigid_bodies() : list(this) {}
  ~collection_of_rigid_bodies();
  collection_of_rigid_bodies(const collection_of_rigid_bodies&) = delete;
  collection_of_rigid_bodies& operator=(const collection_of_rigid_bodies&) = delete;

  // collection_of_rigid_bodies.cpp:15-153: geometry from `ref` (3*nb blob-major).
  void initialise(const fcm_params& p, const std::vector<double>& ref);
  void set_bodies(const std::vector<particle>& b);        // replaces seed_the_bodies / IC read-in
  void set_external_forces(const vec& fe);
  void fill_all_blob_pos();                              // :155-174
  void fill_all_blob_pos_at_midstep();                   // :176-193
  bool advance_to_midstep(const vec& V);                 // :566-621
  void calculate_forces(double t);                       // :623-664
  vec multiply_by_K_at_midstep(const vec& in) const;     // :707-731
  vec multiply_by_KT_at_midstep(const vec& in) const;    // :733-757
  bool end_of_step_update(const vec& V, double nu);      // :759-790
  void reset_to_start_of_step();                         // :792-796
  double calculate_divU(fcm_fluid_solver& fcm);          // :869-953
  bool check_for_overlap();                              // :195-205
  bool check_for_channel_wall_overlap();                 // :207-239
  double calculate_potential();                          // :666-705
  // :798-814 (state part); the reference writes 6 significant digits
  void write_data_to_file(double t, const std::string& name, int digits = 6) const;
  // :816-833, the blob forces of the last calculate_forces
  void write_blob_forces_to_file(double t, const std::string& name, int digits = 6) const;

  fcm_ctx* ctx() const { return ctx_; }
  void pull_bodies();
  void pull_blob_pos();

 private:
  fcm_ctx* ctx_ = nullptr;
};

// fcm_fluid_solver.hpp:18-76.
class fcm_fluid_solver {
 public:
  vec V;                 // last interpolated blob velocities (3 Nb)
  mat ref_Minv, ref_N;   // reference matrices (3nb)^2 and 6x6
  std::vector<double> ux, uy, uz;  // velocity grids in the padded layout (filled on request)

  explicit fcm_fluid_solver(collection_of_rigid_bodies* c = nullptr) : bodies_(c) {}
  void initialise(collection_of_rigid_bodies& c);             // :29-129
  void set_up_gaussians(const mat& Y);                        // :131-165
  void produce_random_velocity_field(unsigned long long seed, unsigned long long counter);  // :167-361
  void inject_random_stress(const std::vector<const double*>& s6);  // :167-361 with given stress
  void calculate_random_blob_velocities();                    // :426-487
  void set_up_force_distribution(const vec& F);               // :552-634
  void produce_deterministic_velocity_field();                // :636-701
  void calculate_deterministic_blob_velocities();             // :363-424
  void produce_reference_matrices(collection_of_rigid_bodies& c);  // :842-881
  void fetch_velocity_field(int which);                       // ux/uy/uz host mirrors (2 = u_shear)
  // SHEARING_FORCES (config.hpp:52-56 values as arguments)
  vec Vshear;                                                  // 3 Nb
  void produce_shear_velocity_field(double scale, double wavenumber);  // :703-842
  void calculate_shear_blob_velocities();                      // :489-550
  std::vector<double> fluid_x_velocity_in_y(const vec& F);     // main.cpp:371-433 (ny values)

 private:
  collection_of_rigid_bodies* bodies_;
  fcm_ctx* ctx() const;
};

// gmres_solver.hpp:18-40.
class gmres_solver {
 public:
  int num_blobs = 0;
  int system_size = 0;
  vec RHS;
  int last_iterations = 0;
  double last_relative_error = 0.0;
  int last_status = FCM_OK;

  void initialise(const collection_of_rigid_bodies& c);                                   // :14-34
  void assemble_RHS(const collection_of_rigid_bodies& c, const fcm_fluid_solver& fcm);   // :58-70
  vec multiply_by_Pinv(const vec& in, const collection_of_rigid_bodies& c, const fcm_fluid_solver& fcm);  // :85-146
  vec multiply_by_saddle_point_matrix(const vec& in, const collection_of_rigid_bodies& c, fcm_fluid_solver& fcm);  // :72-83
  vec invert_saddle_point_system(const collection_of_rigid_bodies& c, fcm_fluid_solver& fcm, int myrank, double t);  // :148-306
};

}  // namespace fcm_host
