// rigid_bodies_main.cpp -- the reference's time-stepping driver (main.cpp:73-109,
// :212-451) on the reference-named classes of fcm_host.hpp.
//
//   rigid_bodies_sim key=value ...
//
// keys: the fcm_params fields (nx ny nz ngauss dx blob_radius viscosity kT dt
// num_bodies blobs_per_body ncells potential steric_fs steric_rc gmres_max_iter
// gmres_tol fd_delta algorithm noise skip_on_overlap slip_channel precision), plus
//   shape=<file>     blob reference positions, one "x y z" line per blob
//   ic=<file>        initial state in the reference's .dat format
//                    ("t x y z q0 q1 q2 q3 ..." per line; the last line is used,
//                    as INITIAL_CONDITIONS_TYPE 0, collection_of_rigid_bodies.cpp:265-339)
//   steps=<n>        accepted steps to run
//   seed=<n>         Philox seed of the fluctuations
//   body_force_z=<f> constant z force on every body (default 0)
//   name=<prefix>    output prefix: <prefix>.dat (states, collection_of_rigid_bodies.cpp:798-814)
//                    and <prefix>_velocities.dat (body velocities, main.cpp:343-367)
//   save_every=<n>   steps between saves (default 1)
//   digits=<n>       significant digits of the saved states (default 6, the reference's)
//   ic_pick=last|random  which state of the ic file to start from (IC_READ_IN_LAST /
//                    IC_READ_IN_RANDOM, collection_of_rigid_bodies.cpp:265-339)
//   mcmc=<n>         Metropolis sampling instead of time stepping (MARKOV_CHAIN_MONTE_CARLO,
//                    main.cpp:113-210): n steps, reported every 200 and saved to
//                    <prefix>.dat every 200 once past mcmc_save_after (default 100000)
//   shear=1          sinusoidal shear forcing (SHEARING_FORCES, main.cpp:98-100, :270-272,
//                    :371-433) with shear_scale=<S> and shear_wavenumber=<w> (default 1 and 1,
//                    config.hpp:54-55); saves add <prefix>_fluid_x_velocity_in_y.dat
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <map>
#include <random>
#include <stdexcept>
#include <algorithm>
#include <sstream>
#include <string>
#include <vector>

#include "fcm_host.hpp"

using namespace fcm_host;

static bool set_param(fcm_params& p, const std::string& k, const std::string& v) {
#define I(name)                        \
  if (k == #name) {                    \
    p.name = (int32_t)std::stol(v);    \
    return true;                       \
  }
#define F(name)                        \
  if (k == #name) {                    \
    p.name = std::stod(v);             \
    return true;                       \
  }
  I(nx) I(ny) I(nz) I(ngauss) F(dx) F(blob_radius) F(viscosity) F(kT) F(dt) I(num_bodies) I(blobs_per_body)
  I(ncells) I(potential) F(steric_fs) F(steric_rc) I(gmres_max_iter) F(gmres_tol) F(fd_delta) I(algorithm)
  I(precision) I(noise) I(skip_on_overlap) I(slip_channel)
#undef I
#undef F
  return false;
}

// The non-empty lines of a state file, each as its numbers.
static std::vector<std::vector<double>> read_states(const std::string& path) {
  std::ifstream f(path);
  std::string line;
  std::vector<std::vector<double>> out;
  while (std::getline(f, line)) {
    if (line.find_first_not_of(" \t\r") == std::string::npos) continue;
    std::istringstream is(line);
    std::vector<double> v;
    double x;
    while (is >> x) v.push_back(x);
    out.push_back(v);
  }
  return out;
}

static std::vector<double> read_numbers_last_line(const std::string& path) {
  std::ifstream f(path);
  std::string line, last;
  while (std::getline(f, line))
    if (line.find_first_not_of(" \t\r") != std::string::npos) last = line;
  std::vector<double> out;
  std::istringstream is(last);
  double v;
  while (is >> v) out.push_back(v);
  return out;
}

int main(int argc, char** argv) {
  fcm_params p;
  fcm_default_params(&p);
  p.algorithm = 2;
  std::map<std::string, std::string> opt;
  for (int i = 1; i < argc; ++i) {
    std::string a(argv[i]);
    const size_t e = a.find('=');
    if (e == std::string::npos) {
      std::fprintf(stderr, "bad argument %s (expected key=value)\n", argv[i]);
      return 2;
    }
    const std::string k = a.substr(0, e), v = a.substr(e + 1);
    if (!set_param(p, k, v)) opt[k] = v;
  }
  const int steps = opt.count("steps") ? std::atoi(opt["steps"].c_str()) : 1;
  const unsigned long long seed = opt.count("seed") ? std::strtoull(opt["seed"].c_str(), nullptr, 10) : 1234ull;
  const double fz = opt.count("body_force_z") ? std::atof(opt["body_force_z"].c_str()) : 0.0;
  const std::string name = opt.count("name") ? opt["name"] : "example";
  const int save_every = opt.count("save_every") ? std::atoi(opt["save_every"].c_str()) : 1;
  const int digits = opt.count("digits") ? std::atoi(opt["digits"].c_str()) : 6;
  if (!opt.count("shape") || !opt.count("ic")) {
    std::fprintf(stderr, "shape=<file> and ic=<file> are required\n");
    return 2;
  }
  std::vector<double> ref;
  {
    std::ifstream f(opt["shape"]);
    double v;
    while (f >> v) ref.push_back(v);
  }
  p.blobs_per_body = (int32_t)(ref.size() / 3);
  std::vector<double> ic = read_numbers_last_line(opt["ic"]);
  if (opt.count("ic_pick") && opt["ic_pick"] == "random") {  // IC_READ_IN_RANDOM
    const std::vector<std::vector<double>> states = read_states(opt["ic"]);
    if (!states.empty()) {
      std::mt19937_64 rng(seed);
      ic = states[std::uniform_int_distribution<size_t>(0, states.size() - 1)(rng)];
      std::printf("Input file contains %zu state(s); one was selected at random.\n", states.size());
    }
  }
  p.num_bodies = (int32_t)((ic.size() - 1) / 7);
  try {
    // main.cpp:73-109
    collection_of_rigid_bodies all_bodies;
    all_bodies.initialise(p, ref);
    std::vector<particle> b(p.num_bodies);
    for (int n = 0; n < p.num_bodies; ++n) {
      for (int d = 0; d < 3; ++d) b[n].x[d] = ic[1 + 7 * n + d];
      b[n].q = quaternion(ic[1 + 7 * n + 3], ic[1 + 7 * n + 4], ic[1 + 7 * n + 5], ic[1 + 7 * n + 6]);
    }
    all_bodies.set_bodies(b);
    vec fe(6 * (size_t)p.num_bodies);
    for (int n = 0; n < p.num_bodies; ++n) fe(6 * n + 2) = fz;
    all_bodies.set_external_forces(fe);
    fcm_fluid_solver fcm;
    fcm.initialise(all_bodies);
    fcm.produce_reference_matrices(all_bodies);
    gmres_solver gmres;
    gmres.initialise(all_bodies);
    const bool shear = opt.count("shear") && std::atoi(opt["shear"].c_str()) != 0;
    if (shear)  // main.cpp:98-100
      fcm.produce_shear_velocity_field(opt.count("shear_scale") ? std::atof(opt["shear_scale"].c_str()) : 1.0,
                                       opt.count("shear_wavenumber") ? std::atof(opt["shear_wavenumber"].c_str()) : 1.0);
    if (opt.count("mcmc")) {  // main.cpp:113-210
      const long long n_total = std::atoll(opt["mcmc"].c_str());
      const long long save_after = opt.count("mcmc_save_after") ? std::atoll(opt["mcmc_save_after"].c_str()) : 100000;
      fcm_mcmc_state st;
      if (fcm_mcmc_state_init(all_bodies.ctx(), &st) != 0) throw std::runtime_error(fcm_last_error());
      while (st.steps < n_total) {
        const long long chunk = std::min<long long>(200 - st.steps % 200, n_total - st.steps);
        const int rc = fcm_mcmc_run(all_bodies.ctx(), seed, chunk, &st);
        if (rc != 0) throw std::runtime_error(fcm_last_error());
        if (st.steps % 200 == 0) {
          all_bodies.pull_bodies();
          if (st.steps > save_after) {
            all_bodies.write_data_to_file((double)st.steps, name + ".dat", digits);
            std::printf("[scale/a = %g, U = %g] Saved sample %lld\n", st.scale / p.blob_radius, st.potential,
                        st.steps);
          } else {
            std::printf("[scale/a = %g, U = %g]\n", st.scale / p.blob_radius, st.potential);
          }
        }
      }
      return 0;
    }
    // main.cpp:212-451
    int skipped_steps = 0, accepted = 0, plotting_step = 0;
    unsigned long long counter = 0;
    double t = 0.0;
    while (accepted < steps) {
      all_bodies.fill_all_blob_pos();
      if (p.noise) fcm.produce_random_velocity_field(seed, counter++);
      fcm.set_up_gaussians(all_bodies.all_blob_pos);
      if (p.noise) fcm.calculate_random_blob_velocities();
      else fcm.V.zeros();
      double nu = 1.0;
      if (p.algorithm == 1) {
        if (all_bodies.advance_to_midstep(fcm.V)) {
          skipped_steps++;
          continue;
        }
        const double divU = p.noise ? all_bodies.calculate_divU(fcm) : 0.0;
        nu = 1.0 + 0.5 * p.dt * divU;
        all_bodies.fill_all_blob_pos_at_midstep();
        fcm.set_up_gaussians(all_bodies.all_blob_pos);
        if (p.noise) fcm.calculate_random_blob_velocities();
        if (shear) fcm.calculate_shear_blob_velocities();  // main.cpp:270-272
      }
      all_bodies.calculate_forces(t);
      gmres.assemble_RHS(all_bodies, fcm);
      const vec soln = gmres.invert_saddle_point_system(all_bodies, fcm, 0, t);
      const vec U = soln.subvec(3 * (size_t)all_bodies.total_num_blobs,
                                3 * (size_t)all_bodies.total_num_blobs + 6 * p.num_bodies - 1);
      if (all_bodies.end_of_step_update(U, nu)) {
        all_bodies.reset_to_start_of_step();
        skipped_steps++;
        continue;
      }
      t += p.dt;
      ++accepted;
      if (++plotting_step == save_every) {
        plotting_step = 0;
        all_bodies.write_data_to_file(t, name + ".dat", digits);
        all_bodies.write_blob_forces_to_file(t, name + "_blob_forces.dat", digits);
        std::ofstream vf(name + "_velocities.dat", std::ios::app);
        vf << std::scientific << std::setprecision(digits) << t << " ";
        for (size_t i = 0; i < U.n_elem(); ++i) vf << U(i) << " ";
        vf << std::endl;
        if (shear) {  // main.cpp:371-433: the flow of the constraint forces plus u_shear
          all_bodies.fill_all_blob_pos_at_midstep();
          fcm.set_up_gaussians(all_bodies.all_blob_pos);
          const std::vector<double> prof =
              fcm.fluid_x_velocity_in_y(soln.subvec(0, 3 * (size_t)all_bodies.total_num_blobs - 1));
          std::ofstream ff(name + "_fluid_x_velocity_in_y.dat", std::ios::app);
          ff << t << " ";
          for (double u : prof) ff << u << " ";
          ff << std::endl;
        }
      }
      std::printf("step %d gmres_iters %d rel %.3e status %d\n", accepted, gmres.last_iterations,
                  gmres.last_relative_error, gmres.last_status);
    }
    std::printf("skipped_steps %d\n", skipped_steps);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
  return 0;
}
