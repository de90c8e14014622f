// pfem2_solver.hpp -- header-only C++ shim with the member functions of the
// reference's pfem2Solver (TurekBenchmarkCuda/pfem2particle.h:126-233,
// TurekBenchmark/pfem2particle.h:139-243), forwarding to the C ABI of
// pfem2.h. A case driver keeps its run() loop:
//
//   for (; time <= final_time; time += time_step, ++timestep_number) {
//     correct_particles_velocities();
//     move_particles();
//     distribute_particle_velocities_to_grid();
//     fem_step();                       // the case's assemble_system()
//     calculate_loads(3, &forces_csv);
//   }
//
// Differences from the reference class, by design: the mesh and the flow
// case are handed over as plain arrays (pfem2_mesh_view, pfem2_case) instead
// of deal.II objects; the nodal vectors live on the GPU and are read or
// written with get_field / set_field; errors throw pfem2b::Error carrying the
// pfem2_status instead of calling exit().
#pragma once

#include <cstdint>
#include <fstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "pfem2.h"

namespace pfem2b {

class Error : public std::runtime_error {
 public:
  Error(pfem2_status s, const std::string& what) : std::runtime_error(what), status(s) {}
  pfem2_status status;
};

inline void check(pfem2_status s) {
  if (s != PFEM2_OK) throw Error(s, std::string("pfem2: ") + pfem2_last_error());
}

class Solver {
 public:
  // pfem2Solver::pfem2Solver + build_grid + setup_system for one instance
  Solver(const pfem2_config& cfg, const pfem2_mesh_view& mesh, const pfem2_case& cs) : cs_(cs) {
    check(pfem2_create(&cfg, &ctx_));
    int32_t inst = 0;
    check(pfem2_add_instance(ctx_, &mesh, &cs, &inst));
    check(pfem2_setup(ctx_));
    n_vertices_ = mesh.n_vertices;
    time_step = cs.dt;
  }
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;
  ~Solver() { pfem2_destroy(ctx_); }

  // ---- the reference's public members
  void seed_particles(const std::vector<unsigned int>& quantities, uint64_t seed = 0, double jitter = 0.0) {
    if (quantities.size() < 2) return;  // as the reference: ignore a bad request
    uint32_t q[3] = {quantities[0], quantities[1], quantities.size() > 2 ? quantities[2] : 1u};
    check(pfem2_seed(ctx_, -1, q, seed, jitter));
  }
  void correct_particles_velocities() { check(pfem2_correct(ctx_)); }
  void move_particles() { check(pfem2_move(ctx_)); }
  void distribute_particle_velocities_to_grid() { check(pfem2_project(ctx_)); }
  void fem_step() { check(pfem2_fem_step(ctx_)); }
  // calculate_loads(patch_id, out): one CSV line "t,Cx,Cy,dP,Cx_nu,Cx_p,Cy_nu,Cy_p"
  // as TurekBenchmark/pfem2particle.cpp:963-967 writes it
  void calculate_loads(int patch_id, std::ofstream* out) {
    double c[5];
    check(pfem2_loads(ctx_, 0, patch_id, c));
    if (out)
      *out << time << "," << c[0] + c[1] << "," << c[2] + c[3] << "," << c[4] << "," << c[0] << "," << c[1] << ","
           << c[2] << "," << c[3] << std::endl;
  }
  // calculate_vorticity (cylinderDyM/pfem2particle.cpp:1000-1050), 2D: the
  // nodal vorticity, also kept in PFEM2_FIELD_VORTICITY
  std::vector<double> calculate_vorticity() {
    check(pfem2_calculate_vorticity(ctx_));
    return get_field(PFEM2_FIELD_VORTICITY);
  }
  // one run() iteration with fused kernels (and a CUDA graph)
  void step() {
    check(pfem2_step(ctx_));
    time += time_step;
    ++timestep_number;
  }

  // ---- the reference's public data, as device fields
  std::vector<double> get_field(pfem2_field f) const {
    std::vector<double> v((size_t)n_vertices_);
    check(pfem2_get_field(ctx_, 0, f, v.data()));
    return v;
  }
  void set_field(pfem2_field f, const std::vector<double>& v) { check(pfem2_set_field(ctx_, 0, f, v.data())); }
  int n_particles() const {
    int32_t n = 0;
    check(pfem2_particle_count(ctx_, 0, &n));
    return n;
  }
  pfem2_stats stats() const {
    pfem2_stats s;
    check(pfem2_get_stats(ctx_, &s));
    return s;
  }

  double time = 0.0, time_step = 0.0;
  int timestep_number = 1;

 private:
  pfem2_ctx* ctx_ = nullptr;
  pfem2_case cs_;
  int n_vertices_ = 0;
};

}  // namespace pfem2b
