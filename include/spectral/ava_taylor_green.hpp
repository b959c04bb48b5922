// TaylorGreenSolver / run_taylor_green over the B200 backend: the reference's benchmarked
// AVA solver interface (src/ava_taylor_green.hpp:8-55 of ovankerm/Spectral_solver) with
// the same records, constructor, methods, run options, CSV columns and stdout lines.
// RunConfig gains optional fields for the seeded perturbation, the final-field dump, the
// storage precision and the viscous treatment; their defaults reproduce the reference's run
// (the reference picks its precision at build time: SPECTRAL_PRECISION, CMakeLists.txt:19-28).
#pragma once

#include <cstdint>
#include <memory>
#include <string>

struct sns_handle;

namespace spectral::ava_solver {

struct Diagnostics {
  double t = 0.0;
  double kinetic_energy = 0.0;
  double dissipation = 0.0;
  double enstrophy = 0.0;
  double max_spectral_divergence = 0.0;
  double max_velocity = 0.0;
  double dt = 0.0;
  double cfl = 0.0;
  double main_dt = 0.0;
  double main_cfl = 0.0;
};

struct RunConfig {
  int n = 64;
  int steps = 80;
  int max_steps = 10000000;
  int output_every = 1;
  int print_every = 10;
  double dt = 0.0025;
  double cfl = 0.4;
  double t_end = 0.2;
  double output_dt = 0.1;
  double reynolds = 1600.0;
  bool adaptive_cfl = false;
  std::string output_dir = "output_ava";
  // additions: seeded k^(-5/3) perturbation and the final velocity dump
  std::uint64_t seed = 0;
  double pert_amp = 0.0;
  int pert_kmax = 0;
  bool dump_final = false;
  int precision = 0;     // 0: FP64 plain form (the drop-in), 1: FP32 precision form
  int viscous_mode = 0;  // 0: explicit viscous term (the reference), 1: integrating factor
  // checkpoint / resume: every checkpoint_every steps (0: never) the spectral state is
  // written to <output_dir>/checkpoint.bin; a run with restart = <path> continues from it
  // (same grid, same CSV columns; rows are appended from the checkpoint's time on)
  int checkpoint_every = 0;
  std::string restart;
};

class TaylorGreenSolver {
 public:
  struct Impl;

  TaylorGreenSolver(int n, double reynolds);
  TaylorGreenSolver(int n, double reynolds, std::uint64_t seed, double pert_amp, int pert_kmax, int precision = 0,
                    int viscous_mode = 0);
  ~TaylorGreenSolver();

  TaylorGreenSolver(const TaylorGreenSolver&) = delete;
  TaylorGreenSolver& operator=(const TaylorGreenSolver&) = delete;

  void step_rk3(double dt);
  Diagnostics diagnostics(double t);
  double max_velocity();
  void print_profile(int rank, double init_time, double run_time) const;
  // Final physical velocity written as a raw file (header: magic, n, then 3 x n^3 doubles).
  void dump_velocity(const std::string& path);
  // Exact checkpoint of the spectral state: header "SNSCKPT1", int64 n, int64 precision,
  // double t, int64 step, then u, v, w as n*n*(n/2+1) complex doubles (modes mx in
  // [0, n/2], x fastest).  load_checkpoint restores the state and returns t and step.
  void save_checkpoint(const std::string& path, double t, long long step);
  void load_checkpoint(const std::string& path, double* t, long long* step);
  sns_handle* handle() const;

 private:
  std::unique_ptr<Impl> impl_;
};

void run_taylor_green(const RunConfig& config);

}  // namespace spectral::ava_solver
