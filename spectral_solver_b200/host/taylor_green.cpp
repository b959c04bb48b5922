// TaylorGreenSolver / run_taylor_green over libsns_b200.so
// (the reference's src/ava_taylor_green.hpp:36-55 and ava_taylor_green_impl.hpp:1289-1410).
#include "spectral/ava_taylor_green.hpp"

#include "sns_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

namespace spectral::ava_solver {

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

double wall() {
  using C = std::chrono::steady_clock;
  static const auto t0 = C::now();
  return std::chrono::duration<double>(C::now() - t0).count();
}

}  // namespace

struct TaylorGreenSolver::Impl {
  sns_handle* h = nullptr;
  int n = 0;
  double step_time = 0.0, diagnostics_time = 0.0, max_velocity_time = 0.0;
  long long step_calls = 0, diagnostics_calls = 0, max_velocity_calls = 0;

  Impl(int n_in, double reynolds, std::uint64_t seed, double amp, int kmax, int precision, int viscous_mode)
      : n(n_in) {
    if (n <= 0) throw std::runtime_error("grid size must be positive");
    if (reynolds <= 0.0) throw std::runtime_error("Reynolds number must be positive");
    const int rc = sns_create(n, 1.0 / reynolds, precision, viscous_mode, seed, amp, kmax, &h);
    if (rc != SNS_OK) throw std::runtime_error(std::string("TaylorGreenSolver: ") + sns_last_error(nullptr));
  }
  ~Impl() {
    if (h) sns_destroy(h);
  }
  void check(int rc, const char* what) const {
    if (rc != SNS_OK) throw std::runtime_error(std::string(what) + ": " + sns_last_error(h));
  }
};

TaylorGreenSolver::TaylorGreenSolver(int n, double reynolds)
    : impl_(std::make_unique<Impl>(n, reynolds, 0, 0.0, 0, SNS_PRECISION_FP64, SNS_VISCOUS_EXPLICIT)) {}

TaylorGreenSolver::TaylorGreenSolver(int n, double reynolds, std::uint64_t seed, double pert_amp, int pert_kmax,
                                     int precision, int viscous_mode)
    : impl_(std::make_unique<Impl>(n, reynolds, seed, pert_amp, pert_kmax, precision, viscous_mode)) {}

TaylorGreenSolver::~TaylorGreenSolver() = default;

sns_handle* TaylorGreenSolver::handle() const { return impl_->h; }

void TaylorGreenSolver::step_rk3(double dt) {
  const double t0 = wall();
  impl_->check(sns_step(impl_->h, dt, 1), "TaylorGreenSolver::step_rk3");
  impl_->step_time += wall() - t0;
  ++impl_->step_calls;
}

Diagnostics TaylorGreenSolver::diagnostics(double t) {
  const double t0 = wall();
  sns_diag d{};
  impl_->check(sns_diagnostics(impl_->h, t, &d), "TaylorGreenSolver::diagnostics");
  impl_->diagnostics_time += wall() - t0;
  ++impl_->diagnostics_calls;
  Diagnostics row;
  row.t = t;
  row.kinetic_energy = d.kinetic_energy;
  row.dissipation = d.dissipation;
  row.enstrophy = d.enstrophy;
  row.max_spectral_divergence = d.max_spectral_divergence;
  row.max_velocity = d.max_velocity;
  return row;
}

double TaylorGreenSolver::max_velocity() {
  const double t0 = wall();
  double v = 0.0;
  impl_->check(sns_max_velocity(impl_->h, &v), "TaylorGreenSolver::max_velocity");
  impl_->max_velocity_time += wall() - t0;
  ++impl_->max_velocity_calls;
  return v;
}

void TaylorGreenSolver::print_profile(int rank, double init_time, double run_time) const {
  if (rank != 0) return;
  const auto& i = *impl_;
  std::cout << std::setprecision(6) << "profile_solver seconds"
            << " init=" << init_time << " run=" << run_time << " step=" << i.step_time
            << " diagnostics=" << i.diagnostics_time << " max_velocity=" << i.max_velocity_time
            << " step_calls=" << i.step_calls << " rhs_calls=" << 3 * i.step_calls
            << " diagnostics_calls=" << i.diagnostics_calls << " max_velocity_calls=" << i.max_velocity_calls << "\n";
}

void TaylorGreenSolver::dump_velocity(const std::string& path) {
  const int n = impl_->n;
  const std::size_t np = static_cast<std::size_t>(n) * n * n;
  std::vector<double> buf(3 * np);
  double* phys[3] = {buf.data(), buf.data() + np, buf.data() + 2 * np};
  impl_->check(sns_dump_velocity(impl_->h, phys), "TaylorGreenSolver::dump_velocity");
  std::ofstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot write " + path);
  // header: 8-byte magic "SNSVEL01", int64 n, then u, v, w as n^3 doubles each (x fastest)
  const char magic[8] = {'S', 'N', 'S', 'V', 'E', 'L', '0', '1'};
  const std::int64_t n64 = n;
  f.write(magic, 8);
  f.write(reinterpret_cast<const char*>(&n64), sizeof(n64));
  f.write(reinterpret_cast<const char*>(buf.data()), static_cast<std::streamsize>(buf.size() * sizeof(double)));
}

void run_taylor_green(const RunConfig& config) {
  if (config.dt <= 0.0 || config.cfl <= 0.0 || config.output_dt <= 0.0)
    throw std::runtime_error("--dt, --cfl, and --output-dt must be positive");
  std::filesystem::create_directories(config.output_dir);
  const std::string csv_path = config.output_dir + "/taylor_green_diagnostics.csv";
  std::ofstream csv(csv_path);
  csv << std::setprecision(17);
  csv << "t,kinetic_energy,dissipation,enstrophy,max_spectral_divergence,max_velocity,dt,cfl,main_dt,main_cfl\n";

  const double init_t0 = wall();
  TaylorGreenSolver solver(config.n, config.reynolds, config.seed, config.pert_amp, config.pert_kmax, config.precision,
                           config.viscous_mode);
  const double init_time = wall() - init_t0;
  const double run_t0 = wall();
  const double dx = 2.0 * kPi / static_cast<double>(config.n);
  double t = 0.0;
  int step = 0;
  int output_count = 0;
  auto write_row = [&](double time, bool force_print, double last_dt, double last_cfl, double main_dt,
                       double main_cfl) {
    const auto row = solver.diagnostics(time);
    csv << row.t << ',' << row.kinetic_energy << ',' << row.dissipation << ',' << row.enstrophy << ','
        << row.max_spectral_divergence << ',' << row.max_velocity << ',' << last_dt << ',' << last_cfl << ','
        << main_dt << ',' << main_cfl << '\n';
    csv.flush();
    if (force_print || output_count % config.print_every == 0) {
      std::cout << std::setprecision(10) << "step " << step << " t=" << row.t << " E=" << row.kinetic_energy
                << " eps=" << row.dissipation << " max_u=" << row.max_velocity << " dt=" << last_dt
                << " cfl=" << last_cfl << " main_dt=" << main_dt << " main_cfl=" << main_cfl << "\n";
    }
    ++output_count;
  };

  if (config.adaptive_cfl) {
    double next_output = 0.0;
    write_row(t, true, 0.0, 0.0, 0.0, 0.0);
    next_output += config.output_dt;
    while (t < config.t_end - 1.0e-14) {
      if (step >= config.max_steps)
        throw std::runtime_error("adaptive CFL run exceeded --max-steps before reaching --t-end");
      const double vmax = solver.max_velocity();
      double main_dt = config.dt;
      if (vmax > 1.0e-14) main_dt = std::min(main_dt, config.cfl * dx / vmax);
      const double main_cfl = vmax * main_dt / dx;
      double dt_step = std::min(main_dt, config.t_end - t);
      if (next_output <= config.t_end + 1.0e-14) dt_step = std::min(dt_step, next_output - t);
      if (dt_step <= 1.0e-14) {
        next_output += config.output_dt;
        continue;
      }
      const double actual_cfl = vmax * dt_step / dx;
      solver.step_rk3(dt_step);
      t += dt_step;
      ++step;
      if (t >= next_output - 1.0e-12 || t >= config.t_end - 1.0e-12) {
        write_row(t, t >= config.t_end - 1.0e-12, dt_step, actual_cfl, main_dt, main_cfl);
        while (next_output <= t + 1.0e-12) next_output += config.output_dt;
      }
    }
  } else {
    for (step = 0; step <= config.steps; ++step) {
      if (step % config.output_every == 0 || step == config.steps) {
        const bool first = step == 0;
        const double fixed_cfl = solver.max_velocity() * config.dt / dx;
        write_row(t, step == config.steps, first ? 0.0 : config.dt, first ? 0.0 : fixed_cfl,
                  first ? 0.0 : config.dt, first ? 0.0 : fixed_cfl);
      }
      if (step != config.steps) {
        solver.step_rk3(config.dt);
        t += config.dt;
      }
    }
  }
  const double run_time = wall() - run_t0;
  solver.print_profile(0, init_time, run_time);
  if (config.dump_final) {
    const std::string path = config.output_dir + "/velocity_final.bin";
    solver.dump_velocity(path);
    std::cout << "saved final velocity: " << path << "\n";
  }
  std::cout << "saved diagnostics: " << csv_path << "\n";
}

}  // namespace spectral::ava_solver
