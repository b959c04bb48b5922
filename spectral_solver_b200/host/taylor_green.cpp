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
  int precision = 0;
  double step_time = 0.0, diagnostics_time = 0.0, max_velocity_time = 0.0;
  long long step_calls = 0, diagnostics_calls = 0, max_velocity_calls = 0;

  Impl(int n_in, double reynolds, std::uint64_t seed, double amp, int kmax, int precision_in, int viscous_mode)
      : n(n_in), precision(precision_in) {
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

void TaylorGreenSolver::save_checkpoint(const std::string& path, double t, long long step) {
  const int n = impl_->n;
  const std::size_t full = static_cast<std::size_t>(n) * n * n;
  const std::size_t nh = static_cast<std::size_t>(n / 2 + 1);
  std::vector<double> buf(3 * 2 * full);
  double* st[3] = {buf.data(), buf.data() + 2 * full, buf.data() + 4 * full};
  impl_->check(sns_get_state(impl_->h, st), "TaylorGreenSolver::save_checkpoint");
  std::ofstream f(path + ".tmp", std::ios::binary);
  if (!f) throw std::runtime_error("cannot write " + path);
  const char magic[8] = {'S', 'N', 'S', 'C', 'K', 'P', 'T', '1'};
  const std::int64_t hdr[2] = {n, impl_->precision};
  const std::int64_t step64 = step;
  f.write(magic, 8);
  f.write(reinterpret_cast<const char*>(hdr), sizeof hdr);
  f.write(reinterpret_cast<const char*>(&t), sizeof t);
  f.write(reinterpret_cast<const char*>(&step64), sizeof step64);
  for (int c = 0; c < 3; ++c)
    for (std::size_t row = 0; row < static_cast<std::size_t>(n) * n; ++row)
      f.write(reinterpret_cast<const char*>(st[c] + 2 * row * n), static_cast<std::streamsize>(2 * nh * sizeof(double)));
  f.close();
  if (!f) throw std::runtime_error("write failed: " + path);
  std::filesystem::rename(path + ".tmp", path);  // a crash mid-write leaves the old checkpoint
}

void TaylorGreenSolver::load_checkpoint(const std::string& path, double* t, long long* step) {
  const int n = impl_->n;
  std::ifstream f(path, std::ios::binary);
  if (!f) throw std::runtime_error("cannot read " + path);
  char magic[8];
  std::int64_t hdr[2] = {0, 0}, step64 = 0;
  double t0 = 0.0;
  f.read(magic, 8);
  f.read(reinterpret_cast<char*>(hdr), sizeof hdr);
  f.read(reinterpret_cast<char*>(&t0), sizeof t0);
  f.read(reinterpret_cast<char*>(&step64), sizeof step64);
  if (!f || std::string(magic, 8) != "SNSCKPT1") throw std::runtime_error(path + " is not a checkpoint");
  if (hdr[0] != n) throw std::runtime_error(path + ": grid " + std::to_string(hdr[0]) + " != " + std::to_string(n));
  const std::size_t full = static_cast<std::size_t>(n) * n * n;
  const std::size_t nh = static_cast<std::size_t>(n / 2 + 1);
  std::vector<double> buf(3 * 2 * full, 0.0);
  double* st[3] = {buf.data(), buf.data() + 2 * full, buf.data() + 4 * full};
  for (int c = 0; c < 3; ++c)
    for (std::size_t row = 0; row < static_cast<std::size_t>(n) * n; ++row)
      f.read(reinterpret_cast<char*>(st[c] + 2 * row * n), static_cast<std::streamsize>(2 * nh * sizeof(double)));
  if (!f) throw std::runtime_error(path + ": truncated checkpoint");
  // the state stores mx in [0, n/2]; set_state reads only those columns of the full layout
  const double* cst[3] = {st[0], st[1], st[2]};
  impl_->check(sns_set_state(impl_->h, cst), "TaylorGreenSolver::load_checkpoint");
  *t = t0;
  *step = step64;
}

void run_taylor_green(const RunConfig& config) {
  if (config.dt <= 0.0 || config.cfl <= 0.0 || config.output_dt <= 0.0)
    throw std::runtime_error("--dt, --cfl, and --output-dt must be positive");
  std::filesystem::create_directories(config.output_dir);
  const std::string csv_path = config.output_dir + "/taylor_green_diagnostics.csv";
  const std::string ckpt_path = config.output_dir + "/checkpoint.bin";
  const bool resume = !config.restart.empty();
  std::ofstream csv(csv_path, resume ? std::ios::app : std::ios::trunc);
  csv << std::setprecision(17);
  if (!resume)
    csv << "t,kinetic_energy,dissipation,enstrophy,max_spectral_divergence,max_velocity,dt,cfl,main_dt,main_cfl\n";

  const double init_t0 = wall();
  TaylorGreenSolver solver(config.n, config.reynolds, config.seed, config.pert_amp, config.pert_kmax, config.precision,
                           config.viscous_mode);
  double t = 0.0;
  int step = 0;
  if (resume) {
    long long s0 = 0;
    solver.load_checkpoint(config.restart, &t, &s0);
    step = static_cast<int>(s0);
    std::cout << "resumed from " << config.restart << " at step " << step << " t=" << t << "\n";
  }
  const int first_step = step;
  auto checkpoint = [&](int s) {
    if (config.checkpoint_every > 0 && s > first_step && s % config.checkpoint_every == 0)
      solver.save_checkpoint(ckpt_path, t, s);
  };
  const double init_time = wall() - init_t0;
  const double run_t0 = wall();
  const double dx = 2.0 * kPi / static_cast<double>(config.n);
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
    if (!resume) {
      write_row(t, true, 0.0, 0.0, 0.0, 0.0);
      next_output += config.output_dt;
    } else {
      while (next_output <= t + 1.0e-12) next_output += config.output_dt;
    }
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
      checkpoint(step);
    }
  } else {
    for (; step <= config.steps; ++step) {
      checkpoint(step);
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
