// SpectralNavierStokes over B200Fft3D (the reference's src/spectral_solver.cpp:35-488 API).
//
// rhs / nonlinear_rhs / step_rk3 / the diagnostics / product_dealiased / the vorticity slice
// run on the GPU: on the benchmark domain (cubic, L = 2 pi, a planned n, phase-shift
// dealiasing) through the fused passes of the backend's solver handle, on every other domain
// (any shape, any lengths, either product form) through the generic-shape device path
// (sns_fft3d_*).  The remaining host-vector helpers (project, truncate, vorticity_hat,
// kinetic_energy of a physical field, max_spectral_divergence) keep the reference's
// semantics on the host.
#include "spectral/spectral_solver.hpp"

#include "sns_b200.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <fstream>
#include <iomanip>
#include <stdexcept>

namespace spectral {

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;
using Clock = std::chrono::steady_clock;

double seconds_since(Clock::time_point t0) { return std::chrono::duration<double>(Clock::now() - t0).count(); }

std::complex<double> at(const std::vector<double>& a, std::size_t id) { return {a[id], a[id + 1]}; }
void put(std::vector<double>& a, std::size_t id, std::complex<double> z) {
  a[id] = z.real();
  a[id + 1] = z.imag();
}

void check(int rc, sns_handle* h, const char* what) {
  if (rc != SNS_OK) throw std::runtime_error(std::string(what) + ": " + sns_last_error(h));
}
void check(int rc, sns_fft3d* h, const char* what) {
  if (rc != SNS_OK) throw std::runtime_error(std::string(what) + ": " + sns_fft3d_last_error(h));
}

VectorSpectral zeros_spectral(std::size_t n) { return {ScalarSpectral(n, 0.0), ScalarSpectral(n, 0.0), ScalarSpectral(n, 0.0)}; }

}  // namespace

struct SpectralNavierStokes::DeviceDiag {
  sns_diag d;
};

SpectralNavierStokes::SpectralNavierStokes(std::array<int, 3> shape, std::array<double, 3> lengths, double viscosity,
                                           MPI_Comm comm, bool phase_shift_dealiasing)
    : fft_(shape, lengths, comm), nu_(viscosity), phase_shift_dealiasing_(phase_shift_dealiasing) {
  if (nu_ < 0.0) throw std::runtime_error("viscosity must be non-negative");
  const std::size_t nmodes = fft_.spectral_storage_size() / 2;
  phase_shift_.resize(nmodes);
  keep_mode_mask_.resize(nmodes);
  const auto& L = fft_.lengths();
  const auto& n = fft_.shape();
  // half-cell shift dx = L/(2n) on every axis, as src/spectral_solver.cpp:48-54
  const double hx = 0.5 * L[0] / n[0], hy = 0.5 * L[1] / n[1], hz = 0.5 * L[2] / n[2];
  fft_.for_each_spectral([&](std::size_t id, const SpectralMode& m) {
    phase_shift_[id / 2] = std::exp(std::complex<double>(0.0, m.kx * hx + m.ky * hy + m.kz * hz));
    keep_mode_mask_[id / 2] = keep_mode(m) ? 1 : 0;
  });
  fused_ = phase_shift_dealiasing_ && fft_.fused_domain();
}

SpectralNavierStokes::~SpectralNavierStokes() = default;

sns_handle* SpectralNavierStokes::solver_handle() {
  sns_handle* h = fft_.handle();
  check(sns_set_viscosity(h, nu_), h, "SpectralNavierStokes");
  return h;
}

VectorPhysical SpectralNavierStokes::taylor_green(double amplitude, int mode) const {
  const auto& n = fft_.shape();
  const auto& L = fft_.lengths();
  const std::size_t np = static_cast<std::size_t>(fft_.physical_size());
  VectorPhysical u = {ScalarPhysical(np, 0.0), ScalarPhysical(np, 0.0), ScalarPhysical(np, 0.0)};
  fft_.for_each_physical([&](std::size_t id, int ix, int iy, int iz) {
    const double ax = 2.0 * kPi * mode * ((ix + 0.5) * L[0] / n[0]) / L[0];
    const double ay = 2.0 * kPi * mode * ((iy + 0.5) * L[1] / n[1]) / L[1];
    const double az = 2.0 * kPi * mode * ((iz + 0.5) * L[2] / n[2]) / L[2];
    u[0][id] = amplitude * std::sin(ax) * std::cos(ay) * std::cos(az);
    u[1][id] = -amplitude * std::cos(ax) * std::sin(ay) * std::cos(az);
  });
  return u;
}

VectorSpectral SpectralNavierStokes::to_spectral(const VectorPhysical& u) {
  VectorSpectral out;
  for (int c = 0; c < 3; ++c) out[c] = fft_.forward(u[c]);
  return out;
}

VectorPhysical SpectralNavierStokes::to_physical(const VectorSpectral& u_hat) {
  VectorPhysical out;
  for (int c = 0; c < 3; ++c) out[c] = fft_.backward(u_hat[c]);
  return out;
}

void SpectralNavierStokes::project(VectorSpectral& u_hat) const {
  fft_.for_each_spectral([&](std::size_t id, const SpectralMode& m) {
    if (m.k2 == 0.0) return;
    const auto ux = at(u_hat[0], id), uy = at(u_hat[1], id), uz = at(u_hat[2], id);
    const auto f = (m.kx * ux + m.ky * uy + m.kz * uz) / m.k2;
    put(u_hat[0], id, ux - m.kx * f);
    put(u_hat[1], id, uy - m.ky * f);
    put(u_hat[2], id, uz - m.kz * f);
  });
  zero_mean(u_hat);
}

void SpectralNavierStokes::truncate(VectorSpectral& u_hat) const {
  fft_.for_each_spectral([&](std::size_t id, const SpectralMode&) {
    if (keep_mode_mask_[id / 2]) return;
    for (auto& comp : u_hat) comp[id] = comp[id + 1] = 0.0;
  });
}

ScalarSpectral SpectralNavierStokes::product_dealiased(const ScalarSpectral& a_hat, const ScalarSpectral& b_hat) {
  // both products, their transforms and the combine on the device (src/spectral_solver.cpp:122-158)
  if (a_hat.size() != fft_.spectral_storage_size() || b_hat.size() != fft_.spectral_storage_size())
    throw std::runtime_error("spectral field has wrong storage size");
  ScalarSpectral out(fft_.spectral_storage_size(), 0.0);
  sns_fft3d* g = fft_.generic();
  check(sns_fft3d_product(g, a_hat.data(), b_hat.data(), out.data()), g, "SpectralNavierStokes::product_dealiased");
  return out;
}

VectorSpectral SpectralNavierStokes::nonlinear_rhs(const VectorSpectral& u_hat) {
  const auto t0 = Clock::now();
  profile_.nonlinear_calls += 1;
  VectorSpectral out = zeros_spectral(fft_.spectral_storage_size());
  const double* in[3] = {u_hat[0].data(), u_hat[1].data(), u_hat[2].data()};
  double* o[3] = {out[0].data(), out[1].data(), out[2].data()};
  if (fused_) {
    sns_handle* h = solver_handle();
    check(sns_nonlinear(h, in, o), h, "SpectralNavierStokes::nonlinear_rhs");
  } else {
    sns_fft3d* g = fft_.generic();
    check(sns_fft3d_rhs(g, nu_, phase_shift_dealiasing_ ? 1 : 0, 0, in, o), g, "SpectralNavierStokes::nonlinear_rhs");
  }
  profile_.nonlinear_rhs += seconds_since(t0);
  return out;
}

VectorSpectral SpectralNavierStokes::rhs(const VectorSpectral& u_hat) {
  const auto t0 = Clock::now();
  profile_.rhs_calls += 1;
  VectorSpectral out = zeros_spectral(fft_.spectral_storage_size());
  const double* in[3] = {u_hat[0].data(), u_hat[1].data(), u_hat[2].data()};
  double* o[3] = {out[0].data(), out[1].data(), out[2].data()};
  if (fused_) {
    sns_handle* h = solver_handle();
    check(sns_rhs(h, in, o), h, "SpectralNavierStokes::rhs");
  } else {
    sns_fft3d* g = fft_.generic();
    check(sns_fft3d_rhs(g, nu_, phase_shift_dealiasing_ ? 1 : 0, 1, in, o), g, "SpectralNavierStokes::rhs");
  }
  profile_.rhs += seconds_since(t0);
  return out;
}

VectorSpectral SpectralNavierStokes::step_rk3(const VectorSpectral& u_hat, double t, double dt) {
  (void)t;
  const auto t0 = Clock::now();
  profile_.steps += 1;
  VectorSpectral out;
  if (fused_) {
    sns_handle* h = solver_handle();
    const double* in[3] = {u_hat[0].data(), u_hat[1].data(), u_hat[2].data()};
    check(sns_set_state(h, in), h, "SpectralNavierStokes::step_rk3");
    check(sns_step(h, dt, 1), h, "SpectralNavierStokes::step_rk3");
    out = zeros_spectral(fft_.spectral_storage_size());
    double* o[3] = {out[0].data(), out[1].data(), out[2].data()};
    check(sns_get_state(h, o), h, "SpectralNavierStokes::step_rk3");
  } else {
    out = u_hat;
    double* o[3] = {out[0].data(), out[1].data(), out[2].data()};
    sns_fft3d* g = fft_.generic();
    check(sns_fft3d_step(g, nu_, phase_shift_dealiasing_ ? 1 : 0, dt, 1, o), g, "SpectralNavierStokes::step_rk3");
  }
  profile_.step_rk3 += seconds_since(t0);
  return out;
}

double SpectralNavierStokes::kinetic_energy(const VectorPhysical& u) const {
  double sum = 0.0;
  for (std::size_t i = 0; i < u[0].size(); ++i) sum += 0.5 * (u[0][i] * u[0][i] + u[1][i] * u[1][i] + u[2][i] * u[2][i]);
  double total = 0.0;
  MPI_Allreduce(&sum, &total, 1, MPI_DOUBLE, MPI_SUM, fft_.comm());
  return total / static_cast<double>(fft_.global_physical_size());
}

SpectralNavierStokes::DeviceDiag SpectralNavierStokes::device_diagnostics(const VectorSpectral& u_hat) {
  const double* in[3] = {u_hat[0].data(), u_hat[1].data(), u_hat[2].data()};
  DeviceDiag d{};
  if (fused_) {
    sns_handle* h = solver_handle();
    check(sns_set_state(h, in), h, "SpectralNavierStokes diagnostics");
    check(sns_diagnostics(h, 0.0, &d.d), h, "SpectralNavierStokes diagnostics");
  } else {
    sns_fft3d* g = fft_.generic();
    check(sns_fft3d_diagnostics(g, nu_, in, 0.0, &d.d), g, "SpectralNavierStokes diagnostics");
  }
  return d;
}

double SpectralNavierStokes::kinetic_energy_spectral(const VectorSpectral& u_hat) {
  return device_diagnostics(u_hat).d.kinetic_energy;
}

double SpectralNavierStokes::max_velocity(const VectorSpectral& u_hat) {
  return device_diagnostics(u_hat).d.max_velocity;
}

VectorSpectral SpectralNavierStokes::vorticity_hat(const VectorSpectral& u_hat) const {
  VectorSpectral w = zeros_spectral(fft_.spectral_storage_size());
  const std::complex<double> I(0.0, 1.0);
  fft_.for_each_spectral([&](std::size_t id, const SpectralMode& m) {
    const auto ux = at(u_hat[0], id), uy = at(u_hat[1], id), uz = at(u_hat[2], id);
    put(w[0], id, I * (m.ky * uz - m.kz * uy));
    put(w[1], id, I * (m.kz * ux - m.kx * uz));
    put(w[2], id, I * (m.kx * uy - m.ky * ux));
  });
  return w;
}

double SpectralNavierStokes::enstrophy(const VectorSpectral& u_hat) { return device_diagnostics(u_hat).d.enstrophy; }

double SpectralNavierStokes::dissipation(const VectorSpectral& u_hat) { return 2.0 * nu_ * enstrophy(u_hat); }

double SpectralNavierStokes::max_spectral_divergence(const VectorSpectral& u_hat) const {
  double mx = 0.0;
  fft_.for_each_spectral([&](std::size_t id, const SpectralMode& m) {
    mx = std::max(mx, std::abs(m.kx * at(u_hat[0], id) + m.ky * at(u_hat[1], id) + m.kz * at(u_hat[2], id)));
  });
  double total = 0.0;
  MPI_Allreduce(&mx, &total, 1, MPI_DOUBLE, MPI_MAX, fft_.comm());
  return total;
}

Diagnostics SpectralNavierStokes::diagnostics(const VectorSpectral& u_hat, double t) {
  const auto t0 = Clock::now();
  const auto d = device_diagnostics(u_hat).d;
  Diagnostics row{t, d.kinetic_energy, 2.0 * nu_ * d.enstrophy, d.enstrophy, d.max_spectral_divergence};
  profile_.diagnostics += seconds_since(t0);
  return row;
}

// On the benchmark domain the state stays in HBM between calls; elsewhere it is kept on the
// host and each step_rk3(dt, n) uploads it once, takes the n steps on the device and reads
// it back.
void SpectralNavierStokes::load_state(const VectorSpectral& u_hat) {
  if (fused_) {
    sns_handle* h = solver_handle();
    const double* in[3] = {u_hat[0].data(), u_hat[1].data(), u_hat[2].data()};
    check(sns_set_state(h, in), h, "SpectralNavierStokes::load_state");
  } else {
    for (const auto& c : u_hat)
      if (c.size() != fft_.spectral_storage_size()) throw std::runtime_error("spectral field has wrong storage size");
    state_ = u_hat;
  }
}

void SpectralNavierStokes::step_rk3(double dt, int nsteps) {
  const auto t0 = Clock::now();
  if (fused_) {
    sns_handle* h = solver_handle();
    check(sns_step(h, dt, nsteps), h, "SpectralNavierStokes::step_rk3");
  } else {
    if (state_[0].empty()) throw std::runtime_error("SpectralNavierStokes::step_rk3: no state loaded");
    double* o[3] = {state_[0].data(), state_[1].data(), state_[2].data()};
    sns_fft3d* g = fft_.generic();
    check(sns_fft3d_step(g, nu_, phase_shift_dealiasing_ ? 1 : 0, dt, nsteps, o), g,
          "SpectralNavierStokes::step_rk3");
  }
  profile_.steps += nsteps;
  profile_.step_rk3 += seconds_since(t0);
}

Diagnostics SpectralNavierStokes::diagnostics(double t) {
  const auto t0 = Clock::now();
  sns_diag d{};
  if (fused_) {
    sns_handle* h = solver_handle();
    check(sns_diagnostics(h, t, &d), h, "SpectralNavierStokes::diagnostics");
  } else {
    if (state_[0].empty()) throw std::runtime_error("SpectralNavierStokes::diagnostics: no state loaded");
    const double* in[3] = {state_[0].data(), state_[1].data(), state_[2].data()};
    sns_fft3d* g = fft_.generic();
    check(sns_fft3d_diagnostics(g, nu_, in, t, &d), g, "SpectralNavierStokes::diagnostics");
  }
  profile_.diagnostics += seconds_since(t0);
  return Diagnostics{t, d.kinetic_energy, 2.0 * nu_ * d.enstrophy, d.enstrophy, d.max_spectral_divergence};
}

VectorSpectral SpectralNavierStokes::state() {
  if (!fused_) return state_;
  sns_handle* h = solver_handle();
  VectorSpectral out = zeros_spectral(fft_.spectral_storage_size());
  double* o[3] = {out[0].data(), out[1].data(), out[2].data()};
  check(sns_get_state(h, o), h, "SpectralNavierStokes::state");
  return out;
}

void SpectralNavierStokes::reset_profile() { profile_ = SolverProfile{}; }

bool SpectralNavierStokes::keep_mode(const SpectralMode& m) const {
  const auto& n = fft_.shape();
  const double hx = n[0] / 2.0, hy = n[1] / 2.0, hz = n[2] / 2.0;
  return (m.mx * m.mx) / (hx * hx) + (m.my * m.my) / (hy * hy) + (m.mz * m.mz) / (hz * hz) <= 1.0;
}

void SpectralNavierStokes::zero_mean(VectorSpectral& u_hat) const {
  for (auto& comp : u_hat) comp[0] = comp[1] = 0.0;  // mode (0,0,0) sits at index 0
}

void write_diagnostics_csv(const std::string& path, const std::vector<Diagnostics>& history) {
  std::ofstream f(path);
  f << "t,kinetic_energy,dissipation,enstrophy,max_spectral_divergence\n" << std::setprecision(17);
  for (const auto& r : history)
    f << r.t << ',' << r.energy << ',' << r.dissipation << ',' << r.enstrophy << ',' << r.max_spectral_divergence << '\n';
}

void write_vorticity_ppm(const std::string& path, SpectralNavierStokes& solver, const VectorSpectral& u_hat) {
  // |omega| on the mid z plane as a binary PPM (src/spectral_solver.cpp:421-486): omega_hat,
  // its inverse transforms and the slice's magnitudes on the device; only the n0 x n1 slice
  // comes back, and the palette below is the reference's
  const auto& n = solver.fft().shape();
  const int iz = n[2] / 2;
  std::vector<double> mag(static_cast<std::size_t>(n[0]) * n[1]);
  for (const auto& c : u_hat)
    if (c.size() != solver.fft().spectral_storage_size()) throw std::runtime_error("spectral field has wrong storage size");
  const double* in[3] = {u_hat[0].data(), u_hat[1].data(), u_hat[2].data()};
  sns_fft3d* g = solver.fft().generic();
  check(sns_fft3d_vorticity_slice(g, in, iz, mag.data()), g, "write_vorticity_ppm");
  double vmax = 0.0;
  for (double v : mag) vmax = std::max(vmax, v);
  if (vmax == 0.0) vmax = 1.0;
  std::ofstream f(path, std::ios::binary);
  f << "P6\n" << n[0] << " " << n[1] << "\n255\n";
  for (int iy = n[1] - 1; iy >= 0; --iy)
    for (int ix = 0; ix < n[0]; ++ix) {
      const double q = std::clamp(mag[static_cast<std::size_t>(ix + n[0] * iy)] / vmax, 0.0, 1.0);
      const unsigned char rgb[3] = {static_cast<unsigned char>(255.0 * std::sqrt(q)),
                                    static_cast<unsigned char>(255.0 * q * q),
                                    static_cast<unsigned char>(255.0 * (1.0 - q) * 0.25)};
      f.write(reinterpret_cast<const char*>(rgb), 3);
    }
}

}  // namespace spectral
