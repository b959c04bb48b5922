// The reference's C++ tests (cpp_tests/spectral_ns_tests.cpp:16-51: 12^3 grid, L = 2*pi,
// nu = 0.05) run against SpectralNavierStokes over the B200 backend: on that grid (the fused
// passes), and again on an anisotropic grid with L = (1, 2, 3), with and without the
// phase-shift pair (the generic-shape device path).
#include "spectral/spectral_solver.hpp"

#include <cmath>
#include <fstream>
#include <iostream>
#include <stdexcept>

namespace {

void require(bool ok, const char* what) {
  if (!ok) throw std::runtime_error(what);
}

void fft_roundtrip(spectral::SpectralNavierStokes& s) {
  constexpr double pi = 3.141592653589793238462643383279502884;
  auto& fft = s.fft();
  const auto& n = fft.shape();
  std::vector<double> u(static_cast<std::size_t>(fft.physical_size()));
  fft.for_each_physical([&](std::size_t id, int ix, int iy, int) {
    u[id] = std::sin(2.0 * pi * (ix + 0.5) / n[0]) + 0.25 * std::cos(2.0 * pi * (iy + 0.5) / n[1]);
  });
  const auto back = fft.backward(fft.forward(u));
  double err = 0.0;
  for (std::size_t i = 0; i < u.size(); ++i) err = std::max(err, std::abs(u[i] - back[i]));
  require(err < 1.0e-10, "FFT roundtrip error too large");
}

void projection_and_energy(spectral::SpectralNavierStokes& s) {
  auto u = s.taylor_green();
  auto u_hat = s.to_spectral(u);
  s.project(u_hat);
  s.truncate(u_hat);
  require(s.max_spectral_divergence(u_hat) < 1.0e-8, "projection did not remove divergence");
  require(std::abs(s.kinetic_energy(u) - 0.125) < 1.0e-12, "Taylor-Green energy mismatch");
}

void viscous_decay(spectral::SpectralNavierStokes& s) {
  auto u_hat = s.to_spectral(s.taylor_green());
  s.project(u_hat);
  const double e0 = s.kinetic_energy_spectral(u_hat);
  const auto u1 = s.step_rk3(u_hat, 0.0, 1.0e-3);
  const double e1 = s.kinetic_energy_spectral(u1);
  require(e1 < e0, "viscous step did not reduce kinetic energy");
  require(s.max_spectral_divergence(u1) < 1.0e-7, "RK step left nonzero divergence");
}

// Not in the reference: the device-resident overloads step the same state bit for bit.
void resident_matches_host_vectors(spectral::SpectralNavierStokes& s) {
  auto u_hat = s.to_spectral(s.taylor_green());
  s.project(u_hat);
  s.truncate(u_hat);
  auto host = u_hat;
  for (int k = 0; k < 5; ++k) host = s.step_rk3(host, 0.0, 2.0e-3);
  s.load_state(u_hat);
  s.step_rk3(2.0e-3, 5);
  const auto dev = s.state();
  for (int c = 0; c < 3; ++c)
    for (std::size_t i = 0; i < dev[c].size(); ++i)
      require(dev[c][i] == host[c][i], "device-resident steps differ from host-vector steps");
  const auto a = s.diagnostics(0.01);
  const auto b = s.diagnostics(host, 0.01);
  require(a.energy == b.energy && a.enstrophy == b.enstrophy, "device-resident diagnostics differ");
}

// write_vorticity_ppm from the device slice: a binary PPM of n0 x n1 pixels.
void vorticity_ppm(spectral::SpectralNavierStokes& s, const char* path) {
  auto u_hat = s.to_spectral(s.taylor_green());
  s.project(u_hat);
  spectral::write_vorticity_ppm(path, s, u_hat);
  std::ifstream f(path, std::ios::binary);
  std::string magic;
  int w = 0, h = 0, mx = 0;
  f >> magic >> w >> h >> mx;
  f.get();
  std::vector<char> px(static_cast<std::size_t>(3 * w * h));
  f.read(px.data(), static_cast<std::streamsize>(px.size()));
  const auto& n = s.fft().shape();
  require(magic == "P6" && w == n[0] && h == n[1] && mx == 255 && f.gcount() == 3 * w * h, "PPM layout");
}

void run_all(spectral::SpectralNavierStokes& s, const char* ppm) {
  fft_roundtrip(s);
  projection_and_energy(s);
  viscous_decay(s);
  resident_matches_host_vectors(s);
  vorticity_ppm(s, ppm);
}

}  // namespace

int main() {
  try {
    constexpr double pi = 3.141592653589793238462643383279502884;
    spectral::SpectralNavierStokes s({12, 12, 12}, {2.0 * pi, 2.0 * pi, 2.0 * pi}, 0.05, MPI_COMM_WORLD);
    run_all(s, "vorticity_12.ppm");
    for (bool dealias : {true, false}) {
      spectral::SpectralNavierStokes g({12, 16, 8}, {1.0, 2.0, 3.0}, 0.05, MPI_COMM_WORLD, dealias);
      run_all(g, "vorticity_12x16x8.ppm");
    }
    std::cout << "all C++ spectral tests passed (B200 backend)\n";
  } catch (const std::exception& e) {
    std::cerr << "test failure: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
