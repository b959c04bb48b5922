// Command-line driver: the reference's flags (src/main_ava.cpp:43-73) plus
// --seed --pert-amp --pert-kmax --dump-final --precision fp64|fp32 --viscous explicit|if
// --checkpoint-every K --restart PATH.
#include "spectral/ava_taylor_green.hpp"

#include <algorithm>
#include <cstdint>
#include <exception>
#include <iostream>
#include <stdexcept>
#include <string>

namespace {

const char* find_arg(int argc, char** argv, const std::string& name) {
  for (int i = 1; i + 1 < argc; ++i)
    if (argv[i] == name) return argv[i + 1];
  return nullptr;
}
int int_arg(int argc, char** argv, const std::string& name, int fallback) {
  const char* v = find_arg(argc, argv, name);
  return v ? std::stoi(v) : fallback;
}
double double_arg(int argc, char** argv, const std::string& name, double fallback) {
  const char* v = find_arg(argc, argv, name);
  return v ? std::stod(v) : fallback;
}
std::string string_arg(int argc, char** argv, const std::string& name, const std::string& fallback) {
  const char* v = find_arg(argc, argv, name);
  return v ? std::string(v) : fallback;
}

}  // namespace

int main(int argc, char** argv) {
  try {
    spectral::ava_solver::RunConfig c;
    c.n = int_arg(argc, argv, "--n", c.n);
    c.steps = int_arg(argc, argv, "--steps", c.steps);
    c.max_steps = int_arg(argc, argv, "--max-steps", c.max_steps);
    c.output_every = std::max(1, int_arg(argc, argv, "--output-every", c.output_every));
    c.print_every = std::max(1, int_arg(argc, argv, "--print-every", c.print_every));
    c.adaptive_cfl = int_arg(argc, argv, "--adaptive-cfl", c.adaptive_cfl ? 1 : 0) != 0;
    c.dt = double_arg(argc, argv, "--dt", c.dt);
    c.cfl = double_arg(argc, argv, "--cfl", c.cfl);
    c.t_end = double_arg(argc, argv, "--t-end", c.steps * c.dt);
    c.output_dt = double_arg(argc, argv, "--output-dt", c.output_dt);
    c.reynolds = double_arg(argc, argv, "--re", c.reynolds);
    c.output_dir = string_arg(argc, argv, "--output-dir", c.output_dir);
    c.seed = static_cast<std::uint64_t>(std::stoull(string_arg(argc, argv, "--seed", "0")));
    c.pert_amp = double_arg(argc, argv, "--pert-amp", c.pert_amp);
    c.pert_kmax = int_arg(argc, argv, "--pert-kmax", c.pert_kmax);
    c.dump_final = int_arg(argc, argv, "--dump-final", 0) != 0;
    const std::string prec = string_arg(argc, argv, "--precision", "fp64");
    if (prec != "fp64" && prec != "fp32") throw std::runtime_error("--precision must be fp64 or fp32");
    c.precision = prec == "fp32" ? 1 : 0;
    const std::string visc = string_arg(argc, argv, "--viscous", "explicit");
    if (visc != "explicit" && visc != "if") throw std::runtime_error("--viscous must be explicit or if");
    c.viscous_mode = visc == "if" ? 1 : 0;
    c.checkpoint_every = int_arg(argc, argv, "--checkpoint-every", 0);
    c.restart = string_arg(argc, argv, "--restart", "");
    spectral::ava_solver::run_taylor_green(c);
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << "\n";
    return 1;
  }
  return 0;
}
