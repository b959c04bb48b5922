// B200Fft3D: FftwFft3D's contract (src/fftw_fft.hpp:13-81, src/fftw_fft.cpp) over libsns_b200.so.
#include "spectral/b200_fft.hpp"

#include "sns_b200.h"

#include <stdexcept>
#include <string>

namespace spectral {

namespace {

void check(int rc, sns_handle* h, const char* what) {
  if (rc != SNS_OK) throw std::runtime_error(std::string(what) + ": " + sns_last_error(h));
}

}  // namespace

B200Fft3D::B200Fft3D(std::array<int, 3> shape, std::array<double, 3> lengths, MPI_Comm comm)
    : shape_(shape), lengths_(lengths) {
  int comm_size = 0;
  MPI_Comm_size(comm, &comm_size);
  if (comm_size != 1) throw std::runtime_error("The B200 backend runs one solve per GPU; it supports one MPI rank");
  for (int n : shape_) {
    if (n <= 1) throw std::runtime_error("all grid sizes must be greater than one");
  }
  for (double length : lengths_) {
    if (length <= 0.0) throw std::runtime_error("all domain lengths must be positive");
  }
  if (shape_[0] != shape_[1] || shape_[1] != shape_[2])
    throw std::runtime_error("The B200 backend supports cubic grids (n x n x n)");
  const int rc = sns_create(shape_[0], 0.0, SNS_PRECISION_FP64, SNS_VISCOUS_EXPLICIT, 0, 0.0, 0, &handle_);
  if (rc != SNS_OK) throw std::runtime_error(std::string("B200Fft3D: ") + sns_last_error(nullptr));
}

B200Fft3D::~B200Fft3D() {
  if (handle_ != nullptr) sns_destroy(handle_);
}

std::vector<double> B200Fft3D::forward(const std::vector<double>& physical) {
  if (physical.size() != static_cast<std::size_t>(physical_size()))
    throw std::runtime_error("physical field has wrong size");
  std::vector<double> spectral(spectral_storage_size(), 0.0);
  check(sns_forward_r2c(handle_, physical.data(), spectral.data()), handle_, "B200Fft3D::forward");
  return spectral;
}

std::vector<double> B200Fft3D::backward(const std::vector<double>& spectral) {
  if (spectral.size() != spectral_storage_size()) throw std::runtime_error("spectral field has wrong storage size");
  std::vector<double> physical(static_cast<std::size_t>(physical_size()), 0.0);
  check(sns_backward_c2r(handle_, spectral.data(), physical.data()), handle_, "B200Fft3D::backward");
  return physical;
}

}  // namespace spectral
