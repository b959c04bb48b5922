// B200Fft3D: FftwFft3D's contract (src/fftw_fft.hpp:13-81, src/fftw_fft.cpp) over libsns_b200.so.
#include "spectral/b200_fft.hpp"

#include "sns_b200.h"

#include <cmath>
#include <stdexcept>
#include <string>

namespace spectral {

namespace {

constexpr double kTwoPiRef = 6.283185307179586476925286766559005768;

void check(int rc, sns_fft3d* h, const char* what) {
  if (rc != SNS_OK) throw std::runtime_error(std::string(what) + ": " + sns_fft3d_last_error(h));
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
  const int rc = sns_fft3d_create(shape_[0], shape_[1], shape_[2], lengths_[0], lengths_[1], lengths_[2], &fft_);
  if (rc != SNS_OK) throw std::runtime_error(std::string("B200Fft3D: ") + sns_last_error(nullptr));
}

B200Fft3D::~B200Fft3D() {
  if (handle_ != nullptr) sns_destroy(handle_);
  if (fft_ != nullptr) sns_fft3d_destroy(fft_);
}

bool B200Fft3D::fused_domain() const {
  if (shape_[0] != shape_[1] || shape_[1] != shape_[2] || !sns_grid_supported(shape_[0])) return false;
  for (double l : lengths_)
    if (std::abs(l - kTwoPiRef) > 1e-12 * kTwoPiRef) return false;
  return true;
}

sns_handle* B200Fft3D::handle() {
  if (handle_ == nullptr) {
    if (!fused_domain())
      throw std::runtime_error("B200Fft3D: the fused passes serve cubic grids with L = 2*pi and a planned n");
    const int rc = sns_create(shape_[0], 0.0, SNS_PRECISION_FP64, SNS_VISCOUS_EXPLICIT, 0, 0.0, 0, &handle_);
    if (rc != SNS_OK) throw std::runtime_error(std::string("B200Fft3D: ") + sns_last_error(nullptr));
  }
  return handle_;
}

std::size_t B200Fft3D::device_bytes() const {
  return sns_fft3d_device_bytes(fft_) + (handle_ ? sns_device_bytes(handle_) : 0);
}

std::vector<double> B200Fft3D::forward(const std::vector<double>& physical) {
  if (physical.size() != static_cast<std::size_t>(physical_size()))
    throw std::runtime_error("physical field has wrong size");
  std::vector<double> spectral(spectral_storage_size(), 0.0);
  check(sns_fft3d_forward(fft_, physical.data(), spectral.data()), fft_, "B200Fft3D::forward");
  return spectral;
}

std::vector<double> B200Fft3D::backward(const std::vector<double>& spectral) {
  if (spectral.size() != spectral_storage_size()) throw std::runtime_error("spectral field has wrong storage size");
  std::vector<double> physical(static_cast<std::size_t>(physical_size()), 0.0);
  check(sns_fft3d_backward(fft_, spectral.data(), physical.data()), fft_, "B200Fft3D::backward");
  return physical;
}

}  // namespace spectral
