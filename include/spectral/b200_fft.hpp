// B200Fft3D: the reference's FFT-backend contract (class FftwFft3D, src/fftw_fft.hpp:13-81
// of ovankerm/Spectral_solver) backed by the sm_100a kernels of libsns_b200.so.
//
// Same constructor, accessors, host layouts and iteration order:
//   physical: N^3 doubles, x fastest, id = ix + n0*(iy + n1*iz)            (fftw_fft.hpp:30-40)
//   spectral: 2*N^3 doubles, interleaved complex, same order; mode m = i <= n/2 ? i : i - n,
//             k = 2*pi*m/L                                                  (fftw_fft.hpp:45-71)
// forward: unnormalised DFT, sign -1; backward: Re(IDFT)/N (fftw_fft.cpp:53-85), for any
// spectral input, Hermitian or not.  Value semantics, synchronous, one host thread.
// The transforms run on the GPU that is current when the object is constructed.
// Errors throw std::runtime_error as the reference's backend does.
// Grids: any nx, ny, nz > 1 (an axis up to 6400 points) and box lengths > 0, like
// FftwFft3D (fftw_fft.cpp:8-36).  The object holds one complex and one real field on the
// device (sns_fft3d, 24 bytes per grid point); the fused solver handle of the benchmark
// domain (cubic, L = 2 pi, n in {8, 12, 16, 24, 32, 48, 64, 96, 128, 256, 512}) is created
// only when a solver asks for it.
#pragma once

#include "spectral/mpi_shim.h"

#include <array>
#include <cstddef>
#include <vector>

struct sns_handle;
struct sns_fft3d;

namespace spectral {

// Mode descriptor handed to for_each_spectral (src/flups_fft.hpp:18-26).
struct SpectralMode {
  double kx = 0.0;
  double ky = 0.0;
  double kz = 0.0;
  double k2 = 0.0;
  int mx = 0;
  int my = 0;
  int mz = 0;
};

class B200Fft3D {
 public:
  B200Fft3D(std::array<int, 3> shape, std::array<double, 3> lengths, MPI_Comm comm);
  ~B200Fft3D();

  B200Fft3D(const B200Fft3D&) = delete;
  B200Fft3D& operator=(const B200Fft3D&) = delete;

  const std::array<int, 3>& shape() const { return shape_; }
  const std::array<double, 3>& lengths() const { return lengths_; }
  int physical_size() const { return shape_[0] * shape_[1] * shape_[2]; }
  int global_physical_size() const { return physical_size(); }
  std::size_t spectral_storage_size() const { return 2 * static_cast<std::size_t>(physical_size()); }
  MPI_Comm comm() const { return MPI_COMM_SELF; }
  int rank() const { return 0; }
  int comm_size() const { return 1; }

  template <class Func>
  void for_each_physical(Func&& func) const {
    for (int iz = 0; iz < shape_[2]; ++iz)
      for (int iy = 0; iy < shape_[1]; ++iy)
        for (int ix = 0; ix < shape_[0]; ++ix)
          func(static_cast<std::size_t>(ix + shape_[0] * (iy + shape_[1] * iz)), ix, iy, iz);
  }

  template <class Func>
  void for_each_spectral(Func&& func) const {
    for (int iz = 0; iz < shape_[2]; ++iz) {
      const int mz = mode_of(iz, 2);
      for (int iy = 0; iy < shape_[1]; ++iy) {
        const int my = mode_of(iy, 1);
        for (int ix = 0; ix < shape_[0]; ++ix) {
          SpectralMode m;
          m.mx = mode_of(ix, 0);
          m.my = my;
          m.mz = mz;
          m.kx = kTwoPi * m.mx / lengths_[0];
          m.ky = kTwoPi * m.my / lengths_[1];
          m.kz = kTwoPi * m.mz / lengths_[2];
          m.k2 = m.kx * m.kx + m.ky * m.ky + m.kz * m.kz;
          func(2 * static_cast<std::size_t>(ix + shape_[0] * (iy + shape_[1] * iz)), m);
        }
      }
    }
  }

  std::vector<double> forward(const std::vector<double>& physical);
  std::vector<double> backward(const std::vector<double>& spectral);

  // The generic-shape transform handle behind this backend (any grid).
  sns_fft3d* generic() const { return fft_; }
  // True for the benchmark domain the fused passes serve: cubic, L = 2 pi on every axis,
  // n with a fused plan.
  bool fused_domain() const;
  // The fused solver handle for that domain (created on first use; throws elsewhere).
  sns_handle* handle();
  // Device bytes held by the backend (the transform handle, plus the fused handle if made).
  std::size_t device_bytes() const;

 private:
  int mode_of(int idx, int dim) const { return idx <= shape_[dim] / 2 ? idx : idx - shape_[dim]; }

  static constexpr double kTwoPi = 6.283185307179586476925286766559005768;
  std::array<int, 3> shape_{};
  std::array<double, 3> lengths_{};
  sns_fft3d* fft_ = nullptr;
  sns_handle* handle_ = nullptr;
};

}  // namespace spectral
