// Kernel-side declarations shared by the pass kernels and the C-ABI host code.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace sns {

// Geometry of a half-spectrum field: rows (z, y) of `pitch` double2, columns
// mx in [0, nh) hold data, column nh holds the mx = N/2 (Nyquist) plane, columns
// nh+1 .. pitch-1 are zero padding that keeps every row 128-byte aligned.
struct Geom {
  int n;
  int nh;
  int pitch;
  long long field;  // double2 elements per half field = n*n*pitch
};

__host__ __device__ inline int pitch_for(int n) { return ((n / 2 + 1) + 7) / 8 * 8; }

// Per-stage scalars of the fused k-space sweep (the reference's Real-typed RK products,
// ava_taylor_green_impl.hpp:998, 1014, 1030).
struct SweepArgs {
  double nu;
  double ga;       // g <- ga*g + r   (stage 1: unused, g <- r)
  double ub;       // u <- u + ub*g
  int stage;       // 0, 1, 2
  int mode;        // 0: RK update of (u, g); 1: projected RHS to `rhs`; 2: masked nonlinear term only
  int dealias;     // 1: phase-shift pair, 0: plain product only
};

// Arguments of the TMA-fed streaming y/z pass.
struct TmaArgs {
  int f_in0;      // first field of the tensor map to read
  int nf;         // number of fields
  int ncb;        // 8-column tiles per row
  double2* out;   // output field set (field 0)
  int f_out0;     // first output field (phase variant: 2 outputs per input field)
  double scale;   // applied to every element on load
  int* err;       // device error word (bounded-wait timeout)
};

// Launch table for one grid size.  All launches go to `st`.
struct Ops {
  int n;
  void (*init)();  // kernel attributes; call once before the first launch
  // inverse z pass of u[3] with the phase shift: work fields 2c (U_c), 2c+1 (phase*U_c)
  void (*zpass_inv_phase)(const double2* u, double2* work, const double2* tw, const double2* phase,
                          double scale, int ntiles, Geom g, cudaStream_t st);
  // y pass (dir -1 forward, +1 inverse) of `nf` consecutive fields, in place; `ncols` tiles of 8 columns
  void (*ypass)(double2* f, int nf, int dir, int ntiles, const double2* tw, Geom g, cudaStream_t st);
  // z pass src -> dst (may alias), optional scale applied on load
  void (*zpass)(const double2* src, double2* dst, int nf, int dir, int ntiles, double scale, const double2* tw,
                Geom g, cudaStream_t st);
  // fused x pass: 6 inverse fields -> 12 product half-spectra; optional energy/vmax partials
  void (*xpass_products)(double2* work, const double2* unyq, const double2* phase, double scale,
                         int nyq_scalar, double* partials, const double2* tw, Geom g, cudaStream_t st);
  // Nyquist-plane sums of the 12 product fields (column nh, summed over rows)
  void (*nyq_reduce)(const double2* work, double* sums, Geom g, cudaStream_t st);
  // fused k-space sweep; rhs may be null in RK mode; the (N/2,0,0) product values are the
  // fixed-order sums of nparts partials per field ([field][nparts])
  void (*sweep)(const double2* work, double2* u, double2* gbuf, double2* rhs, const double* nyq_part, int nparts,
                const double2* phase, SweepArgs a, Geom g, cudaStream_t st);
  // generic real rows -> half rows (x r2c), nf fields of real data with row pitch n doubles
  void (*xpass_r2c)(const double* in, double2* out, int nf, const double2* tw, Geom g, cudaStream_t st);
  // generic half rows -> real rows (x c2r), Hermitian-part rule at mx = 0 and N/2
  void (*xpass_c2r)(const double2* in, double* out, int nf, const double2* tw, Geom g, cudaStream_t st);
  // physical velocity energy / vmax partials from 3 inverse-transformed fields
  void (*xpass_diag)(const double2* work, const double2* unyq, double scale, int nyq_scalar,
                     double* partials, const double2* tw, Geom g, cudaStream_t st);
  // persistent TMA-fed y (axis 1) or z (axis 2) pass; variant 1 = inverse z with the phase shift
  void (*yz_tma)(const CUtensorMap& map, int axis, int dir, int variant, TmaArgs a, const double2* tw,
                 const double2* phase, Geom g, int grid, cudaStream_t st);
  int (*tma_blocks_per_sm)();
  // two-stage persistent x pass (N = 256, 512); writes [12][grid] Nyquist partials
  void (*xpass2)(double2* work, const double2* unyq, const double2* phase, double scale, int nyq_scalar,
                 double* nyq_part, const double2* tw2, Geom g, int grid, int* err, cudaStream_t st);
  int (*xpass2_grid)(int nsm);
  // fused forward z pass + k-space sweep (N = 128, 256, 512), TMA-fed, accumulators in TMEM
  void (*p5)(const CUtensorMap& map, double2* u, double2* gbuf, double2* rhs, const double* nyq_part, int nparts,
             const double2* tw, const double2* phase, SweepArgs a, int ncb, Geom g, int grid, int* err,
             cudaStream_t st);
  int (*p5_grid)(int nsm);
};

const Ops* ops_for(int n);  // nullptr when the size has no FFT plan

// Size-independent kernels -------------------------------------------------------------
void launch_tgv_init(double* phys, Geom g, cudaStream_t st);
void launch_project_truncate(double2* u, Geom g, cudaStream_t st);
void launch_add_sparse(double2* u, const long long* idx, const double2* val, int count, cudaStream_t st);
void launch_half_to_full(const double2* half, double2* full, Geom g, cudaStream_t st);
void launch_full_to_half(const double2* full, double2* half, int hermitian_part, Geom g, cudaStream_t st);
void launch_spectral_diag(const double2* u, double* partials, int nblocks, Geom g, cudaStream_t st);
void launch_reduce(const double* partials, int count, int stride, int op_max, double* out, cudaStream_t st);

// Host helpers shared by the C-ABI files (sns_api.cu).
void fill_twiddles(int L, double2* tw);        // exp(-2*pi*i*t/L), t < L
void set_handleless_error(const char* msg);    // message for sns_last_error(NULL)

constexpr int kXDiagPartials = 2;   // (sum 0.5|u|^2, max |u|^2) per row
constexpr int kSpecDiagPartials = 2;  // (sum w*|H(omega)|^2, max |k.u|) per block

}  // namespace sns
