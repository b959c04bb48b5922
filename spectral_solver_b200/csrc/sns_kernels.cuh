// Kernel-side declarations shared by the pass kernels and the C-ABI host code.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace sns {

// Geometry of a half-spectrum field: rows (z, y) of `pitch` complex values, columns
// mx in [0, nh) hold data, column nh holds the mx = N/2 (Nyquist) plane, columns
// nh+1 .. pitch-1 are zero padding that keeps every row 128-byte aligned.
struct Geom {
  int n;
  int nh;
  int pitch;
  long long field;  // complex elements per half field = n*n*pitch
};

// Row pitch in complex elements: N/2 + 1 rounded up to a 128-byte row (8 complex doubles,
// 16 complex floats).
__host__ __device__ inline int pitch_for(int n, int complex_bytes) {
  const int per_row = 128 / complex_bytes;
  return ((n / 2 + 1) + per_row - 1) / per_row * per_row;
}
__host__ __device__ inline int pitch_for(int n) { return pitch_for(n, 16); }

// Compensation word of one complex value of u in the FP32 precision form: the remainder of
// the real and imaginary parts as signed multiples of 1/255 of their FP32 ulp (int8 each,
// real part in the low byte).
using CompWord = uint16_t;

// Per-stage scalars of the fused k-space sweep (the reference's Real-typed RK products,
// ava_taylor_green_impl.hpp:998, 1014, 1030).
struct SweepArgs {
  double nu;
  double ga;       // g <- ga*g + r   (stage 1: unused, g <- r)
  double ub;       // u <- u + ub*g
  double if_tau;   // integrating factor: u, g <- exp(-nu*k^2*if_tau) * (u, g) after the update
  int stage;       // 0, 1, 2
  int mode;        // 0: RK update of (u, g); 1: projected RHS to `rhs`; 2: masked nonlinear term only
  int dealias;     // 1: phase-shift pair, 0: plain product only
  int visc_if;     // 0: explicit viscous term in the RHS (the reference); 1: integrating factor
  // FP32 precision form, compensated state: one word per complex value of u (same index as
  // u) holding the part of the FP64 update that the FP32 value cannot; null: u is the FP32
  // value alone (and always in the FP64 form)
  CompWord* ulo;
  // Step taken on the device (adaptive CFL): null, or the handle's clock (kClock* slots),
  // whose current step size replaces the host's dt in ub and if_tau; when the clock is
  // stopped (its horizon reached) the stage leaves u and g as they are
  const double* clock;
  int frozen;  // set in the kernel from the clock
};

// Device clock of a solve stepped with an adaptive CFL step (doubles): the step size of the
// current step, time, horizon, CFL number, step cap, grid spacing, steps taken, stopped flag,
// and the viscosity (so a step graph captured once serves every solve a pooled handle runs).
enum { kClockDt = 0, kClockT, kClockTEnd, kClockCfl, kClockDtMax, kClockDx, kClockSteps, kClockStopped, kClockNu,
       kClockWords = 9 };

// Arguments of the TMA-fed streaming y/z pass.
struct TmaArgs {
  int f_in0;      // first field of the tensor map to read
  int nf;         // number of fields
  int ncb;        // tiles of 128-byte column blocks per row
  void* out;      // output field set (field 0)
  int f_out0;     // first output field (phase variant: 2 outputs per input field)
  double scale;   // applied to every element on load
  int* err;       // device error word (bounded-wait timeout)
};

// Launch table for one (grid size, precision).  Field and table pointers are complex
// arrays of the table's element type (double2 for FP64, float2 for FP32).  All launches go
// to `st`.
struct Ops {
  int n;
  int complex_bytes;  // 16 (FP64) or 8 (FP32)
  int tile_cols;      // columns per y/z tile (one 128-byte row segment)
  void (*init)();     // kernel attributes; call once per device before the first launch
  // inverse z pass of u[3] with the phase shift: work fields 2c (U_c), 2c+1 (phase*U_c)
  void (*zpass_inv_phase)(const void* u, void* work, const void* tw, const void* phase, double scale, int ntiles,
                          Geom g, cudaStream_t st);
  // y pass (dir -1 forward, +1 inverse) of `nf` consecutive fields, in place; `ntiles` column tiles
  void (*ypass)(void* f, int nf, int dir, int ntiles, const void* tw, Geom g, cudaStream_t st);
  // z pass src -> dst (may alias), optional scale applied on load
  void (*zpass)(const void* src, void* dst, int nf, int dir, int ntiles, double scale, const void* tw, Geom g,
                cudaStream_t st);
  // fused x pass: 6 inverse fields -> 12 product half-spectra; optional energy/vmax partials
  void (*xpass_products)(void* work, const void* unyq, const void* phase, double scale, int nyq_scalar,
                         double* partials, const void* tw, Geom g, cudaStream_t st);
  // Nyquist-plane sums of the 12 product fields (column nh, summed over rows)
  void (*nyq_reduce)(const void* work, double* sums, Geom g, cudaStream_t st);
  // fused k-space sweep; rhs may be null in RK mode; the (N/2,0,0) product values are the
  // fixed-order sums of nparts partials per field ([field][nparts])
  void (*sweep)(const void* work, void* u, void* gbuf, void* rhs, const double* nyq_part, int nparts,
                const void* phase, SweepArgs a, Geom g, cudaStream_t st);
  // generic real rows (doubles) -> half rows (x r2c), nf fields of real data with row pitch n
  void (*xpass_r2c)(const double* in, void* out, int nf, const void* tw, Geom g, cudaStream_t st);
  // generic half rows -> real rows (doubles, x c2r), Hermitian-part rule at mx = 0 and N/2
  void (*xpass_c2r)(const void* in, double* out, int nf, const void* tw, Geom g, cudaStream_t st);
  // physical velocity energy / vmax partials from 3 inverse-transformed fields
  void (*xpass_diag)(const void* work, const void* unyq, double scale, int nyq_scalar, double* partials,
                     const void* tw, Geom g, cudaStream_t st);
  // persistent TMA-fed y (axis 1) or z (axis 2) pass; variant 1 = inverse z with the phase shift
  void (*yz_tma)(const CUtensorMap& map, int axis, int dir, int variant, TmaArgs a, const void* tw,
                 const void* phase, Geom g, int grid, cudaStream_t st);
  int (*tma_blocks_per_sm)();
  // two-stage persistent x pass (N = 256, 512); writes [12][grid] Nyquist partials
  void (*xpass2)(void* work, const void* unyq, const void* phase, double scale, int nyq_scalar, double* nyq_part,
                 const void* tw2, Geom g, int grid, int* err, cudaStream_t st);
  int (*xpass2_grid)(int nsm);
  // fused forward z pass + k-space sweep (N = 128, 256, 512), TMA-fed, accumulators in TMEM;
  // `live` (nlive entries of my * ncb + cb) restricts it to those tiles, null: all
  void (*p5)(const CUtensorMap& map, void* u, void* gbuf, void* rhs, const double* nyq_part, int nparts,
             const void* tw, const void* phase, SweepArgs a, int ncb, const int* live, int nlive, Geom g, int grid,
             int* err, cudaStream_t st);
  int (*p5_grid)(int nsm);
  // rotational form: omega_hat = i k x u_hat (3 fields); the x pass forming u x omega on both
  // grids (12 inputs -> 6 outputs in work fields 0..5); the sweep combining the two grids
  void (*omega_hat)(const void* u, void* w, Geom g, cudaStream_t st);
  void (*xpass_rot)(void* work, const void* unyq, const void* wnyq, const void* phase, double scale, int nyq_scalar,
                    const void* tw, Geom g, cudaStream_t st);
  void (*sweep_rot)(const void* work, void* u, void* gbuf, void* rhs, const double* nyq_sums, const void* phase,
                    SweepArgs a, Geom g, cudaStream_t st);
  // xpass_diag on the warp-per-row x pass where the handle runs it (FP32, N = 128, 256, 512;
  // grid = its x-pass grid, > 0: one (energy, vmax^2) pair per CTA), else xpass_diag (one pair
  // per row); returns the number of pairs written; tw2 as for xpass2
  int (*xpass_diag2)(const void* work, const void* unyq, double scale, int nyq_scalar, double* partials,
                     const void* tw, const void* tw2, Geom g, int grid, int* err, cudaStream_t st);
};

// nullptr when the size has no FFT plan; precision 0 = FP64, 1 = FP32
const Ops* ops_for(int n, int precision = 0);

// Size-independent kernels -------------------------------------------------------------
void launch_tgv_init(double* phys, Geom g, cudaStream_t st);
void launch_project_truncate(void* u, int precision, Geom g, cudaStream_t st);
void launch_add_sparse(void* u, int precision, const long long* idx, const double2* val, int count,
                       cudaStream_t st);
// half field <-> the reference's full layout (always complex doubles on that side)
// `lo` (FP32 form, may be null): the compensation words of the half field (see SweepArgs::ulo);
// half_to_full adds them, full_to_half writes the remainder the FP32 value drops
void launch_half_to_full(const void* half, int precision, double2* full, Geom g, cudaStream_t st,
                         const CompWord* lo = nullptr);
// src_pitch: complex values between rows of `full` (0: n, the full layout; n/2 + 1 when only
// the left half of each row was staged, which is all the plain conversion reads)
void launch_full_to_half(const double2* full, void* half, int precision, int hermitian_part, Geom g,
                         cudaStream_t st, CompWord* lo = nullptr, long long src_pitch = 0);
void launch_spectral_diag(const void* u, int precision, double* partials, int nblocks, Geom g, cudaStream_t st);
void launch_reduce(const double* partials, int count, int stride, int op_max, double* out, cudaStream_t st);
// The next step of a device clock from vmax^2 (the reference's adaptive rule,
// ava_taylor_green_impl.hpp:1363-1368): dt = min(dt_max, cfl dx / vmax), clipped to the
// horizon; stops the clock at the horizon; advances t and the step count.
void launch_clock_step(const double* vmax2, double* clock, cudaStream_t st);
void launch_clock_step_partials(const double* partials, int count, int stride, double* clock, cudaStream_t st);
// the index-check record of the debug build (count -1 without checks); a cudaError_t or 0
int bounds_record(long long* out3);

}  // namespace sns

struct sns_handle;

namespace sns {

// Handle hooks for the batch and serving layers (defined in sns_api.cu).
void enqueue_step(sns_handle* h, double dt);  // one RK3 step on the handle's stream, no sync
void enqueue_clock_step(sns_handle* h);       // one adaptive-CFL step on the device clock, no sync
double* handle_clock(sns_handle* h);
cudaStream_t handle_stream(const sns_handle* h);
int handle_device(const sns_handle* h);
int finish_handle(sns_handle* h, const char* what);  // sync + device error word -> SNS code
const char* handle_error(const sns_handle* h);
bool set_launch_shape(sns_handle* h, const int* cfg);  // {tma_grid, x2_grid, p5_grid}
void set_handle_error(sns_handle* h, const char* msg);
// the handle back in its creation state for a new solve (same N and precision), no allocation
int reset_handle(sns_handle* h, double nu, uint64_t seed, double pert_amp, int pert_kmax);

// Host helpers shared by the C-ABI files (sns_api.cu).
void fill_twiddles(int L, double2* tw);        // exp(-2*pi*i*t/L), t < L
void set_handleless_error(const char* msg);    // message for sns_last_error(NULL)

constexpr int kXDiagPartials = 2;   // (sum 0.5|u|^2, max |u|^2) per row
constexpr int kSpecDiagPartials = 2;  // (sum w*|H(omega)|^2, max |k.u|) per block

}  // namespace sns
