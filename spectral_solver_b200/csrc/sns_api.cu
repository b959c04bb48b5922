// C ABI of the B200 Taylor-Green solver: handle, device memory, tables, step orchestration.
//
// Device memory of a handle, in half fields of N*N*pitch complex values (double2 in the FP64
// plain form, float2 in the FP32 precision form):
//   state : u[3], g[3]            (the reference's u_hat and g, ava_taylor_green_impl.hpp:665-667)
//   work  : 12 fields             (inverse-transformed velocity on both grids, then the
//                                  12 product spectra; the fused x pass reads 6 and writes
//                                  12 rows in place, so one buffer serves both)
//   tables: twiddles (N), phase exp(i*pi*(mx+my+mz)/N) for mx+my+mz in [-3N/2, 3N/2],
//           reduction partials, the 12 Nyquist-plane sums.
#include "sns_kernels.cuh"
#include "../../include/sns_b200.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <exception>
#include <new>
#include <string>
#include <vector>

namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;

struct SnsError : std::exception {
  int code;
  std::string msg;
  SnsError(int c, std::string m) : code(c), msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

void ck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw SnsError(SNS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

thread_local std::string g_create_error;

}  // namespace

namespace sns {

// exp(-2*pi*i*t/L) for t < L, rounded from long double; exact at the quarter points.
void fill_twiddles(int L, double2* tw) {
  for (int t = 0; t < L; ++t) {
    const int q = (4 * t) % (4 * L);
    if (q % L == 0) {
      const int k = q / L;  // t*4/L in {0,1,2,3}
      const double c[4] = {1.0, 0.0, -1.0, 0.0};
      const double s[4] = {0.0, -1.0, 0.0, 1.0};
      tw[t] = make_double2(c[k], s[k]);
    } else {
      const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)t / (long double)L;
      tw[t] = make_double2((double)cosl(a), (double)sinl(a));
    }
  }
}

// Message slot that sns_last_error(NULL) reads: failures of calls made without a handle.
void set_handleless_error(const char* msg) { g_create_error = msg; }

}  // namespace sns

struct sns_handle {
  int n = 0;
  int device = 0;
  double nu = 0.0;
  int precision = 0;
  int viscous_mode = 0;
  sns::Geom g{};
  const sns::Ops* ops = nullptr;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int cbytes = 16;          // bytes per complex value: 16 (FP64) or 8 (FP32)
  size_t fbytes = 0;        // bytes per half field
  char* state = nullptr;    // u[3] then g[3]
  char* work = nullptr;     // 12 fields
  void* tw = nullptr;
  void* phase = nullptr;
  double* partials = nullptr;
  double* red = nullptr;  // reduction results
  int* err_word = nullptr;  // device error word written by bounded waits
  double* clock = nullptr;  // device clock of adaptive-CFL stepping (sns::kClock* slots)
  bool on_clock = false;    // the stages being enqueued take their step from the clock
  int tma_grid = 0;         // persistent CTAs of the TMA passes
  int x2_grid = 0;          // persistent CTAs of the two-stage x pass (0: generic x pass)
  int p5_grid = 0;          // persistent CTAs of the fused forward-z + sweep pass (0: two kernels)
  void* tw2 = nullptr;      // W_N^(r*j), r < N/16, j < 16 (two-stage x pass)
  double* nyq_part = nullptr;  // [12][max(1, x2_grid)] Nyquist-plane partial sums
  CUtensorMap map_state_z{};  // state fields (u[3], g[3]), z-pencil boxes
  CUtensorMap map_work_y{};   // 12 work fields, y-pencil boxes
  CUtensorMap map_work_z{};   // 12 work fields, z-pencil boxes
  int form = 0;               // nonlinear form: 0 conservative (the reference), 1 rotational
  char* xf = nullptr;         // rotational form: omega_hat (3 fields), allocated on first use
  CUtensorMap map_x_z{};      // the omega_hat fields, z-pencil boxes
  size_t partial_count = 0;
  size_t bytes = 0;
  int fail_after = 0;
  // true when the state's mx = N/2 plane is zero off (N/2,0,0), as every masked state is;
  // then the passes skip that column and take the Nyquist mode from the state directly
  bool nyq_clean = true;
  // Sphere pruning.  live: the (my * ncb + cb) column-block tiles of the z pencils with a mode
  // inside the sphere |k| <= N/2 (4 ((cb * TW)^2 + my^2) <= N^2, ncb = tiles_data()); the
  // others hold only modes that every RK stage zeroes.  sphere_clean: u is known to be exactly
  // zero outside the sphere (after creation and after any RK stage that ran, not one only
  // captured into a graph; false after the state is set).
  int* live = nullptr;
  int nlive = 0;
  bool sphere_clean = false;
  bool prune = true;  // sns_set_sphere_pruning
  // FP32 precision form: compensation words of u (3 fields of one 16-bit word per complex
  // value, the index of u), so the RK update keeps the low bits the FP32 state drops;
  // comp: in use (sns_set_compensation)
  sns::CompWord* ulo = nullptr;
  bool comp = false;
  std::string err;

  char* u() const { return state; }
  char* gb() const { return state + 3 * fbytes; }
  char* ucomp(int c) const { return state + (size_t)c * fbytes; }
  sns::CompWord* locomp(int c) const { return comp ? ulo + (size_t)c * g.field : nullptr; }
  char* wf(int i) const { return work + (size_t)i * fbytes; }
  int tcols() const { return ops->tile_cols; }
  int tiles_data() const { return (g.nh + tcols() - 1) / tcols(); }  // columns [0, N/2)
  int tiles_all() const { return g.pitch / tcols(); }                // Nyquist column included
  double inv_size() const { return 1.0 / ((double)n * n * n); }
};

namespace {

int complex_bytes(int precision) { return precision == SNS_PRECISION_FP32 ? 8 : 16; }
size_t field_bytes(int n, int precision) {
  const int cb = complex_bytes(precision);
  return (size_t)n * n * sns::pitch_for(n, cb) * cb;
}

// Device copy of a complex table given in FP64: as is, or rounded to FP32.
void upload_table(void* dst, const std::vector<double2>& t, int precision, cudaStream_t st) {
  if (precision == SNS_PRECISION_FP32) {
    std::vector<float2> f(t.size());
    for (size_t i = 0; i < t.size(); ++i) f[i] = make_float2((float)t[i].x, (float)t[i].y);
    ck(cudaMemcpyAsync(dst, f.data(), f.size() * sizeof(float2), cudaMemcpyHostToDevice, st), "table upload");
    ck(cudaStreamSynchronize(st), "table upload");
  } else {
    ck(cudaMemcpyAsync(dst, t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, st), "table upload");
    ck(cudaStreamSynchronize(st), "table upload");
  }
}

// Bytes of the compensation words of u (FP32 form): 3 fields of 2 bytes per complex value.
size_t comp_bytes(int n, int precision) {
  if (precision != SNS_PRECISION_FP32) return 0;
  return (size_t)3 * n * n * sns::pitch_for(n, 8) * sizeof(sns::CompWord);
}

size_t partial_slots(int n) {
  const size_t rows = (size_t)n * n;
  return 2 * rows + 4096;
}

std::vector<double2> twiddle_table(int L) {
  std::vector<double2> tw(L);
  sns::fill_twiddles(L, tw.data());
  return tw;
}

// Phase table computed exactly as the reference does on the host
// (initialize_metadata, ava_taylor_green_impl.hpp:782-783): angle = (msum * pi) / n.
std::vector<double2> phase_table(int n) {
  std::vector<double2> ph(3 * n + 1);
  for (int i = 0; i <= 3 * n; ++i) {
    const int msum = i - 3 * n / 2;
    const double angle = (static_cast<double>(msum) * kPi) / static_cast<double>(n);
    ph[i] = make_double2(std::cos(angle), std::sin(angle));
  }
  return ph;
}

uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}


// Seeded solenoidal k^(-5/3) perturbation (the project's own specification; the reference
// starts from the pure Taylor-Green field).  Returns sparse (index, value) entries in the
// half layout of the 3 consecutive state fields.
void perturbation_entries(int n, uint64_t seed, double amp, int kmax, const sns::Geom& g,
                          std::vector<long long>& idx, std::vector<double2>& val) {
  idx.clear();
  val.clear();
  if (amp == 0.0 || kmax < 1) return;
  if (2 * kmax >= n) throw SnsError(SNS_ERR_INVALID, "perturbation kmax must be below N/2");
  struct Mode { int mx, my, mz; double v[6]; };
  std::vector<Mode> modes;
  const uint64_t h = splitmix64(seed);
  double total = 0.0;
  for (int mz = -kmax; mz <= kmax; ++mz)
    for (int my = -kmax; my <= kmax; ++my)
      for (int mx = 0; mx <= kmax; ++mx) {
        const int k2 = mx * mx + my * my + mz * mz;
        if (k2 < 1 || k2 > kmax * kmax) continue;
        const bool canon = mx > 0 || my > 0 || (my == 0 && mz > 0);
        if (!canon) continue;
        const uint64_t flat = (uint64_t)mx + (uint64_t)n * ((uint64_t)((my % n + n) % n) +
                                                            (uint64_t)n * (uint64_t)((mz % n + n) % n));
        const double kk = (double)k2;
        const double a = std::pow(std::sqrt(kk), -5.0 / 3.0);
        double re[3], im[3];
        for (int c = 0; c < 3; ++c) {
          const uint64_t r = splitmix64(h ^ (3ULL * flat + (uint64_t)c));
          const double theta = (double)(r >> 11) * (1.0 / 9007199254740992.0);
          const double ang = 2.0 * kPi * theta;
          re[c] = a * std::cos(ang);
          im[c] = a * std::sin(ang);
        }
        const double fx = mx, fy = my, fz = mz;
        const double dre = (re[0] * fx + re[1] * fy) + re[2] * fz;
        const double dim = (im[0] * fx + im[1] * fy) + im[2] * fz;
        const double kv[3] = {fx, fy, fz};
        Mode m{mx, my, mz, {}};
        for (int c = 0; c < 3; ++c) {
          m.v[2 * c] = re[c] - (dre / kk) * kv[c];
          m.v[2 * c + 1] = im[c] - (dim / kk) * kv[c];
          total += 2.0 * (m.v[2 * c] * m.v[2 * c] + m.v[2 * c + 1] * m.v[2 * c + 1]);
        }
        modes.push_back(m);
      }
  const double n6 = std::pow((double)n, 6.0);
  const double s = amp / std::sqrt(total / n6);
  for (const Mode& m : modes) {
    const long long row = (long long)((m.mz % n + n) % n) * n + ((m.my % n + n) % n);
    for (int c = 0; c < 3; ++c) {
      idx.push_back((long long)c * g.field + row * g.pitch + m.mx);
      val.push_back(make_double2(m.v[2 * c] * s, m.v[2 * c + 1] * s));
      if (m.mx == 0) {
        const long long rowm = (long long)(((-m.mz) % n + n) % n) * n + (((-m.my) % n + n) % n);
        idx.push_back((long long)c * g.field + rowm * g.pitch);
        val.push_back(make_double2(m.v[2 * c] * s, -m.v[2 * c + 1] * s));
      }
    }
  }
}

using EncodeTiled = PFN_cuTensorMapEncodeTiled_v12000;

EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  if (fn == nullptr) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    ck(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q), "cudaGetDriverEntryPoint");
    if (q != cudaDriverEntryPointSuccess || p == nullptr)
      throw SnsError(SNS_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
    fn = reinterpret_cast<EncodeTiled>(p);
  }
  return fn;
}

// Tensor map over `nf` consecutive half fields viewed as [field][z][y][2*pitch reals],
// box = 128 bytes (16 doubles = 8 complex, or 32 floats = 16 complex) x up to 256 rows
// along y (axis 1) or z (axis 2).
CUtensorMap make_field_map(void* base, int nf, int axis, const sns::Geom& g, int cbytes) {
  CUtensorMap m;
  const cuuint64_t row = (cuuint64_t)g.pitch * cbytes;
  cuuint64_t dims[4] = {(cuuint64_t)2 * g.pitch, (cuuint64_t)g.n, (cuuint64_t)g.n, (cuuint64_t)nf};
  cuuint64_t strides[3] = {row, row * g.n, (cuuint64_t)g.field * cbytes};
  const cuuint32_t br = g.n < 256 ? (cuuint32_t)g.n : 256u;
  cuuint32_t box[4] = {(cuuint32_t)(256 / cbytes), axis == 1 ? br : 1u, axis == 2 ? br : 1u, 1u};
  cuuint32_t es[4] = {1u, 1u, 1u, 1u};
  const CUtensorMapDataType dt = cbytes == 16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const CUresult r = encode_fn()(&m, dt, 4, base, dims, strides, box, es,
                                 CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw SnsError(SNS_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
  return m;
}

sns::TmaArgs tma_args(sns_handle* h, int f_in0, int nf, int ncb, void* out, int f_out0, double scale) {
  sns::TmaArgs a{};
  a.f_in0 = f_in0;
  a.nf = nf;
  a.ncb = ncb;
  a.out = out;
  a.f_out0 = f_out0;
  a.scale = scale;
  a.err = h->err_word;
  return a;
}

void check_inject(sns_handle* h) {
  if (h->fail_after > 0) {
    if (--h->fail_after == 0) throw SnsError(SNS_ERR_INJECTED, "failure injected by sns_debug_fail_after");
  }
}

void sync(sns_handle* h, const char* what) {
  ck(cudaGetLastError(), what);
  ck(cudaStreamSynchronize(h->stream), what);
  int e = 0;
  ck(cudaMemcpy(&e, h->err_word, sizeof(int), cudaMemcpyDeviceToHost), what);
  if (e != 0) {
    cudaMemset(h->err_word, 0, sizeof(int));
    throw SnsError(SNS_ERR_CUDA, std::string(what) + ": a pass gave up waiting for its TMA tile (code " +
                                     std::to_string(e) + ")");
  }
}

// Optional per-pass event marks (profiling entry point only).
struct PassMarks {
  cudaEvent_t ev[8];
  bool on = false;
};

inline void mark(PassMarks* pm, int i, cudaStream_t st) {
  if (pm && pm->on) cudaEventRecord(pm->ev[i], st);
}

// Is `st` being captured into a graph (launches recorded now, run later)?
bool capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  return cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone;
}

sns::SweepArgs stage_args(const sns_handle* h, int stage, double dt, int mode, const char* u_src) {
  sns::SweepArgs a{};
  a.nu = h->nu;
  // the compensated update applies to the handle's own state only (not to sns_rhs inputs)
  a.ulo = (h->comp && mode == 0 && u_src == h->u()) ? h->ulo : nullptr;
  // adaptive stepping: the step size comes from the device clock
  a.clock = (h->on_clock && mode == 0) ? h->clock : nullptr;
  a.stage = stage;
  a.mode = mode;
  a.dealias = 1;
  // integrating-factor mode: after stage s, u and g advance from c_s*dt to c_{s+1}*dt with
  // the stage times c = (0, 1/3, 3/4, 1) of the Williamson scheme
  a.visc_if = h->viscous_mode == SNS_VISCOUS_INTEGRATING_FACTOR ? 1 : 0;
  a.if_tau = stage == 0 ? dt / 3.0 : (stage == 1 ? 5.0 * dt / 12.0 : dt / 4.0);
  if (stage == 0) {
    a.ga = 0.0;
    a.ub = dt / 3.0;
  } else if (stage == 1) {
    a.ga = -5.0 / 9.0;
    a.ub = 15.0 * dt / 16.0;
  } else {
    a.ga = -153.0 / 128.0;
    a.ub = 8.0 * dt / 15.0;
  }
  return a;
}

// One stage in the rotational form: omega_hat, inverse z (+ phase) of u and omega, inverse y
// of the 12 fields, the u x omega x pass, forward y and z of the 6 products, the sweep.
void run_stage_rot(sns_handle* h, char* u_src, char* g_buf, int stage, double dt, int mode, char* rhs_out,
                   PassMarks* pm) {
  const sns::Ops* o = h->ops;
  const sns::Geom& g = h->g;
  cudaStream_t st = h->stream;
  const int tiles_in = h->nyq_clean ? h->tiles_data() : h->tiles_all();
  const int f_src = (int)((size_t)(u_src - h->state) / h->fbytes);
  mark(pm, 0, st);
  o->omega_hat(u_src, h->xf, g, st);
  o->yz_tma(h->map_state_z, 2, +1, 1, tma_args(h, f_src, 3, tiles_in, h->work, 0, h->inv_size()), h->tw, h->phase, g,
            h->tma_grid, st);
  o->yz_tma(h->map_x_z, 2, +1, 1, tma_args(h, 0, 3, tiles_in, h->work, 6, h->inv_size()), h->tw, h->phase, g,
            h->tma_grid, st);
  mark(pm, 1, st);
  o->yz_tma(h->map_work_y, 1, +1, 0, tma_args(h, 0, 12, tiles_in, h->work, 0, 1.0), h->tw, h->phase, g, h->tma_grid,
            st);
  mark(pm, 2, st);
  o->xpass_rot(h->work, u_src, h->xf, h->phase, h->inv_size(), h->nyq_clean ? 1 : 0, h->tw, g, st);
  mark(pm, 3, st);
  o->nyq_reduce(h->work, h->nyq_part, g, st);  // the first 6 sums are the products'
  mark(pm, 4, st);
  o->yz_tma(h->map_work_y, 1, -1, 0, tma_args(h, 0, 6, h->tiles_data(), h->work, 0, 1.0), h->tw, h->phase, g,
            h->tma_grid, st);
  mark(pm, 5, st);
  o->yz_tma(h->map_work_z, 2, -1, 0, tma_args(h, 0, 6, h->tiles_data(), h->work, 0, 1.0), h->tw, h->phase, g,
            h->tma_grid, st);
  mark(pm, 6, st);
  o->sweep_rot(h->work, u_src, g_buf, rhs_out, h->nyq_part, h->phase, stage_args(h, stage, dt, mode, u_src), g, st);
  mark(pm, 7, st);
}

// One RK3 stage (or the RHS only, mode 1) on u_src: the five fused passes.
void run_stage(sns_handle* h, char* u_src, char* g_buf, int stage, double dt, int mode, char* rhs_out,
               double* partials, PassMarks* pm = nullptr) {
  if (h->form == 1) {
    run_stage_rot(h, u_src, g_buf, stage, dt, mode, rhs_out, pm);
    return;
  }
  const sns::Ops* o = h->ops;
  const sns::Geom& g = h->g;
  cudaStream_t st = h->stream;
  const int tiles_in = h->nyq_clean ? h->tiles_data() : h->tiles_all();
  const int f_src = (int)((size_t)(u_src - h->state) / h->fbytes);  // u (0) or the g slot (3)
  const bool fused = h->p5_grid > 0;
  // Sphere pruning (RK update with the fused P5 only).  A column-block tile (my, cb) outside
  // the disk 4 ((cb * TW)^2 + my^2) <= N^2 holds only modes outside the sphere: u is zero
  // there before the stage (every stage's sweep zeroes those modes, so stages 1 and 2 may
  // rely on stage 0; stage 0 relies on the handle's flag, and never inside a graph capture,
  // where the graph may later be replayed on a new state) and the stage leaves it zero.  So
  // P5 neither loads, transforms nor sweeps these tiles (their forward-z inputs are never
  // needed); every other value is computed as without pruning.
  const bool prune = h->prune && fused && mode == 0 && h->nyq_clean && h->nlive > 0 &&
                     (stage > 0 || (h->sphere_clean && !capturing(st)));
  mark(pm, 0, st);
  o->yz_tma(h->map_state_z, 2, +1, 1, tma_args(h, f_src, 3, tiles_in, h->work, 0, h->inv_size()), h->tw, h->phase,
            g, h->tma_grid, st);
  mark(pm, 1, st);
  o->yz_tma(h->map_work_y, 1, +1, 0, tma_args(h, 0, 6, tiles_in, h->work, 0, 1.0), h->tw, h->phase, g, h->tma_grid,
            st);
  mark(pm, 2, st);
  int nparts = 1;
  if (h->x2_grid > 0 && partials == nullptr) {
    o->xpass2(h->work, u_src, h->phase, h->inv_size(), h->nyq_clean ? 1 : 0, h->nyq_part, h->tw2, g, h->x2_grid,
              h->err_word, st);
    nparts = h->x2_grid;
    mark(pm, 3, st);
  } else {
    o->xpass_products(h->work, u_src, h->phase, h->inv_size(), h->nyq_clean ? 1 : 0, partials, h->tw, g, st);
    mark(pm, 3, st);
    o->nyq_reduce(h->work, h->nyq_part, g, st);
  }
  mark(pm, 4, st);
  o->yz_tma(h->map_work_y, 1, -1, 0, tma_args(h, 0, 12, h->tiles_data(), h->work, 0, 1.0), h->tw, h->phase, g,
            h->tma_grid, st);
  mark(pm, 5, st);
  if (!fused)
    o->yz_tma(h->map_work_z, 2, -1, 0, tma_args(h, 0, 12, h->tiles_data(), h->work, 0, 1.0), h->tw, h->phase, g,
              h->tma_grid, st);
  mark(pm, 6, st);
  const sns::SweepArgs a = stage_args(h, stage, dt, mode, u_src);
  if (fused)
    o->p5(h->map_work_z, u_src, g_buf, rhs_out, h->nyq_part, nparts, h->tw, h->phase, a, h->tiles_data(),
          prune ? h->live : nullptr, prune ? h->nlive : 0, g, h->p5_grid, h->err_word, st);
  else
    o->sweep(h->work, u_src, g_buf, rhs_out, h->nyq_part, nparts, h->phase, a, g, st);
  mark(pm, 7, st);
}

void step_once(sns_handle* h, double dt) {
  const bool deferred = capturing(h->stream);  // a captured graph runs later, on whatever state
  for (int s = 0; s < 3; ++s) {
    run_stage(h, h->u(), h->gb(), s, dt, 0, nullptr, nullptr);
    h->nyq_clean = true;  // the sweep zeroes the plane mx = N/2 off (N/2,0,0)
    // and every mode outside the sphere, once the stage has run
    if (!deferred) h->sphere_clean = true;
  }
}

int velocity_partials(sns_handle* h);

// One step with the adaptive CFL rule on the device: vmax of the current state (the same
// per-row partials as sns_max_velocity; their max and the clock's next step in one launch),
// then the three stages on that step.  Nothing here waits for the host, so the step can be
// captured into a graph.
void step_on_clock(sns_handle* h) {
  const int pairs = velocity_partials(h);
  sns::launch_clock_step_partials(h->partials + 1, pairs, 2, h->clock, h->stream);
  h->on_clock = true;
  try {
    step_once(h, 0.0);
  } catch (...) {
    h->on_clock = false;
    throw;
  }
  h->on_clock = false;
}

// Does a reference full-layout spectrum carry content on the plane mx = N/2 off (N/2,0,0)?
bool nyquist_plane_dirty(int n, const double* full) {
  const int nh = n / 2;
  for (long long z = 0; z < n; ++z)
    for (long long y = 0; y < n; ++y) {
      if (y == 0 && z == 0) continue;
      const double* v = full + 2 * ((z * n + y) * n + nh);
      if (v[0] != 0.0 || v[1] != 0.0) return true;
    }
  return false;
}

// Upload a reference full-layout field into half field `dst` (optionally Hermitian part).
// The N^3 complex doubles of a full-layout field fit in work fields 4..11 for either precision.
// With `lo` (FP32 form, compensated state) the remainder the FP32 value drops goes there.
// The plain conversion reads columns 0..N/2 of each row only, so only those cross the bus (one
// pitched copy, half the bytes); the Hermitian part needs the mirror columns too.
void upload_full(sns_handle* h, const double* host, void* dst, int herm, sns::CompWord* lo = nullptr) {
  double2* staging = reinterpret_cast<double2*>(h->wf(4));
  const size_t n = (size_t)h->n;
  if (herm) {
    ck(cudaMemcpyAsync(staging, host, n * n * n * sizeof(double2), cudaMemcpyHostToDevice, h->stream), "upload");
    sns::launch_full_to_half(staging, dst, h->precision, herm, h->g, h->stream, lo);
  } else {
    const size_t w = (n / 2 + 1) * sizeof(double2);
    ck(cudaMemcpy2DAsync(staging, w, host, n * sizeof(double2), w, n * n, cudaMemcpyHostToDevice, h->stream),
       "upload");
    sns::launch_full_to_half(staging, dst, h->precision, 0, h->g, h->stream, lo, (long long)(n / 2 + 1));
  }
}

void download_full(sns_handle* h, const void* src, double* host, const sns::CompWord* lo = nullptr) {
  double2* staging = reinterpret_cast<double2*>(h->wf(4));
  const size_t bytes = (size_t)h->n * h->n * h->n * sizeof(double2);
  sns::launch_half_to_full(src, h->precision, staging, h->g, h->stream, lo);
  ck(cudaMemcpyAsync(host, staging, bytes, cudaMemcpyDeviceToHost, h->stream), "download");
}

// Physical velocity of the state: inverse z and y passes of u without the phase shift, then
// the diagnostic x pass; (energy, vmax^2) partials in h->partials, per row or per CTA of the
// warp-per-row kernel; returns how many pairs.
int velocity_partials(sns_handle* h) {
  const sns::Ops* o = h->ops;
  const sns::Geom& g = h->g;
  const int tiles = h->nyq_clean ? h->tiles_data() : h->tiles_all();
  o->yz_tma(h->map_state_z, 2, +1, 0, tma_args(h, 0, 3, tiles, h->work, 0, h->inv_size()), h->tw, h->phase, g,
            h->tma_grid, h->stream);
  o->yz_tma(h->map_work_y, 1, +1, 0, tma_args(h, 0, 3, tiles, h->work, 0, 1.0), h->tw, h->phase, g, h->tma_grid,
            h->stream);
  return o->xpass_diag2(h->work, h->u(), h->inv_size(), h->nyq_clean ? 1 : 0, h->partials, h->tw, h->tw2, g,
                        h->x2_grid, h->err_word, h->stream);
}

// The same reduced: energy sum in h->red[0], vmax^2 in h->red[1].
void velocity_reductions(sns_handle* h) {
  const int rows = velocity_partials(h);  // (energy, vmax^2) pairs
  sns::launch_reduce(h->partials, rows, 2, 0, h->red + 0, h->stream);
  sns::launch_reduce(h->partials + 1, rows, 2, 1, h->red + 1, h->stream);
}

// The initial state on the handle's own memory: Taylor-Green at cell centres -> forward
// transform -> + seeded perturbation -> project_truncate; g, the work fields and the FP32
// form's compensation words zeroed.  Allocates nothing (sns_create and the server's reuse of
// a retired handle both run it).
void initial_field(sns_handle* h, uint64_t seed, double pert_amp, int pert_kmax) {
  const sns::Ops* ops = h->ops;
  const size_t fb = h->fbytes;
  ck(cudaMemsetAsync(h->state, 0, 6 * fb, h->stream), "memset");
  ck(cudaMemsetAsync(h->work, 0, 12 * fb, h->stream), "memset");
  if (h->ulo) ck(cudaMemsetAsync(h->ulo, 0, comp_bytes(h->n, h->precision), h->stream), "memset");
  double* phys = reinterpret_cast<double*>(h->wf(6));
  sns::launch_tgv_init(phys, h->g, h->stream);
  ops->xpass_r2c(phys, h->u(), 2, h->tw, h->g, h->stream);  // w = 0: its spectrum stays zero
  ops->ypass(h->u(), 2, -1, h->tiles_all(), h->tw, h->g, h->stream);
  ops->zpass(h->u(), h->u(), 2, -1, h->tiles_all(), 1.0, h->tw, h->g, h->stream);
  std::vector<long long> idx;
  std::vector<double2> val;
  perturbation_entries(h->n, seed, pert_amp, pert_kmax, h->g, idx, val);
  if (!idx.empty()) {
    long long* d_idx = reinterpret_cast<long long*>(h->wf(8));
    double2* d_val = reinterpret_cast<double2*>(h->wf(9));
    ck(cudaMemcpyAsync(d_idx, idx.data(), idx.size() * sizeof(long long), cudaMemcpyHostToDevice, h->stream), "p");
    ck(cudaMemcpyAsync(d_val, val.data(), val.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream), "p");
    sns::launch_add_sparse(h->u(), h->precision, d_idx, d_val, (int)idx.size(), h->stream);
    ck(cudaStreamSynchronize(h->stream), "perturbation");
  }
  sns::launch_project_truncate(h->u(), h->precision, h->g, h->stream);
  ck(cudaMemsetAsync(h->work, 0, 12 * fb, h->stream), "memset");
  h->nyq_clean = true;
  h->sphere_clean = true;  // project_truncate zeroed every mode outside the sphere
}

template <class F>
int guarded(sns_handle* h, F&& f) {
  if (h == nullptr) return SNS_ERR_INVALID;
  try {
    check_inject(h);
    ck(cudaSetDevice(h->device), "cudaSetDevice");
    f();
    h->err.clear();
    return SNS_OK;
  } catch (const SnsError& e) {
    h->err = e.msg;
    return e.code;
  } catch (const std::bad_alloc&) {
    h->err = "host allocation failed";
    return SNS_ERR_NOMEM;
  } catch (const std::exception& e) {
    h->err = e.what();
    return SNS_ERR_INVALID;
  }
}

void release(sns_handle* h) {
  if (h == nullptr) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  cudaFree(h->state);
  cudaFree(h->work);
  cudaFree(h->tw);
  cudaFree(h->phase);
  cudaFree(h->partials);
  cudaFree(h->red);
  cudaFree(h->err_word);
  cudaFree(h->clock);
  cudaFree(h->tw2);
  cudaFree(h->nyq_part);
  cudaFree(h->xf);
  cudaFree(h->live);
  cudaFree(h->ulo);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

}  // namespace

namespace sns {

// Hooks for the batch and serving layers in this library (not part of the C ABI).
void enqueue_step(sns_handle* h, double dt) { step_once(h, dt); }
void enqueue_clock_step(sns_handle* h) { step_on_clock(h); }
double* handle_clock(sns_handle* h) { return h->clock; }
cudaStream_t handle_stream(const sns_handle* h) { return h->stream; }
int handle_device(const sns_handle* h) { return h->device; }
// Synchronise the handle's stream and check its device error word; SNS code, message in h.
int finish_handle(sns_handle* h, const char* what) {
  try {
    sync(h, what);
    return SNS_OK;
  } catch (const SnsError& e) {
    h->err = e.msg;
    return e.code;
  }
}
const char* handle_error(const sns_handle* h) { return h->err.c_str(); }
// Persistent grid of the TMA passes for a small grid (N <= 128): at most max(16, 2N) CTAs.
// Such solves run many at a time (ensembles, the server), and a pass whose grid covers every
// SM for a few microseconds of work leaves no room for the other solves' passes; with 2N
// CTAs the 64-solve ensemble (N = 32..128) steps 11 % faster in FP32, 4 % in FP64.  A lone
// small solve tuned by sns_autotune keeps the tuned grid.
int small_grid_cap(int n, int grid) { return n <= 128 ? std::min(grid, std::max(16, 2 * n)) : grid; }

// Launch shape {tma_grid, x2_grid, p5_grid} as sns_autotune reports it; false if the handle
// cannot run it (its Nyquist partial buffer is sized for its own two-stage x-pass grid).
bool set_launch_shape(sns_handle* h, const int* cfg) {
  int nsm = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess) return false;
  const int x2_full = h->ops->xpass2_grid(nsm), p5_full = h->ops->p5_grid(nsm);
  const int tma_max = h->ops->tma_blocks_per_sm();
  if (cfg[0] < nsm || cfg[0] > nsm * tma_max || (cfg[1] != 0 && cfg[1] != x2_full) ||
      (cfg[2] != 0 && cfg[2] != p5_full))
    return false;
  h->tma_grid = small_grid_cap(h->n, cfg[0]);
  h->x2_grid = cfg[1];
  h->p5_grid = cfg[2];
  return true;
}
void set_handle_error(sns_handle* h, const char* msg) { h->err = msg; }
// A handle returned to its creation state for a new solve of the same N and precision
// (viscosity, seed and perturbation of the new solve), on its own memory: no allocation.
int reset_handle(sns_handle* h, double nu, uint64_t seed, double pert_amp, int pert_kmax) {
  return guarded(h, [&] {
    if (!(nu >= 0.0) || !std::isfinite(nu)) throw SnsError(SNS_ERR_INVALID, "viscosity must be finite and >= 0");
    if (!(pert_amp >= 0.0) || (pert_amp > 0.0 && 2 * pert_kmax >= h->n))
      throw SnsError(SNS_ERR_INVALID, "perturbation amplitude must be >= 0 and kmax below N/2");
    h->nu = nu;
    h->form = 0;
    h->prune = true;
    h->comp = h->ulo != nullptr;
    initial_field(h, seed, pert_amp, pert_kmax);
    sync(h, "reset");
  });
}

}  // namespace sns

extern "C" {

const char* sns_version(void) { return "sns_b200 0.2 (sm_100a, fp64 plain form, fp32 precision form)"; }

int sns_grid_supported(int n) { return n > 0 && sns::ops_for(n, 0) != nullptr ? 1 : 0; }

size_t sns_bytes_required(int n, int precision) {
  if (n <= 0 || (precision != SNS_PRECISION_FP64 && precision != SNS_PRECISION_FP32)) return 0;
  return 18 * field_bytes(n, precision) + comp_bytes(n, precision) + partial_slots(n) * sizeof(double) +
         (size_t)(4 * n + 64) * complex_bytes(precision) + (size_t)n * (n / 16 + 1) * sizeof(int) +
         sns::kClockWords * sizeof(double);
}

int sns_create(int n, double nu, int precision, int viscous_mode, uint64_t seed, double pert_amp, int pert_kmax,
               sns_handle** out) {
  g_create_error.clear();
  if (out == nullptr) {
    g_create_error = "null output pointer";
    return SNS_ERR_INVALID;
  }
  *out = nullptr;
  if (n <= 0) {
    g_create_error = "grid size must be positive";
    return SNS_ERR_INVALID;
  }
  if (!(nu >= 0.0) || !std::isfinite(nu)) {
    g_create_error = "viscosity must be finite and non-negative (Reynolds number must be positive)";
    return SNS_ERR_INVALID;
  }
  if (precision != SNS_PRECISION_FP64 && precision != SNS_PRECISION_FP32) {
    g_create_error = "precision must be SNS_PRECISION_FP64 (0) or SNS_PRECISION_FP32 (1)";
    return SNS_ERR_UNSUPPORTED;
  }
  if (viscous_mode != SNS_VISCOUS_EXPLICIT && viscous_mode != SNS_VISCOUS_INTEGRATING_FACTOR) {
    g_create_error = "viscous mode must be SNS_VISCOUS_EXPLICIT (0) or SNS_VISCOUS_INTEGRATING_FACTOR (1)";
    return SNS_ERR_UNSUPPORTED;
  }
  const sns::Ops* ops = sns::ops_for(n, precision);
  if (ops == nullptr) {
    g_create_error = "grid size " + std::to_string(n) + " has no FFT plan (supported: 8 12 16 24 32 48 64 96 128 256 512)";
    return SNS_ERR_UNSUPPORTED;
  }
  if (!(pert_amp >= 0.0) || (pert_amp > 0.0 && 2 * pert_kmax >= n)) {
    g_create_error = "perturbation amplitude must be >= 0 and kmax below N/2";
    return SNS_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    g_create_error = "no CUDA device visible";
    return SNS_ERR_NO_DEVICE;
  }
  sns_handle* h = new (std::nothrow) sns_handle();
  if (h == nullptr) {
    g_create_error = "host allocation failed";
    return SNS_ERR_NOMEM;
  }
  try {
    ck(cudaGetDevice(&h->device), "cudaGetDevice");
    h->n = n;
    h->nu = nu;
    h->precision = precision;
    h->viscous_mode = viscous_mode;
    h->ops = ops;
    h->cbytes = complex_bytes(precision);
    const int pitch = sns::pitch_for(n, h->cbytes);
    h->g = sns::Geom{n, n / 2, pitch, (long long)n * n * pitch};
    h->fbytes = field_bytes(n, precision);
    const size_t need = sns_bytes_required(n, precision);
    size_t free_b = 0, total_b = 0;
    ck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    if (need > free_b) throw SnsError(SNS_ERR_NOMEM, "grid needs " + std::to_string(need) + " bytes, device has " +
                                                         std::to_string(free_b) + " free");
    ops->init();
    ck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    ck(cudaEventCreate(&h->ev0), "cudaEventCreate");
    ck(cudaEventCreate(&h->ev1), "cudaEventCreate");
    const size_t fb = h->fbytes;
    h->partial_count = partial_slots(n);
    auto alloc = [&](void** p, size_t bytes) {
      cudaError_t e = cudaMalloc(p, bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        throw SnsError(SNS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
      }
      h->bytes += bytes;
    };
    alloc((void**)&h->state, 6 * fb);
    alloc((void**)&h->work, 12 * fb);
    alloc((void**)&h->tw, (size_t)n * h->cbytes);
    alloc((void**)&h->phase, (size_t)(3 * n + 1) * h->cbytes);
    alloc((void**)&h->partials, h->partial_count * sizeof(double));
    alloc((void**)&h->red, 16 * sizeof(double));
    alloc((void**)&h->err_word, sizeof(int));
    alloc((void**)&h->clock, sns::kClockWords * sizeof(double));
    ck(cudaMemsetAsync(h->clock, 0, sns::kClockWords * sizeof(double), h->stream), "memset");
    ck(cudaMemsetAsync(h->err_word, 0, sizeof(int), h->stream), "memset");
    int nsm = 0;
    ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device), "cudaDeviceGetAttribute");
    h->tma_grid = sns::small_grid_cap(n, nsm * ops->tma_blocks_per_sm());
    h->x2_grid = ops->xpass2_grid(nsm);
    h->p5_grid = ops->p5_grid(nsm);
    alloc((void**)&h->nyq_part, (size_t)12 * (h->x2_grid > 0 ? h->x2_grid : 1) * sizeof(double));
    alloc((void**)&h->tw2, (size_t)n * h->cbytes);
    {
      // tw2[r*16 + j] = exp(-2*pi*i*r*j/n) for r < n/16, j < 16
      const auto tw = twiddle_table(n);
      std::vector<double2> t2((size_t)n);
      for (int r = 0; r < n / 16; ++r)
        for (int j = 0; j < 16; ++j) t2[(size_t)r * 16 + j] = tw[(size_t)(r * j) % n];
      upload_table(h->tw2, t2, precision, h->stream);
    }
    {
      // live column-block tiles of the sphere pruning, in (my, cb) order
      const int ncb = h->tiles_data(), tcw = h->tcols();
      std::vector<int> lv;
      for (int my = 0; my < n; ++my) {
        const long long m = my <= n / 2 ? my : my - n;
        for (int cb = 0; cb < ncb; ++cb) {
          const long long mx0 = (long long)cb * tcw;
          if (4 * (mx0 * mx0 + m * m) <= (long long)n * n) lv.push_back(my * ncb + cb);
        }
      }
      h->nlive = (int)lv.size();
      alloc((void**)&h->live, lv.size() * sizeof(int));
      ck(cudaMemcpyAsync(h->live, lv.data(), lv.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream), "live");
      ck(cudaStreamSynchronize(h->stream), "live");
    }
    h->map_state_z = make_field_map(h->state, 6, 2, h->g, h->cbytes);
    h->map_work_y = make_field_map(h->work, 12, 1, h->g, h->cbytes);
    h->map_work_z = make_field_map(h->work, 12, 2, h->g, h->cbytes);
    ck(cudaMemsetAsync(h->state, 0, 6 * fb, h->stream), "memset");
    ck(cudaMemsetAsync(h->work, 0, 12 * fb, h->stream), "memset");
    if (precision == SNS_PRECISION_FP32) {
      // the precision form carries u compensated (hi + lo); the initial state has lo = 0
      alloc((void**)&h->ulo, comp_bytes(n, precision));
      ck(cudaMemsetAsync(h->ulo, 0, comp_bytes(n, precision), h->stream), "memset");
      h->comp = true;
    }
    const auto tw = twiddle_table(n);
    const auto ph = phase_table(n);
    upload_table(h->tw, tw, precision, h->stream);
    upload_table(h->phase, ph, precision, h->stream);
    initial_field(h, seed, pert_amp, pert_kmax);
    sync(h, "sns_create");
  } catch (const SnsError& e) {
    g_create_error = e.msg;
    release(h);
    return e.code;
  } catch (const std::exception& e) {
    g_create_error = e.what();
    release(h);
    return SNS_ERR_INVALID;
  }
  *out = h;
  return SNS_OK;
}

int sns_destroy(sns_handle* h) {
  if (h == nullptr) return SNS_ERR_INVALID;
  release(h);
  return SNS_OK;
}

const char* sns_last_error(const sns_handle* h) {
  if (h == nullptr) return g_create_error.c_str();
  return h->err.c_str();
}

int sns_set_viscosity(sns_handle* h, double nu) {
  if (h == nullptr) return SNS_ERR_INVALID;
  if (!(nu >= 0.0) || !std::isfinite(nu)) {
    h->err = "viscosity must be finite and non-negative";
    return SNS_ERR_INVALID;
  }
  h->nu = nu;
  // the device clock carries the viscosity for adaptive steps
  if (cudaSetDevice(h->device) != cudaSuccess ||
      cudaMemcpyAsync(h->clock + sns::kClockNu, &nu, sizeof(double), cudaMemcpyHostToDevice, h->stream) !=
          cudaSuccess ||
      cudaStreamSynchronize(h->stream) != cudaSuccess) {
    h->err = std::string("sns_set_viscosity: ") + cudaGetErrorString(cudaGetLastError());
    return SNS_ERR_CUDA;
  }
  return SNS_OK;
}

int sns_set_compensation(sns_handle* h, int enabled) {
  return guarded(h, [&] {
    if (enabled != 0 && enabled != 1) throw SnsError(SNS_ERR_INVALID, "enabled must be 0 or 1");
    if (h->precision != SNS_PRECISION_FP32) {
      if (enabled) throw SnsError(SNS_ERR_UNSUPPORTED, "the compensated state belongs to the FP32 precision form");
      return;
    }
    if (enabled && !h->comp) {
      // lo was not kept while off: the state restarts from its FP32 value
      ck(cudaMemsetAsync(h->ulo, 0, comp_bytes(h->n, h->precision), h->stream), "memset");
      sync(h, "sns_set_compensation");
    }
    h->comp = enabled == 1;
  });
}

int sns_set_sphere_pruning(sns_handle* h, int enabled) {
  return guarded(h, [&] {
    if (enabled != 0 && enabled != 1) throw SnsError(SNS_ERR_INVALID, "enabled must be 0 or 1");
    h->prune = enabled == 1;
  });
}

int sns_set_nonlinear_form(sns_handle* h, int form) {
  return guarded(h, [&] {
    if (form != SNS_FORM_CONSERVATIVE && form != SNS_FORM_ROTATIONAL)
      throw SnsError(SNS_ERR_INVALID, "form must be SNS_FORM_CONSERVATIVE (0) or SNS_FORM_ROTATIONAL (1)");
    if (form == SNS_FORM_ROTATIONAL && h->xf == nullptr) {
      size_t free_b = 0, total_b = 0;
      ck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
      if (3 * h->fbytes > free_b) throw SnsError(SNS_ERR_NOMEM, "no room for the 3 vorticity fields");
      const cudaError_t e = cudaMalloc((void**)&h->xf, 3 * h->fbytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        h->xf = nullptr;
        throw SnsError(SNS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
      }
      h->bytes += 3 * h->fbytes;
      ck(cudaMemsetAsync(h->xf, 0, 3 * h->fbytes, h->stream), "memset");  // padding columns stay zero
      h->map_x_z = make_field_map(h->xf, 3, 2, h->g, h->cbytes);
      sync(h, "sns_set_nonlinear_form");
    }
    h->form = form;
  });
}

int sns_launch_config(const sns_handle* h, int* out, int count) {
  if (h == nullptr || out == nullptr || count < 4) return SNS_ERR_INVALID;
  out[0] = h->tma_grid;
  out[1] = h->x2_grid;
  out[2] = h->p5_grid;
  int nb = 0;
  cudaDeviceGetAttribute(&nb, cudaDevAttrMultiProcessorCount, h->device);
  out[3] = nb;
  return SNS_OK;
}

int sns_grid_size(const sns_handle* h) { return h ? h->n : 0; }
size_t sns_device_bytes(const sns_handle* h) { return h ? h->bytes : 0; }

int sns_autotune(sns_handle* h, int trial_steps, const char* cache_path, int* out_config) {
  return guarded(h, [&] {
    if (trial_steps <= 0) throw SnsError(SNS_ERR_INVALID, "trial_steps must be positive");
    cudaDeviceProp prop{};
    ck(cudaGetDeviceProperties(&prop, h->device), "cudaGetDeviceProperties");
    std::string dev = prop.name;
    for (char& c : dev)
      if (c == ' ' || c == '\t') c = '_';
    const std::string key = dev + " " + std::to_string(h->n) + " " + std::to_string(h->precision);
    int nsm = 0;
    ck(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device), "cudaDeviceGetAttribute");
    const int x2_full = h->ops->xpass2_grid(nsm), p5_full = h->ops->p5_grid(nsm);
    const int tma_max = h->ops->tma_blocks_per_sm();
    auto apply = [&](int tma, int x2, int p5) {
      // only shapes this handle was built for: its Nyquist partial buffer is sized for x2_full
      if (tma < nsm || tma > nsm * tma_max || (x2 != 0 && x2 != x2_full) || (p5 != 0 && p5 != p5_full))
        return false;
      h->tma_grid = tma;
      h->x2_grid = x2;
      h->p5_grid = p5;
      return true;
    };
    bool cached = false;
    if (cache_path != nullptr) {
      if (FILE* f = std::fopen(cache_path, "r")) {
        char line[512];
        while (std::fgets(line, sizeof line, f)) {
          char name[256];
          int n = 0, prec = 0, tma = 0, x2 = 0, p5 = 0;
          if (std::sscanf(line, "sns-autotune %255s %d %d %d %d %d", name, &n, &prec, &tma, &x2, &p5) == 6 &&
              dev == name && n == h->n && prec == h->precision)
            cached = apply(tma, x2, p5);
        }
        std::fclose(f);
      }
    }
    if (!cached) {
      struct Shape {
        int tma, x2, p5;
      };
      std::vector<Shape> shapes;
      for (int k = 1; k <= tma_max && k <= 4; ++k)
        for (int x2 : {x2_full, 0})
          for (int p5 : {p5_full, 0}) {
            const Shape sh{nsm * k, x2, p5};
            bool dup = false;
            for (const Shape& o : shapes) dup = dup || (o.tma == sh.tma && o.x2 == sh.x2 && o.p5 == sh.p5);
            if (!dup) shapes.push_back(sh);
          }
      double best = 1e300;
      Shape pick = {h->tma_grid, h->x2_grid, h->p5_grid};
      for (const Shape& sh : shapes) {
        apply(sh.tma, sh.x2, sh.p5);
        step_once(h, 1.0e-4);  // warm-up of this shape
        ck(cudaEventRecord(h->ev0, h->stream), "event");
        for (int k = 0; k < trial_steps; ++k) step_once(h, 1.0e-4);
        ck(cudaEventRecord(h->ev1, h->stream), "event");
        sync(h, "sns_autotune");
        float ms = 0.f;
        ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
        if (ms < best) {
          best = ms;
          pick = sh;
        }
      }
      apply(pick.tma, pick.x2, pick.p5);
      if (cache_path != nullptr) {
        if (FILE* f = std::fopen(cache_path, "a")) {
          std::fprintf(f, "sns-autotune %s %d %d %d %d %d\n", dev.c_str(), h->n, h->precision, pick.tma, pick.x2,
                       pick.p5);
          std::fclose(f);
        }
      }
    }
    if (out_config) {
      out_config[0] = h->tma_grid;
      out_config[1] = h->x2_grid;
      out_config[2] = h->p5_grid;
    }
  });
}

int sns_set_clock(sns_handle* h, double t, double t_end, double cfl, double dt_max) {
  return guarded(h, [&] {
    if (!std::isfinite(t) || !(t_end > t) || !(cfl > 0.0) || !(dt_max > 0.0))
      throw SnsError(SNS_ERR_INVALID, "the clock needs t finite, t_end > t (INFINITY allowed), cfl > 0, dt_max > 0");
    double c[sns::kClockWords] = {};
    c[sns::kClockT] = t;
    c[sns::kClockTEnd] = t_end;
    c[sns::kClockCfl] = cfl;
    c[sns::kClockDtMax] = dt_max;
    c[sns::kClockDx] = 2.0 * kPi / static_cast<double>(h->n);
    c[sns::kClockNu] = h->nu;
    ck(cudaMemcpyAsync(h->clock, c, sizeof c, cudaMemcpyHostToDevice, h->stream), "clock");
    sync(h, "sns_set_clock");
  });
}

int sns_step_cfl(sns_handle* h, int nsteps) {
  return guarded(h, [&] {
    if (nsteps < 0) throw SnsError(SNS_ERR_INVALID, "negative step count");
    for (int k = 0; k < nsteps; ++k) step_on_clock(h);
    sync(h, "sns_step_cfl");
  });
}

int sns_get_clock(sns_handle* h, double* out, int count) {
  return guarded(h, [&] {
    if (out == nullptr || count < 4) throw SnsError(SNS_ERR_INVALID, "out needs 4 doubles");
    double c[sns::kClockWords];
    ck(cudaMemcpyAsync(c, h->clock, sizeof c, cudaMemcpyDeviceToHost, h->stream), "clock");
    sync(h, "sns_get_clock");
    out[0] = c[sns::kClockT];
    out[1] = c[sns::kClockDt];
    out[2] = c[sns::kClockSteps];
    out[3] = c[sns::kClockStopped];
  });
}

int sns_debug_set_error_word(sns_handle* h, int code) {
  return guarded(h, [&] {
    ck(cudaMemcpyAsync(h->err_word, &code, sizeof(int), cudaMemcpyHostToDevice, h->stream), "error word");
    ck(cudaStreamSynchronize(h->stream), "error word");
  });
}

int sns_debug_fail_after(sns_handle* h, int k) {
  if (h == nullptr) return SNS_ERR_INVALID;
  h->fail_after = k > 0 ? k : 0;
  return SNS_OK;
}

int sns_forward_r2c(sns_handle* h, const double* host_physical, double* host_spectral) {
  return guarded(h, [&] {
    if (!host_physical || !host_spectral) throw SnsError(SNS_ERR_INVALID, "null buffer");
    const size_t np = (size_t)h->n * h->n * h->n;
    double* phys = reinterpret_cast<double*>(h->wf(8));
    ck(cudaMemcpyAsync(phys, host_physical, np * sizeof(double), cudaMemcpyHostToDevice, h->stream), "upload");
    h->ops->xpass_r2c(phys, h->wf(0), 1, h->tw, h->g, h->stream);
    h->ops->ypass(h->wf(0), 1, -1, h->tiles_all(), h->tw, h->g, h->stream);
    h->ops->zpass(h->wf(0), h->wf(0), 1, -1, h->tiles_all(), 1.0, h->tw, h->g, h->stream);
    download_full(h, h->wf(0), host_spectral);
    sync(h, "sns_forward_r2c");
  });
}

int sns_backward_c2r(sns_handle* h, const double* host_spectral, double* host_physical) {
  return guarded(h, [&] {
    if (!host_physical || !host_spectral) throw SnsError(SNS_ERR_INVALID, "null buffer");
    const size_t np = (size_t)h->n * h->n * h->n;
    upload_full(h, host_spectral, h->wf(0), 1);
    h->ops->zpass(h->wf(0), h->wf(0), 1, +1, h->tiles_all(), h->inv_size(), h->tw, h->g, h->stream);
    h->ops->ypass(h->wf(0), 1, +1, h->tiles_all(), h->tw, h->g, h->stream);
    double* phys = reinterpret_cast<double*>(h->wf(8));
    h->ops->xpass_c2r(h->wf(0), phys, 1, h->tw, h->g, h->stream);
    ck(cudaMemcpyAsync(host_physical, phys, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "download");
    sync(h, "sns_backward_c2r");
  });
}

int sns_set_state(sns_handle* h, const double* const uhat_full[3]) {
  return guarded(h, [&] {
    if (!uhat_full || !uhat_full[0] || !uhat_full[1] || !uhat_full[2]) throw SnsError(SNS_ERR_INVALID, "null buffer");
    ck(cudaMemsetAsync(h->u(), 0, 3 * h->fbytes, h->stream), "memset");
    if (h->comp) ck(cudaMemsetAsync(h->ulo, 0, comp_bytes(h->n, h->precision), h->stream), "memset");
    bool dirty = false;
    for (int c = 0; c < 3; ++c) {
      upload_full(h, uhat_full[c], h->ucomp(c), 0, h->locomp(c));
      dirty = dirty || nyquist_plane_dirty(h->n, uhat_full[c]);
      sync(h, "sns_set_state");
    }
    h->nyq_clean = !dirty;
    h->sphere_clean = false;
  });
}

int sns_get_state(sns_handle* h, double* const uhat_full[3]) {
  return guarded(h, [&] {
    if (!uhat_full || !uhat_full[0] || !uhat_full[1] || !uhat_full[2]) throw SnsError(SNS_ERR_INVALID, "null buffer");
    for (int c = 0; c < 3; ++c) {
      download_full(h, h->ucomp(c), uhat_full[c], h->locomp(c));
      sync(h, "sns_get_state");
    }
  });
}

int sns_rhs(sns_handle* h, const double* const uhat_full[3], double* const rhs_full[3]) {
  return guarded(h, [&] {
    if (!uhat_full || !rhs_full) throw SnsError(SNS_ERR_INVALID, "null buffer");
    for (int c = 0; c < 3; ++c)
      if (!uhat_full[c] || !rhs_full[c]) throw SnsError(SNS_ERR_INVALID, "null buffer");
    // the RK scratch g doubles as the input state (g carries nothing between steps)
    char* uin = h->gb();
    ck(cudaMemsetAsync(uin, 0, 3 * h->fbytes, h->stream), "memset");
    bool dirty = false;
    for (int c = 0; c < 3; ++c) {
      upload_full(h, uhat_full[c], uin + (size_t)c * h->fbytes, 0);
      dirty = dirty || nyquist_plane_dirty(h->n, uhat_full[c]);
      sync(h, "sns_rhs upload");
    }
    const bool saved = h->nyq_clean;
    h->nyq_clean = !dirty;
    run_stage(h, uin, nullptr, 0, 0.0, 1, h->work, nullptr);
    h->nyq_clean = saved;
    for (int c = 0; c < 3; ++c) {
      download_full(h, h->wf(c), rhs_full[c]);
      sync(h, "sns_rhs");
    }
  });
}

int sns_nonlinear(sns_handle* h, const double* const uhat_full[3], double* const out_full[3]) {
  return guarded(h, [&] {
    if (!uhat_full || !out_full) throw SnsError(SNS_ERR_INVALID, "null buffer");
    for (int c = 0; c < 3; ++c)
      if (!uhat_full[c] || !out_full[c]) throw SnsError(SNS_ERR_INVALID, "null buffer");
    char* uin = h->gb();
    ck(cudaMemsetAsync(uin, 0, 3 * h->fbytes, h->stream), "memset");
    bool dirty = false;
    for (int c = 0; c < 3; ++c) {
      upload_full(h, uhat_full[c], uin + (size_t)c * h->fbytes, 0);
      dirty = dirty || nyquist_plane_dirty(h->n, uhat_full[c]);
      sync(h, "sns_nonlinear upload");
    }
    const bool saved = h->nyq_clean;
    h->nyq_clean = !dirty;
    run_stage(h, uin, nullptr, 0, 0.0, 2, h->work, nullptr);
    h->nyq_clean = saved;
    for (int c = 0; c < 3; ++c) {
      download_full(h, h->wf(c), out_full[c]);
      sync(h, "sns_nonlinear");
    }
  });
}

int sns_step(sns_handle* h, double dt, int nsteps) {
  return guarded(h, [&] {
    if (nsteps < 0 || !std::isfinite(dt)) throw SnsError(SNS_ERR_INVALID, "invalid dt or step count");
    for (int s = 0; s < nsteps; ++s) step_once(h, dt);
    sync(h, "sns_step");
  });
}

int sns_time_steps(sns_handle* h, double dt, int nsteps, double* elapsed_ms) {
  return guarded(h, [&] {
    if (nsteps < 0 || !std::isfinite(dt) || !elapsed_ms) throw SnsError(SNS_ERR_INVALID, "invalid argument");
    ck(cudaEventRecord(h->ev0, h->stream), "event");
    for (int s = 0; s < nsteps; ++s) step_once(h, dt);
    ck(cudaEventRecord(h->ev1, h->stream), "event");
    sync(h, "sns_time_steps");
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, h->ev0, h->ev1), "elapsed");
    *elapsed_ms = ms;
  });
}

int sns_profile_passes(sns_handle* h, double dt, int nsteps, double* pass_ms) {
  return guarded(h, [&] {
    if (nsteps <= 0 || !pass_ms) throw SnsError(SNS_ERR_INVALID, "invalid argument");
    PassMarks pm;
    pm.on = true;
    for (int i = 0; i < 8; ++i) ck(cudaEventCreate(&pm.ev[i]), "event");
    double acc[SNS_NUM_PASSES] = {0};
    for (int s = 0; s < nsteps; ++s) {
      for (int st = 0; st < 3; ++st) {
        run_stage(h, h->u(), h->gb(), st, dt, 0, nullptr, nullptr, &pm);
        h->nyq_clean = true;
        h->sphere_clean = true;
        sync(h, "sns_profile_passes");
        for (int i = 0; i < SNS_NUM_PASSES; ++i) {
          float ms = 0.f;
          ck(cudaEventElapsedTime(&ms, pm.ev[i], pm.ev[i + 1]), "elapsed");
          acc[i] += ms;
        }
      }
    }
    for (int i = 0; i < 8; ++i) cudaEventDestroy(pm.ev[i]);
    for (int i = 0; i < SNS_NUM_PASSES; ++i) pass_ms[i] = acc[i] / (3.0 * nsteps);
  });
}

int sns_max_velocity(sns_handle* h, double* out) {
  return guarded(h, [&] {
    if (!out) throw SnsError(SNS_ERR_INVALID, "null output");
    velocity_reductions(h);
    double r[2];
    ck(cudaMemcpyAsync(r, h->red, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "download");
    sync(h, "sns_max_velocity");
    *out = std::sqrt(r[1]);
  });
}

int sns_diagnostics(sns_handle* h, double t, sns_diag* out) {
  return guarded(h, [&] {
    if (!out) throw SnsError(SNS_ERR_INVALID, "null output");
    velocity_reductions(h);
    const int nb = 1184;  // 8 CTAs per SM on 148 SMs
    sns::launch_spectral_diag(h->u(), h->precision, h->partials + 2 * (size_t)h->n * h->n, nb, h->g, h->stream);
    sns::launch_reduce(h->partials + 2 * (size_t)h->n * h->n, nb, 2, 0, h->red + 2, h->stream);
    sns::launch_reduce(h->partials + 2 * (size_t)h->n * h->n + 1, nb, 2, 1, h->red + 3, h->stream);
    double r[4];
    ck(cudaMemcpyAsync(r, h->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "download");
    sync(h, "sns_diagnostics");
    const double n3 = (double)h->n * h->n * h->n;
    out->t = t;
    out->kinetic_energy = r[0] / n3;
    out->enstrophy = 0.5 * r[2] / (n3 * n3);
    out->dissipation = 2.0 * h->nu * out->enstrophy;
    out->max_spectral_divergence = r[3];
    out->max_velocity = std::sqrt(r[1]);
  });
}

int sns_dump_velocity(sns_handle* h, double* const phys[3]) {
  return guarded(h, [&] {
    if (!phys || !phys[0] || !phys[1] || !phys[2]) throw SnsError(SNS_ERR_INVALID, "null buffer");
    const size_t np = (size_t)h->n * h->n * h->n;
    h->ops->zpass(h->u(), h->work, 3, +1, h->tiles_all(), h->inv_size(), h->tw, h->g, h->stream);
    h->ops->ypass(h->work, 3, +1, h->tiles_all(), h->tw, h->g, h->stream);
    double* real = reinterpret_cast<double*>(h->wf(4));
    h->ops->xpass_c2r(h->work, real, 3, h->tw, h->g, h->stream);
    for (int c = 0; c < 3; ++c)
      ck(cudaMemcpyAsync(phys[c], real + c * np, np * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "dl");
    sync(h, "sns_dump_velocity");
  });
}

}  // extern "C"
