// Generic-shape transforms and the legacy solver's right-hand side on the device:
// sns_fft3d_* (the FFT-backend contract of FftwFft3D for any nx, ny, nz > 1 and any box
// lengths, src/fftw_fft.cpp:8-85 of ovankerm/Spectral_solver) and the host-vector
// SpectralNavierStokes numerics for those domains (src/spectral_solver.cpp:94-486:
// project, truncate, product_dealiased, nonlinear_rhs with or without the phase-shift pair,
// rhs, step_rk3, the diagnostics and the vorticity slice of write_vorticity_ppm).
//
// The fused pass kernels (sns_kernels.cu) serve the reference's benchmark domain: cubic,
// L = 2 pi, N in a fixed list, half spectrum.  This file serves everything else, in the
// reference's own storage: full complex fields [nz][ny][nx] of double2, x fastest.  One
// kernel transforms along any axis with a mixed-radix Stockham FFT whose radices are a
// runtime plan (8, 4, 2, 3, 5, 7 and any other prime as a direct DFT of that length):
// a CTA loads a tile of TW sequences into shared memory (TW consecutive x columns for the
// y and z axes, so every global access is a coalesced row segment; TW whole rows for x),
// runs the stages between two shared buffers, and writes the tile back.
#include "sns_kernels.cuh"
#include "../../include/sns_b200.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <exception>
#include <new>
#include <string>
#include <vector>

namespace {

constexpr int kMaxFactors = 24;
constexpr int kNT = 256;                    // threads per CTA of the axis kernel
constexpr int kMaxRegRadix = 16;            // radices up to this run from registers
constexpr size_t kSmemBudget = 200 * 1024;  // two tile buffers of L x TW complex doubles

struct AxisPlan {
  int L;                 // transform length
  int nfac;              // number of radices
  int fac[kMaxFactors];  // radices in application order (product L)
  int tw;                // sequences per tile
};

struct Dims {
  int nx, ny, nz;
};

// Element e of sequence s of tile t, as a flat index of the [nz][ny][nx] array; -1 when the
// sequence lies past the array's edge (partial last tile).
__device__ __forceinline__ long long axis_index(int axis, Dims d, int tw, long long t, int s, int e) {
  if (axis == 0) {
    const long long row = t * tw + s;
    if (row >= (long long)d.ny * d.nz) return -1;
    return row * d.nx + e;
  }
  const int xt = (d.nx + tw - 1) / tw;  // tiles across x
  const int x = (int)(t % xt) * tw + s;
  if (x >= d.nx) return -1;
  const long long other = t / xt;  // iz (axis 1) or iy (axis 2)
  if (axis == 1) return (other * d.ny + e) * d.nx + x;
  return ((long long)e * d.ny + other) * d.nx + x;
}

// One Stockham stage of radix r on all TW sequences: src -> dst (element e of sequence s
// at e * TW + s).  Butterfly j reads src[j + p L/r], p < r, and writes
// dst[(j / Ns) Ns r + j % Ns + q Ns] = sum_p src[j + p L/r] W_L^(p (k L/(Ns r) + q L/r)),
// k = j % Ns, W_L = exp(DIR 2 pi i / L): the stage twiddle and the radix-r DFT in one table
// lookup per term.
template <int DIR>
__device__ void generic_stage(const double2* __restrict__ src, double2* __restrict__ dst, int L, int tw, int r,
                              int Ns, const double2* __restrict__ twl) {
  const int m = L / r;
  const int stride = L / (Ns * r);
  const int total = tw * m;
  for (int b = threadIdx.x; b < total; b += blockDim.x) {
    const int s = b % tw, j = b / tw;
    const int k = j % Ns;
    const int base = (j / Ns) * Ns * r + k;
    if (r <= kMaxRegRadix) {
      double2 x[kMaxRegRadix];
#pragma unroll
      for (int p = 0; p < kMaxRegRadix; ++p)
        if (p < r) x[p] = src[(j + p * m) * tw + s];
      for (int q = 0; q < r; ++q) {
        const int a = k * stride + q * m;  // exponent step of this output (< L)
        double re = 0.0, im = 0.0;
        int e = 0;
#pragma unroll
        for (int p = 0; p < kMaxRegRadix; ++p) {
          if (p < r) {
            double2 w = __ldg(&twl[e]);
            if (DIR > 0) w.y = -w.y;
            re += x[p].x * w.x - x[p].y * w.y;
            im += x[p].x * w.y + x[p].y * w.x;
            e += a;
            if (e >= L) e -= L;
          }
        }
        dst[(base + q * Ns) * tw + s] = make_double2(re, im);
      }
    } else {
      for (int q = 0; q < r; ++q) {
        const int a = k * stride + q * m;
        double re = 0.0, im = 0.0;
        int e = 0;
        for (int p = 0; p < r; ++p) {
          const double2 v = src[(j + p * m) * tw + s];
          double2 w = __ldg(&twl[e]);
          if (DIR > 0) w.y = -w.y;
          re += v.x * w.x - v.y * w.y;
          im += v.x * w.y + v.y * w.x;
          e += a;
          if (e >= L) e -= L;
        }
        dst[(base + q * Ns) * tw + s] = make_double2(re, im);
      }
    }
  }
}

// Transform every sequence along `axis`.  in_real: the source is a real array (imaginary
// part 0; the forward transform of FftwFft3D::forward); out_real: only the real part, times
// `scale`, is written to a real array (FftwFft3D::backward).  Otherwise complex in -> complex
// out (may alias: each tile is read whole before it is written, and tiles are disjoint).
template <int DIR>
__global__ void __launch_bounds__(kNT)
k_axis_fft(const double2* __restrict__ in, const double* __restrict__ in_real, double2* __restrict__ out,
           double* __restrict__ out_real, double scale, int axis, Dims d, AxisPlan plan,
           const double2* __restrict__ twl) {
  extern __shared__ double2 sm[];
  const int L = plan.L, tw = plan.tw;
  double2* A = sm;
  double2* B = sm + (size_t)L * tw;
  const long long t = blockIdx.x;
  const int total = L * tw;
  // consecutive threads take consecutive x where the axis is strided, consecutive elements
  // along the row where it is x
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int s, e;
    if (axis == 0) {
      s = i / L;
      e = i % L;
    } else {
      s = i % tw;
      e = i / tw;
    }
    const long long g = axis_index(axis, d, tw, t, s, e);
    double2 v = make_double2(0.0, 0.0);
    if (g >= 0) v = in_real ? make_double2(in_real[g], 0.0) : in[g];
    A[e * tw + s] = v;
  }
  __syncthreads();
  double2* src = A;
  double2* dst = B;
  int Ns = 1;
  for (int f = 0; f < plan.nfac; ++f) {
    generic_stage<DIR>(src, dst, L, tw, plan.fac[f], Ns, twl);
    __syncthreads();
    Ns *= plan.fac[f];
    double2* tmp = src;
    src = dst;
    dst = tmp;
  }
  for (int i = threadIdx.x; i < total; i += blockDim.x) {
    int s, e;
    if (axis == 0) {
      s = i / L;
      e = i % L;
    } else {
      s = i % tw;
      e = i / tw;
    }
    const long long g = axis_index(axis, d, tw, t, s, e);
    if (g < 0) continue;
    const double2 v = src[e * tw + s];
    if (out_real) out_real[g] = v.x * scale;
    else out[g] = v;
  }
}

// ------------------------------------------------------------------------------------
// Point-wise kernels of the legacy solver (src/spectral_solver.cpp).  Mode numbers follow
// FftwFft3D::signed_mode (index n/2 -> +n/2), k = (2 pi m) / L per axis.
struct Modes {
  Dims d;
  double lx, ly, lz;  // box lengths
  double hx, hy, hz;  // half-cell shift L / (2 n) per axis (the phase-shift pair)
};

__device__ __forceinline__ int smode(int i, int n) { return i <= n / 2 ? i : i - n; }

struct Mode {
  double kx, ky, kz, k2;
  int mx, my, mz;
};

__device__ __forceinline__ Mode mode_of(long long id, const Modes& md) {
  constexpr double kTwoPi = 6.283185307179586476925286766559005768;
  Mode m;
  const int ix = (int)(id % md.d.nx);
  const int iy = (int)((id / md.d.nx) % md.d.ny);
  const int iz = (int)(id / ((long long)md.d.nx * md.d.ny));
  m.mx = smode(ix, md.d.nx);
  m.my = smode(iy, md.d.ny);
  m.mz = smode(iz, md.d.nz);
  m.kx = kTwoPi * m.mx / md.lx;
  m.ky = kTwoPi * m.my / md.ly;
  m.kz = kTwoPi * m.mz / md.lz;
  m.k2 = m.kx * m.kx + m.ky * m.ky + m.kz * m.kz;
  return m;
}

// keep_mode (src/spectral_solver.cpp:392-398): the ellipsoid sum (m / (n/2))^2 <= 1
__device__ __forceinline__ bool keep_of(const Mode& m, const Dims& d) {
  const double hx = d.nx / 2.0, hy = d.ny / 2.0, hz = d.nz / 2.0;
  return (m.mx * m.mx) / (hx * hx) + (m.my * m.my) / (hy * hy) + (m.mz * m.mz) / (hz * hz) <= 1.0;
}

// phase_shift_ (src/spectral_solver.cpp:48-54): exp(i (kx dx + ky dy + kz dz))
__device__ __forceinline__ double2 phase_of(const Mode& m, const Modes& md) {
  double s, c;
  sincos(m.kx * md.hx + m.ky * md.hy + m.kz * md.hz, &s, &c);
  return make_double2(c, s);
}

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// nf consecutive fields times the phase (the shifted grid's spectra)
__global__ void k_times_phase(const double2* __restrict__ u, double2* __restrict__ out, int nf, long long n3,
                              Modes md) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n3) return;
  const double2 ph = phase_of(mode_of(id, md), md);
  for (int c = 0; c < nf; ++c) out[c * n3 + id] = cm(u[c * n3 + id], ph);
}

__global__ void k_product(const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ p,
                          long long n3) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id < n3) p[id] = a[id] * b[id];
}

// One pair (a, b) of nonlinear_rhs (:186-228): the masked, dealiased (or plain) product
// spectrum into its slot.
__global__ void k_pair_value(const double2* __restrict__ c0, const double2* __restrict__ cs, double2* __restrict__ out,
                             long long n3, Modes md, int dealias) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n3) return;
  const Mode m = mode_of(id, md);
  double2 v = c0[id];
  if (dealias) {
    const double2 ph = phase_of(m, md);
    const double2 sb = cm(cs[id], make_double2(ph.x, -ph.y));
    v = make_double2(0.5 * (v.x + sb.x), 0.5 * (v.y + sb.y));
  }
  if (!keep_of(m, md.d)) v = make_double2(0.0, 0.0);
  out[id] = v;
}

// rhs_i = -i (kx P_0i + ky P_1i + kz P_2i), truncated (:230-238); then, for the full RHS
// (:242-260), minus nu k^2 u_hat, the projection with zero mean (:94-109, 400-409) and the
// truncation again.  P holds the 6 symmetric products in the order 00 01 02 11 12 22.
__global__ void k_rhs_finish(const double2* __restrict__ P, const double2* __restrict__ u, double2* __restrict__ r,
                             long long n3, Modes md, double nu, int full) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n3) return;
  const Mode m = mode_of(id, md);
  const bool keep = keep_of(m, md.d);
  const int slot[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
  double2 out[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const double2 p0 = P[slot[0][i] * n3 + id], p1 = P[slot[1][i] * n3 + id], p2 = P[slot[2][i] * n3 + id];
    const double sx = m.kx * p0.x + m.ky * p1.x + m.kz * p2.x;
    const double sy = m.kx * p0.y + m.ky * p1.y + m.kz * p2.y;
    out[i] = keep ? make_double2(sy, -sx) : make_double2(0.0, 0.0);  // -i (sx + i sy)
  }
  if (full) {
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      const double2 ui = u[i * n3 + id];
      out[i] = make_double2(out[i].x - nu * m.k2 * ui.x, out[i].y - nu * m.k2 * ui.y);
    }
    if (m.k2 != 0.0) {
      const double2 dot = make_double2(m.kx * out[0].x + m.ky * out[1].x + m.kz * out[2].x,
                                       m.kx * out[0].y + m.ky * out[1].y + m.kz * out[2].y);
      const double2 f = make_double2(dot.x / m.k2, dot.y / m.k2);
      const double kv[3] = {m.kx, m.ky, m.kz};
#pragma unroll
      for (int i = 0; i < 3; ++i) out[i] = make_double2(out[i].x - kv[i] * f.x, out[i].y - kv[i] * f.y);
    }
    if (id == 0 || !keep) out[0] = out[1] = out[2] = make_double2(0.0, 0.0);  // zero_mean, truncate
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) r[i * n3 + id] = out[i];
}

// One stage of step_rk3 (:262-309): g = a g + h (first stage: g = h), u += b g, project
// with zero mean, truncate.
__global__ void k_rk_stage(double2* __restrict__ u, double2* __restrict__ g, const double2* __restrict__ h,
                           long long n3, Modes md, double a, double b, int first) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n3) return;
  const Mode m = mode_of(id, md);
  double2 uu[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double2 hh = h[c * n3 + id];
    double2 gg = hh;
    if (!first) {
      const double2 go = g[c * n3 + id];
      gg = make_double2(a * go.x + hh.x, a * go.y + hh.y);
    }
    g[c * n3 + id] = gg;
    const double2 u0 = u[c * n3 + id];
    uu[c] = make_double2(u0.x + b * gg.x, u0.y + b * gg.y);
  }
  if (m.k2 != 0.0) {
    const double2 dot = make_double2(m.kx * uu[0].x + m.ky * uu[1].x + m.kz * uu[2].x,
                                     m.kx * uu[0].y + m.ky * uu[1].y + m.kz * uu[2].y);
    const double2 f = make_double2(dot.x / m.k2, dot.y / m.k2);
    const double kv[3] = {m.kx, m.ky, m.kz};
#pragma unroll
    for (int c = 0; c < 3; ++c) uu[c] = make_double2(uu[c].x - kv[c] * f.x, uu[c].y - kv[c] * f.y);
  }
  if (id == 0 || !keep_of(m, md.d)) uu[0] = uu[1] = uu[2] = make_double2(0.0, 0.0);
#pragma unroll
  for (int c = 0; c < 3; ++c) u[c * n3 + id] = uu[c];
}

// omega_hat = i k x u_hat (vorticity_hat, src/spectral_solver.cpp:338-351)
__global__ void k_vorticity_hat(const double2* __restrict__ u, double2* __restrict__ w, long long n3, Modes md) {
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n3) return;
  const Mode m = mode_of(id, md);
  const double2 ux = u[id], uy = u[n3 + id], uz = u[2 * n3 + id];
  const double2 cx = make_double2(m.ky * uz.x - m.kz * uy.x, m.ky * uz.y - m.kz * uy.y);
  const double2 cy = make_double2(m.kz * ux.x - m.kx * uz.x, m.kz * ux.y - m.kx * uz.y);
  const double2 cz = make_double2(m.kx * uy.x - m.ky * ux.x, m.kx * uy.y - m.ky * ux.y);
  w[id] = make_double2(-cx.y, cx.x);  // i (x + i y) = (-y, x)
  w[n3 + id] = make_double2(-cy.y, cy.x);
  w[2 * n3 + id] = make_double2(-cz.y, cz.x);
}

// Per-block partials of sum(0.5 |v|^2) and max |v|^2 over 3 real fields (fixed order).
__global__ void __launch_bounds__(256) k_sq_partials(const double* __restrict__ f, long long n3,
                                                     double* __restrict__ part) {
  __shared__ double ss[256], sm[256];
  double acc = 0.0, mx = 0.0;
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n3; i += (long long)gridDim.x * 256) {
    const double a = f[i], b = f[n3 + i], c = f[2 * n3 + i];
    const double q = a * a + b * b + c * c;
    acc += 0.5 * q;
    mx = fmax(mx, q);
  }
  ss[threadIdx.x] = acc;
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      ss[threadIdx.x] += ss[threadIdx.x + o];
      sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = ss[0];
    part[2 * blockIdx.x + 1] = sm[0];
  }
}

// max |k . u_hat| per block (max_spectral_divergence, :367-378)
__global__ void __launch_bounds__(256) k_div_partials(const double2* __restrict__ u, long long n3, Modes md,
                                                      double* __restrict__ part) {
  __shared__ double sm[256];
  double mx = 0.0;
  for (long long i = (long long)blockIdx.x * 256 + threadIdx.x; i < n3; i += (long long)gridDim.x * 256) {
    const Mode m = mode_of(i, md);
    const double2 a = u[i], b = u[n3 + i], c = u[2 * n3 + i];
    const double re = m.kx * a.x + m.ky * b.x + m.kz * c.x, im = m.kx * a.y + m.ky * b.y + m.kz * c.y;
    mx = fmax(mx, sqrt(re * re + im * im));
  }
  sm[threadIdx.x] = mx;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

// |v| on one z-plane of 3 real fields -> nx * ny doubles
__global__ void k_slice_mag(const double* __restrict__ f, long long n3, long long plane0, int nxy,
                            double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nxy) return;
  const double a = f[plane0 + i], b = f[n3 + plane0 + i], c = f[2 * n3 + plane0 + i];
  out[i] = sqrt(a * a + b * b + c * c);
}

// ------------------------------------------------------------------------------------
// Host side
struct GenericError : std::exception {
  int code;
  std::string msg;
  GenericError(int c, std::string m) : code(c), msg(std::move(m)) {}
  const char* what() const noexcept override { return msg.c_str(); }
};

void gck(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw GenericError(SNS_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// Radices of L in application order: 8s, a 4 or 2 for the rest of the power of two, then
// 3, 5, 7 and any larger prime (a direct DFT of that length).
bool factor(int L, AxisPlan& p) {
  p.L = L;
  p.nfac = 0;
  int rest = L;
  auto push = [&](int r) {
    if (p.nfac >= kMaxFactors) return false;
    p.fac[p.nfac++] = r;
    rest /= r;
    return true;
  };
  while (rest % 8 == 0)
    if (!push(8)) return false;
  if (rest % 4 == 0 && !push(4)) return false;
  if (rest % 2 == 0 && !push(2)) return false;
  for (int f = 3; rest > 1; f += 2) {
    if ((long long)f * f > rest) f = rest;
    while (rest % f == 0)
      if (!push(f)) return false;
  }
  return true;
}

unsigned blocks(long long n, int bs) { return (unsigned)((n + bs - 1) / bs); }

}  // namespace

struct sns_fft3d {
  Dims d{};
  double len[3] = {0, 0, 0};
  int device = 0;
  cudaStream_t stream = nullptr;
  long long n3 = 0;
  AxisPlan plan[3]{};
  double2* tw[3] = {nullptr, nullptr, nullptr};
  double2* work = nullptr;  // one complex field
  double* real = nullptr;   // one real field
  // the legacy solver's working set, allocated by the first solver call
  double2* sw = nullptr;  // 18 complex fields: u (3), g (3), h (3), products (6), scratch (3)
  double* pr = nullptr;   // 8 real fields: velocity on both grids (6), two products
  double* part = nullptr;  // reduction partials
  double* red = nullptr;
  size_t bytes = 0;
  std::string err;
};

namespace {

constexpr int kRedBlocks = 1184;

void launch_axis(sns_fft3d* h, int axis, int dir, const double2* in, const double* in_real, double2* out,
                 double* out_real, double scale) {
  const AxisPlan& p = h->plan[axis];
  const Dims& d = h->d;
  long long tiles;
  if (axis == 0) tiles = ((long long)d.ny * d.nz + p.tw - 1) / p.tw;
  else tiles = (long long)((d.nx + p.tw - 1) / p.tw) * (axis == 1 ? d.nz : d.ny);
  const size_t smem = 2 * (size_t)p.L * p.tw * sizeof(double2);
  if (dir < 0)
    k_axis_fft<-1><<<(unsigned)tiles, kNT, smem, h->stream>>>(in, in_real, out, out_real, scale, axis, d, p,
                                                                 h->tw[axis]);
  else
    k_axis_fft<+1><<<(unsigned)tiles, kNT, smem, h->stream>>>(in, in_real, out, out_real, scale, axis, d, p,
                                                                 h->tw[axis]);
}

// Forward transform of one real field into a complex field (x, y, z passes).
void forward_real(sns_fft3d* h, const double* real, double2* spec) {
  launch_axis(h, 0, -1, nullptr, real, spec, nullptr, 1.0);
  launch_axis(h, 1, -1, spec, nullptr, spec, nullptr, 1.0);
  launch_axis(h, 2, -1, spec, nullptr, spec, nullptr, 1.0);
}

// Re(IDFT(spec)) / N into a real field; `scratch` (a complex field) may alias `spec` when the
// spectrum need not survive.
void backward_real(sns_fft3d* h, const double2* spec, double2* scratch, double* real) {
  launch_axis(h, 2, +1, spec, nullptr, scratch, nullptr, 1.0);
  launch_axis(h, 1, +1, scratch, nullptr, scratch, nullptr, 1.0);
  launch_axis(h, 0, +1, scratch, nullptr, nullptr, real, 1.0 / (double)h->n3);
}

Modes modes_of(const sns_fft3d* h) {
  Modes m;
  m.d = h->d;
  m.lx = h->len[0];
  m.ly = h->len[1];
  m.lz = h->len[2];
  m.hx = 0.5 * h->len[0] / h->d.nx;
  m.hy = 0.5 * h->len[1] / h->d.ny;
  m.hz = 0.5 * h->len[2] / h->d.nz;
  return m;
}

void dalloc(sns_fft3d* h, void** p, size_t bytes) {
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw GenericError(SNS_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  h->bytes += bytes;
}

void ensure_solver_memory(sns_fft3d* h) {
  if (h->sw) return;
  const size_t cf = (size_t)h->n3 * sizeof(double2), rf = (size_t)h->n3 * sizeof(double);
  size_t free_b = 0, total_b = 0;
  gck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
  const size_t need = 18 * cf + 8 * rf + (2 * kRedBlocks + 16) * sizeof(double);
  if (need > free_b)
    throw GenericError(SNS_ERR_NOMEM, "the solver working set needs " + std::to_string(need) + " bytes, device has " +
                                          std::to_string(free_b) + " free");
  dalloc(h, (void**)&h->sw, 18 * cf);
  dalloc(h, (void**)&h->pr, 8 * rf);
  dalloc(h, (void**)&h->part, 2 * kRedBlocks * sizeof(double));
  dalloc(h, (void**)&h->red, 16 * sizeof(double));
}

double2* SW(sns_fft3d* h, int f) { return h->sw + (size_t)f * h->n3; }
double* PR(sns_fft3d* h, int f) { return h->pr + (size_t)f * h->n3; }
// slots of the working set
constexpr int kU = 0, kG = 3, kH = 6, kP = 9, kS = 15;

// nonlinear_rhs of u (slots kU) into slots `dst`; full = 1: the whole rhs
void rhs_device(sns_fft3d* h, double nu, int dealias, int full, int dst) {
  const long long n3 = h->n3;
  const Modes md = modes_of(h);
  const unsigned nb = blocks(n3, 256);
  for (int c = 0; c < 3; ++c) backward_real(h, SW(h, kU + c), SW(h, kS), PR(h, c));
  if (dealias) {
    k_times_phase<<<nb, 256, 0, h->stream>>>(SW(h, kU), SW(h, kS), 3, n3, md);
    for (int c = 0; c < 3; ++c) backward_real(h, SW(h, kS + c), SW(h, kS + c), PR(h, 3 + c));
  }
  const int pa[6] = {0, 0, 0, 1, 1, 2}, pb[6] = {0, 1, 2, 1, 2, 2};
  for (int p = 0; p < 6; ++p) {
    k_product<<<nb, 256, 0, h->stream>>>(PR(h, pa[p]), PR(h, pb[p]), PR(h, 6), n3);
    forward_real(h, PR(h, 6), SW(h, kS));
    if (dealias) {
      k_product<<<nb, 256, 0, h->stream>>>(PR(h, 3 + pa[p]), PR(h, 3 + pb[p]), PR(h, 7), n3);
      forward_real(h, PR(h, 7), SW(h, kS + 1));
    }
    k_pair_value<<<nb, 256, 0, h->stream>>>(SW(h, kS), SW(h, kS + 1), SW(h, kP + p), n3, md, dealias);
  }
  k_rhs_finish<<<nb, 256, 0, h->stream>>>(SW(h, kP), SW(h, kU), SW(h, dst), n3, md, nu, full);
}

void gsync(sns_fft3d* h, const char* what) {
  gck(cudaGetLastError(), what);
  gck(cudaStreamSynchronize(h->stream), what);
}

void upload3(sns_fft3d* h, const double* const f[3], int slot) {
  for (int c = 0; c < 3; ++c)
    gck(cudaMemcpyAsync(SW(h, slot + c), f[c], (size_t)h->n3 * sizeof(double2), cudaMemcpyHostToDevice, h->stream),
        "upload");
}
void download3(sns_fft3d* h, int slot, double* const f[3]) {
  for (int c = 0; c < 3; ++c)
    gck(cudaMemcpyAsync(f[c], SW(h, slot + c), (size_t)h->n3 * sizeof(double2), cudaMemcpyDeviceToHost, h->stream),
        "download");
}

bool null3(const void* const f[3]) { return f == nullptr || !f[0] || !f[1] || !f[2]; }

template <class F>
int guard(sns_fft3d* h, F&& f) {
  if (h == nullptr) return SNS_ERR_INVALID;
  try {
    gck(cudaSetDevice(h->device), "cudaSetDevice");
    f();
    h->err.clear();
    return SNS_OK;
  } catch (const GenericError& e) {
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

void release(sns_fft3d* h) {
  if (!h) return;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (auto* t : h->tw) cudaFree(t);
  cudaFree(h->work);
  cudaFree(h->real);
  cudaFree(h->sw);
  cudaFree(h->pr);
  cudaFree(h->part);
  cudaFree(h->red);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
}

}  // namespace

extern "C" {

int sns_fft3d_create(int nx, int ny, int nz, double lx, double ly, double lz, sns_fft3d** out) {
  sns::set_handleless_error("");
  if (out == nullptr) {
    sns::set_handleless_error("null output pointer");
    return SNS_ERR_INVALID;
  }
  *out = nullptr;
  if (nx <= 1 || ny <= 1 || nz <= 1) {
    sns::set_handleless_error("FFT grid dimensions must be greater than one");
    return SNS_ERR_INVALID;
  }
  if (!(lx > 0.0) || !(ly > 0.0) || !(lz > 0.0) || !std::isfinite(lx) || !std::isfinite(ly) || !std::isfinite(lz)) {
    sns::set_handleless_error("FFT box lengths must be positive and finite");
    return SNS_ERR_INVALID;
  }
  const int n[3] = {nx, ny, nz};
  AxisPlan plans[3];
  for (int a = 0; a < 3; ++a) {
    if (!factor(n[a], plans[a])) {
      sns::set_handleless_error("FFT axis length has too many factors");
      return SNS_ERR_UNSUPPORTED;
    }
    int tw = 8;
    while (tw > 1 && 2 * (size_t)n[a] * tw * sizeof(double2) > kSmemBudget) tw /= 2;
    if (2 * (size_t)n[a] * tw * sizeof(double2) > kSmemBudget) {
      char buf[160];
      std::snprintf(buf, sizeof buf, "FFT axis length %d is above the %zu points one CTA's shared memory holds", n[a],
                    kSmemBudget / (2 * sizeof(double2)));
      sns::set_handleless_error(buf);
      return SNS_ERR_UNSUPPORTED;
    }
    plans[a].tw = tw;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    sns::set_handleless_error("no CUDA device visible");
    return SNS_ERR_NO_DEVICE;
  }
  sns_fft3d* h = new (std::nothrow) sns_fft3d();
  if (h == nullptr) {
    sns::set_handleless_error("host allocation failed");
    return SNS_ERR_NOMEM;
  }
  try {
    gck(cudaGetDevice(&h->device), "cudaGetDevice");
    h->d = Dims{nx, ny, nz};
    h->len[0] = lx;
    h->len[1] = ly;
    h->len[2] = lz;
    h->n3 = (long long)nx * ny * nz;
    for (int a = 0; a < 3; ++a) h->plan[a] = plans[a];
    gck(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    size_t free_b = 0, total_b = 0;
    gck(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    const size_t need = (size_t)h->n3 * (sizeof(double2) + sizeof(double));
    if (need > free_b)
      throw GenericError(SNS_ERR_NOMEM, "grid needs " + std::to_string(need) + " bytes, device has " +
                                            std::to_string(free_b) + " free");
    dalloc(h, (void**)&h->work, (size_t)h->n3 * sizeof(double2));
    dalloc(h, (void**)&h->real, (size_t)h->n3 * sizeof(double));
    for (int a = 0; a < 3; ++a) {
      std::vector<double2> t((size_t)n[a]);
      sns::fill_twiddles(n[a], t.data());
      dalloc(h, (void**)&h->tw[a], t.size() * sizeof(double2));
      gck(cudaMemcpyAsync(h->tw[a], t.data(), t.size() * sizeof(double2), cudaMemcpyHostToDevice, h->stream), "tw");
      gck(cudaStreamSynchronize(h->stream), "tw");
    }
    gck(cudaFuncSetAttribute(k_axis_fft<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget), "attr");
    gck(cudaFuncSetAttribute(k_axis_fft<+1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBudget), "attr");
    gsync(h, "sns_fft3d_create");
  } catch (const GenericError& e) {
    sns::set_handleless_error(e.msg.c_str());
    release(h);
    return e.code;
  }
  *out = h;
  return SNS_OK;
}

int sns_fft3d_destroy(sns_fft3d* h) {
  if (h == nullptr) return SNS_ERR_INVALID;
  release(h);
  return SNS_OK;
}

const char* sns_fft3d_last_error(const sns_fft3d* h) { return h ? h->err.c_str() : "null handle"; }

size_t sns_fft3d_device_bytes(const sns_fft3d* h) { return h ? h->bytes : 0; }

int sns_fft3d_forward(sns_fft3d* h, const double* host_physical, double* host_spectral) {
  return guard(h, [&] {
    if (!host_physical || !host_spectral) throw GenericError(SNS_ERR_INVALID, "null buffer");
    gck(cudaMemcpyAsync(h->real, host_physical, (size_t)h->n3 * sizeof(double), cudaMemcpyHostToDevice, h->stream),
        "upload");
    forward_real(h, h->real, h->work);
    gck(cudaMemcpyAsync(host_spectral, h->work, (size_t)h->n3 * sizeof(double2), cudaMemcpyDeviceToHost, h->stream),
        "download");
    gsync(h, "sns_fft3d_forward");
  });
}

int sns_fft3d_backward(sns_fft3d* h, const double* host_spectral, double* host_physical) {
  return guard(h, [&] {
    if (!host_physical || !host_spectral) throw GenericError(SNS_ERR_INVALID, "null buffer");
    gck(cudaMemcpyAsync(h->work, host_spectral, (size_t)h->n3 * sizeof(double2), cudaMemcpyHostToDevice, h->stream),
        "upload");
    backward_real(h, h->work, h->work, h->real);
    gck(cudaMemcpyAsync(host_physical, h->real, (size_t)h->n3 * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
        "download");
    gsync(h, "sns_fft3d_backward");
  });
}

int sns_fft3d_rhs(sns_fft3d* h, double nu, int dealias, int full, const double* const uhat[3], double* const out[3]) {
  return guard(h, [&] {
    if (null3((const void* const*)uhat) || null3((const void* const*)out))
      throw GenericError(SNS_ERR_INVALID, "null buffer");
    if (!(nu >= 0.0) || (dealias != 0 && dealias != 1) || (full != 0 && full != 1))
      throw GenericError(SNS_ERR_INVALID, "nu must be >= 0, dealias and full 0 or 1");
    ensure_solver_memory(h);
    upload3(h, uhat, kU);
    rhs_device(h, nu, dealias, full, kH);
    download3(h, kH, out);
    gsync(h, "sns_fft3d_rhs");
  });
}

int sns_fft3d_step(sns_fft3d* h, double nu, int dealias, double dt, int nsteps, double* const uhat[3]) {
  return guard(h, [&] {
    if (null3((const void* const*)uhat)) throw GenericError(SNS_ERR_INVALID, "null buffer");
    if (!(nu >= 0.0) || (dealias != 0 && dealias != 1) || nsteps < 0 || !std::isfinite(dt))
      throw GenericError(SNS_ERR_INVALID, "nu must be >= 0, dealias 0 or 1, nsteps >= 0, dt finite");
    ensure_solver_memory(h);
    upload3(h, uhat, kU);
    const Modes md = modes_of(h);
    const unsigned nb = blocks(h->n3, 256);
    // Williamson low-storage RK3 with the reference's coefficient products (:262-309)
    const double a[3] = {0.0, -(5.0 / 9.0), -(153.0 / 128.0)};
    const double b[3] = {dt / 3.0, (15.0 / 16.0) * dt, (8.0 / 15.0) * dt};
    for (int s = 0; s < nsteps; ++s)
      for (int st = 0; st < 3; ++st) {
        rhs_device(h, nu, dealias, 1, kH);
        k_rk_stage<<<nb, 256, 0, h->stream>>>(SW(h, kU), SW(h, kG), SW(h, kH), h->n3, md, a[st], b[st], st == 0);
      }
    download3(h, kU, uhat);
    gsync(h, "sns_fft3d_step");
  });
}

int sns_fft3d_diagnostics(sns_fft3d* h, double nu, const double* const uhat[3], double t, sns_diag* out) {
  return guard(h, [&] {
    if (null3((const void* const*)uhat) || !out) throw GenericError(SNS_ERR_INVALID, "null buffer");
    ensure_solver_memory(h);
    upload3(h, uhat, kU);
    const Modes md = modes_of(h);
    const long long n3 = h->n3;
    for (int c = 0; c < 3; ++c) backward_real(h, SW(h, kU + c), SW(h, kS), PR(h, c));
    k_sq_partials<<<kRedBlocks, 256, 0, h->stream>>>(PR(h, 0), n3, h->part);
    sns::launch_reduce(h->part, kRedBlocks, 2, 0, h->red + 0, h->stream);
    sns::launch_reduce(h->part + 1, kRedBlocks, 2, 1, h->red + 1, h->stream);
    k_vorticity_hat<<<blocks(n3, 256), 256, 0, h->stream>>>(SW(h, kU), SW(h, kG), n3, md);
    for (int c = 0; c < 3; ++c) backward_real(h, SW(h, kG + c), SW(h, kS), PR(h, c));
    k_sq_partials<<<kRedBlocks, 256, 0, h->stream>>>(PR(h, 0), n3, h->part);
    sns::launch_reduce(h->part, kRedBlocks, 2, 0, h->red + 2, h->stream);
    k_div_partials<<<kRedBlocks, 256, 0, h->stream>>>(SW(h, kU), n3, md, h->part);
    sns::launch_reduce(h->part, kRedBlocks, 1, 1, h->red + 3, h->stream);
    double r[4];
    gck(cudaMemcpyAsync(r, h->red, sizeof r, cudaMemcpyDeviceToHost, h->stream), "download");
    gsync(h, "sns_fft3d_diagnostics");
    out->t = t;
    out->kinetic_energy = r[0] / (double)n3;
    out->enstrophy = r[2] / (double)n3;
    out->dissipation = 2.0 * nu * out->enstrophy;
    out->max_spectral_divergence = r[3];
    out->max_velocity = std::sqrt(r[1]);
  });
}

int sns_fft3d_product(sns_fft3d* h, const double* a_hat, const double* b_hat, double* out) {
  return guard(h, [&] {
    if (!a_hat || !b_hat || !out) throw GenericError(SNS_ERR_INVALID, "null buffer");
    ensure_solver_memory(h);
    const long long n3 = h->n3;
    const size_t cf = (size_t)n3 * sizeof(double2);
    gck(cudaMemcpyAsync(SW(h, kU), a_hat, cf, cudaMemcpyHostToDevice, h->stream), "upload");
    gck(cudaMemcpyAsync(SW(h, kU + 1), b_hat, cf, cudaMemcpyHostToDevice, h->stream), "upload");
    const Modes md = modes_of(h);
    const unsigned nb = blocks(n3, 256);
    // product_dealiased (src/spectral_solver.cpp:122-158): both grids, whatever the solver's
    // dealiasing flag
    for (int c = 0; c < 2; ++c) backward_real(h, SW(h, kU + c), SW(h, kS), PR(h, c));
    k_product<<<nb, 256, 0, h->stream>>>(PR(h, 0), PR(h, 1), PR(h, 6), n3);
    forward_real(h, PR(h, 6), SW(h, kH));
    k_times_phase<<<nb, 256, 0, h->stream>>>(SW(h, kU), SW(h, kS), 2, n3, md);
    for (int c = 0; c < 2; ++c) backward_real(h, SW(h, kS + c), SW(h, kS + c), PR(h, 3 + c));
    k_product<<<nb, 256, 0, h->stream>>>(PR(h, 3), PR(h, 4), PR(h, 7), n3);
    forward_real(h, PR(h, 7), SW(h, kH + 1));
    k_pair_value<<<nb, 256, 0, h->stream>>>(SW(h, kH), SW(h, kH + 1), SW(h, kP), n3, md, 1);
    gck(cudaMemcpyAsync(out, SW(h, kP), cf, cudaMemcpyDeviceToHost, h->stream), "download");
    gsync(h, "sns_fft3d_product");
  });
}

int sns_fft3d_vorticity_slice(sns_fft3d* h, const double* const uhat[3], int iz, double* host_mag) {
  return guard(h, [&] {
    if (null3((const void* const*)uhat) || !host_mag) throw GenericError(SNS_ERR_INVALID, "null buffer");
    if (iz < 0 || iz >= h->d.nz) throw GenericError(SNS_ERR_INVALID, "plane index out of range");
    ensure_solver_memory(h);
    upload3(h, uhat, kU);
    const long long n3 = h->n3;
    k_vorticity_hat<<<blocks(n3, 256), 256, 0, h->stream>>>(SW(h, kU), SW(h, kG), n3, modes_of(h));
    for (int c = 0; c < 3; ++c) backward_real(h, SW(h, kG + c), SW(h, kS), PR(h, c));
    const int nxy = h->d.nx * h->d.ny;
    k_slice_mag<<<blocks(nxy, 256), 256, 0, h->stream>>>(PR(h, 0), n3, (long long)iz * nxy, nxy, PR(h, 6));
    gck(cudaMemcpyAsync(host_mag, PR(h, 6), (size_t)nxy * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
        "download");
    gsync(h, "sns_fft3d_vorticity_slice");
  });
}

}  // extern "C"
