// Pass kernels of the B200 pseudo-spectral Taylor-Green step.  Every kernel is generic
// over the complex type C: double2 for the FP64 plain form, float2 for the FP32 precision
// form (fields stored in FP32; reductions, Nyquist sums and diagnostics accumulate in FP64).
//
// One RK3 stage of the reference (ava_taylor_green_impl.hpp:847-977 compute_rhs plus the
// stage update :994-1039) is five streaming passes over HBM:
//   P1 zpass_inv_phase : inverse z transform of u_hat, both grids from one read
//                        (the phase-shift kernel :866-873 fused in), 1/N^3 folded in
//   P2 ypass (inverse) : 6 fields
//   P3 xpass_products  : inverse x (c2r), the 6 products u_a*u_b on both grids,
//                        forward x (r2c) of all 12 (product kernel :903-906 fused)
//   P4 ypass (forward) : 12 fields
//   P5 zpass (forward) + sweep : dealias combine, mask, -i k, viscous term, Leray
//                        projection, low-storage RK3 update, projection of u
//                        (accumulate :926-936, add_viscous_project :955-974,
//                        RK update :994-1033, project_truncate :825-844)
// Two real transforms share one complex FFT along x (z = u + i*u_shifted on the way in,
// z = p0 + i*p_shifted on the way out), so every x transform is a full-length complex
// FFT with no r2c post-twiddle.
#include "sns_fft.cuh"
#include "sns_kernels.cuh"
#include "sns_tma.cuh"

#include <algorithm>
#include <type_traits>
#include <cstdio>

namespace sns {

// Columns per y/z tile: one 128-byte row segment (8 complex doubles, 16 complex floats).
template <class C>
constexpr int tile_cols() { return (int)(128 / sizeof(C)); }

__device__ __forceinline__ int signed_mode(int i, int n) { return i <= n / 2 ? i : i - n; }

template <int N, class C>
__device__ __forceinline__ void load_twiddles(C* sm_tw, const C* tw, int tid, int nt) {
  for (int t = tid; t < N; t += nt) sm_tw[t] = tw[t];
}

template <int N>
constexpr int nt_yz() { return N < 32 ? 32 : (N > 256 ? 256 : N); }
// x-pass block: N/2 threads clamped to [32, 256] and rounded up to whole warps (the block
// reductions and their full-mask shuffles need every warp complete: N = 96 gives 64)
template <int N>
constexpr int nt_x() { return ((N / 2 < 32 ? 32 : (N / 2 > 256 ? 256 : N / 2)) + 31) / 32 * 32; }

// ------------------------------------------------------------------------------------
// P1: inverse z transform with the fused phase shift.
// grid (ntiles, N [my], 3 [component]); tile = kT columns (one 128-byte row segment) x N rows (mz).
template <int N, class C>
__global__ void __launch_bounds__(nt_yz<N>())
k_zpass_inv_phase(const C* __restrict__ u, C* __restrict__ work, const C* __restrict__ tw,
                  const C* __restrict__ phase, double scale, Geom g) {
  constexpr int NT = nt_yz<N>();
  constexpr int kT = tile_cols<C>();
  extern __shared__ __align__(16) unsigned char smraw_yz[];
  C* smem = reinterpret_cast<C*>(smraw_yz);
  C* s_tw = smem;
  C* tile = smem + N;
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const int mx0 = blockIdx.x * kT;
  const int my = blockIdx.y;
  const int c = blockIdx.z;
  const C* src = u + (long long)c * g.field;
  C* dst0 = work + (long long)(2 * c) * g.field;
  C* dst1 = work + (long long)(2 * c + 1) * g.field;
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    tile[e] = cscale(src[((long long)row * N + my) * g.pitch + mx0 + col], scale);
  }
  __syncthreads();
  smem_fft<N, +1, kT, NT, ColTile<kT>>(tile, s_tw, tid);
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    dst0[((long long)row * N + my) * g.pitch + mx0 + col] = tile[e];
  }
  __syncthreads();
  const int smy = signed_mode(my, N);
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    // padding columns (> N/2) carry nothing; the Nyquist column mx = N/2 is transformed
    // too (consumed only when the state's Nyquist plane has content off (N/2,0,0))
    // Modes with 0 < mx < N/2 and index N/2 in exactly one of y, z: signed_mode gives +N/2
    // to the mode and to its mirror, so phase(-m) = -conj(phase(m)) and the reference's
    // shifted field is anti-Hermitian there; the real part it keeps of their inverse
    // transform is zero.  (With N/2 in both the two shifts cancel.  All of these modes
    // are zero in a masked state.)
    const int mx = mx0 + col;
    const bool anti = mx > 0 && mx < N / 2 && ((my == N / 2) != (row == N / 2));
    if (mx <= N / 2 && !anti) {
      const int msum = mx + smy + signed_mode(row, N);
      const C v = cscale(src[((long long)row * N + my) * g.pitch + mx], scale);
      tile[e] = cmul(v, phase[msum + 3 * N / 2]);
    } else {
      tile[e] = czero<C>();
    }
  }
  __syncthreads();
  smem_fft<N, +1, kT, NT, ColTile<kT>>(tile, s_tw, tid);
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    dst1[((long long)row * N + my) * g.pitch + mx0 + col] = tile[e];
  }
}

// y pass, in place.  grid (ntiles, N [z], nf).
template <int N, int DIR, class C>
__global__ void __launch_bounds__(nt_yz<N>())
k_ypass(C* __restrict__ f, const C* __restrict__ tw, Geom g) {
  constexpr int NT = nt_yz<N>();
  constexpr int kT = tile_cols<C>();
  extern __shared__ __align__(16) unsigned char smraw_yz[];
  C* smem = reinterpret_cast<C*>(smraw_yz);
  C* s_tw = smem;
  C* tile = smem + N;
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const int mx0 = blockIdx.x * kT;
  const int z = blockIdx.y;
  C* fld = f + (long long)blockIdx.z * g.field;
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    tile[e] = fld[((long long)z * N + row) * g.pitch + mx0 + col];
  }
  __syncthreads();
  smem_fft<N, DIR, kT, NT, ColTile<kT>>(tile, s_tw, tid);
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    fld[((long long)z * N + row) * g.pitch + mx0 + col] = tile[e];
  }
}

// z pass, src -> dst (may alias), optional scale on load.  grid (ntiles, N [y], nf).
template <int N, int DIR, class C>
__global__ void __launch_bounds__(nt_yz<N>())
k_zpass(const C* src, C* dst, double scale, const C* __restrict__ tw, Geom g) {
  constexpr int NT = nt_yz<N>();
  constexpr int kT = tile_cols<C>();
  extern __shared__ __align__(16) unsigned char smraw_yz[];
  C* smem = reinterpret_cast<C*>(smraw_yz);
  C* s_tw = smem;
  C* tile = smem + N;
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const int mx0 = blockIdx.x * kT;
  const int y = blockIdx.y;
  const C* fin = src + (long long)blockIdx.z * g.field;
  C* fout = dst + (long long)blockIdx.z * g.field;
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    tile[e] = cscale(fin[((long long)row * N + y) * g.pitch + mx0 + col], scale);
  }
  __syncthreads();
  smem_fft<N, DIR, kT, NT, ColTile<kT>>(tile, s_tw, tid);
  for (int e = tid; e < kT * N; e += NT) {
    const int row = e / kT, col = e % kT;
    fout[((long long)row * N + y) * g.pitch + mx0 + col] = tile[e];
  }
}


// ------------------------------------------------------------------------------------
// Streaming y/z pass, persistent and TMA-fed.  Each CTA walks tiles (field, fixed
// coordinate, TW-column block) with stride gridDim.x.  A tile (TW = 8 complex doubles or
// 16 complex floats x N rows, 128 bytes per row) lands in one of two shared-memory input buffers through
// cp.async.bulk.tensor (no multicast) while the previous tile is transformed, so HBM
// reads overlap the FFT.  The first radix stage reads the input buffer (scale and
// phase shift fused into that read), middle stages run in a work buffer, and the last
// stage stores straight to HBM as 128-byte row segments.
// VARIANT 1 is the inverse z pass of u_hat with the phase shift: one read, two outputs
// (U on field 2f and the shifted-grid V on field 2f+1).
template <int N>
constexpr int nt_tma() { return N < 64 ? 64 : (N > 512 ? 512 : N); }
template <int N>
constexpr int box_rows() { return N < 256 ? N : 256; }
template <int N, class C>
constexpr size_t tma_smem() { return (size_t)3 * 128 * N + (size_t)N * sizeof(C) + 128 + 2 * sizeof(uint64_t); }
// resident CTAs per SM the register budget is built for (shared memory allows this many)
template <int N>
constexpr int tma_minb() { return N >= 512 ? 1 : (N == 256 ? 2 : 4); }

template <int N, int AXIS, int DIR, int VARIANT, class C>
__global__ void __launch_bounds__(nt_tma<N>(), tma_minb<N>())
k_yz_tma(const __grid_constant__ CUtensorMap map, TmaArgs a, const C* __restrict__ tw,
         const C* __restrict__ phase, Geom g) {
  constexpr int NT = nt_tma<N>();
  constexpr int BR = box_rows<N>();
  constexpr int NBOX = N / BR;
  constexpr int TW = tile_cols<C>();
  constexpr uint32_t kTileBytes = 128u * N;
  using RT = real_of<C>;
  extern __shared__ unsigned char smraw[];
  __shared__ int s_fail;
  // 128-byte aligned layout: IN[0], IN[1], W (TW*N complex each), twiddles (N), 2 mbarriers
  const uint32_t pad = (128u - (smem_u32(smraw) & 127u)) & 127u;
  C* in0 = reinterpret_cast<C*>(smraw + pad);
  C* in1 = in0 + TW * N;
  C* W = in1 + TW * N;
  C* s_tw = W + TW * N;
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_tw + N);
  const int tid = threadIdx.x;
  for (int t = tid; t < N; t += NT) s_tw[t] = tw[t];
  const long long ntiles = (long long)a.nf * N * a.ncb;
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    s_fail = 0;
  }
  __syncthreads();
  auto issue = [&](long long t, int b) {
    const int cb = (int)(t % a.ncb);
    const long long q = t / a.ncb;
    const int c = (int)(q % N);
    const int f = a.f_in0 + (int)(q / N);
    C* dst = b ? in1 : in0;
    mbar_arrive_expect_tx(&bars[b], kTileBytes);
#pragma unroll
    for (int k = 0; k < NBOX; ++k) {
      if constexpr (AXIS == 1) tma_load_4d(dst + k * BR * TW, &map, &bars[b], cb * 2 * TW, k * BR, c, f);
      else tma_load_4d(dst + k * BR * TW, &map, &bars[b], cb * 2 * TW, c, k * BR, f);
    }
  };
  long long t = blockIdx.x;
  if (tid == 0) {
    if (t < ntiles) issue(t, 0);
    if (t + gridDim.x < ntiles) issue(t + gridDim.x, 1);
  }
  for (int k = 0; t < ntiles; ++k, t += gridDim.x) {
    const int b = k & 1;
    const uint32_t parity = (uint32_t)(k >> 1) & 1u;
    if (tid == 0 && !mbar_wait_bounded(&bars[b], parity)) s_fail = 1;
    __syncthreads();
    if (s_fail) {
      if (tid == 0) {
        atomicExch(a.err, kErrTmaTimeout);
        // let the other buffer's copy (if one is in flight) land before the CTA exits
        (void)mbar_wait_bounded(&bars[b ^ 1], (uint32_t)((k + 1) >> 1) & 1u);
      }
      return;
    }
    (void)mbar_try_wait(&bars[b], parity);  // acquire the landed tile in every thread
    const C* IN = b ? in1 : in0;
    const int cb = (int)(t % a.ncb);
    const long long q = t / a.ncb;
    const int c = (int)(q % N);
    const int fi = (int)(q / N);
    const int mx0 = cb * TW;
    const RT sc = (RT)a.scale;
    if constexpr (VARIANT == 0) {
      C* outf = static_cast<C*>(a.out) + (long long)(a.f_out0 + fi) * g.field;
      auto src = [&](int s, int e) {
        const C v = IN[SNS_IDX(e * TW + s, TW * N)];
        return sc == RT(1) ? v : cscale(v, sc);
      };
      auto dst = [&](int s, int e, C v) {
        const long long at = AXIS == 1 ? ((long long)c * N + e) * g.pitch : ((long long)e * N + c) * g.pitch;
        outf[SNS_IDX(at + mx0 + s, g.field)] = v;
      };
      tile_fft<N, DIR, NT, TW>(src, W, dst, s_tw, tid);
    } else {
      static_assert(AXIS == 2, "phase variant is the inverse z pass");
      C* out_u = static_cast<C*>(a.out) + (long long)(a.f_out0 + 2 * fi) * g.field;
      C* out_v = out_u + g.field;
      auto dst_u = [&](int s, int e, C v) { out_u[SNS_IDX(((long long)e * N + c) * g.pitch + mx0 + s, g.field)] = v; };
      auto dst_v = [&](int s, int e, C v) { out_v[SNS_IDX(((long long)e * N + c) * g.pitch + mx0 + s, g.field)] = v; };
      auto src_u = [&](int s, int e) { return cscale(IN[SNS_IDX(e * TW + s, TW * N)], sc); };
      tile_fft<N, DIR, NT, TW>(src_u, W, dst_u, s_tw, tid);
      __syncthreads();
      const int smy = signed_mode(c, N);
      auto src_v = [&](int s, int e) {
        // shifted grid: phase exp(i*pi*(mx+my+mz)/N); modes with 0 < mx < N/2 and index N/2
        // in exactly one of y, z are anti-Hermitian in the reference and drop out; columns
        // past N/2 are padding
        const int mx = mx0 + s;
        const bool anti = mx > 0 && mx < N / 2 && ((c == N / 2) != (e == N / 2));
        if (mx > N / 2 || anti) return czero<C>();
        const C v = cscale(IN[SNS_IDX(e * TW + s, TW * N)], sc);
        return cmul(v, __ldg(&phase[SNS_IDX(mx + smy + signed_mode(e, N) + 3 * N / 2, 3 * N + 1)]));
      };
      tile_fft<N, DIR, NT, TW>(src_v, W, dst_v, s_tw, tid);
    }
    __syncthreads();
    if (tid == 0 && t + 2LL * gridDim.x < ntiles) issue(t + 2LL * gridDim.x, b);
  }
}

// ------------------------------------------------------------------------------------
// Packing two Hermitian half spectra A, B (k in [0, N/2]) into Z = A + iB over k in [0, N).
// At k = 0 and k = N/2 only the real parts enter: that is the Hermitian part of the
// (y,z)-transformed mx = 0 and mx = N/2 planes, i.e. Re(IDFT) of the reference.
template <class C>
__device__ __forceinline__ void pack_pair(C A, C B, int k, int nh, int n, C* seq_at_k,
                                          C* seq_at_mirror) {
  if (k == 0 || k == nh) {
    *seq_at_k = cmk(A.x, B.x);
  } else {
    *seq_at_k = cmk(A.x - B.y, A.y + B.x);
    *seq_at_mirror = cmk(A.x + B.y, B.x - A.y);
  }
}

// Unpack Z = FFT(a + i b) into the half spectra of a and b at k.
template <class C>
__device__ __forceinline__ void unpack_pair(C Zk, C Zm, C* A, C* B) {
  using RT = real_of<C>;
  constexpr RT h = RT(0.5);
  *A = cmk(h * (Zk.x + Zm.x), h * (Zk.y - Zm.y));
  *B = cmk(h * (Zk.y + Zm.y), -h * (Zk.x - Zm.x));
}

template <int NT>
__device__ __forceinline__ void block_sum_max(double& s, double& m, double* red) {
  static_assert(NT % 32 == 0, "whole warps");
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  constexpr int NW = NT / 32;
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  __syncthreads();
  if (l == 0) { red[w] = s; red[NW + w] = m; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ss = 0.0, mm = 0.0;
    for (int i = 0; i < NW; ++i) { ss += red[i]; mm = fmax(mm, red[NW + i]); }
    s = ss;
    m = mm;
  }
}

// P3: fused inverse x / products / forward x.  One row (y, z) per CTA.
// Input work fields 0..5 = (U_0, V_0, U_1, V_1, U_2, V_2) [V = shifted grid] after the
// y and z inverse passes; output work fields 2p, 2p+1 = (P0_p, Ps_p) for the pairs
// p = 00, 01, 02, 11, 12, 22, columns 0..N/2 (column N/2: per-row Nyquist value).
template <int N, class C>
__global__ void __launch_bounds__(nt_x<N>())
k_xpass_products(C* __restrict__ work, const C* __restrict__ unyq, const C* __restrict__ phase,
                 double scale, int nyq_scalar, double* __restrict__ partials, const C* __restrict__ tw,
                 Geom g) {
  constexpr int NT = nt_x<N>();
  constexpr int NH = N / 2;
  constexpr int RP = row_pitch(N);
  extern __shared__ __align__(16) unsigned char smraw_x[];
  C* smem = reinterpret_cast<C*>(smraw_x);
  C* s_tw = smem;
  C* seq = smem + N;  // 6 sequences of pitch RP
  __shared__ double red[2 * (NT / 32)];
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const long long row = blockIdx.x;
  const long long rbase = row * g.pitch;
  // pack Z_c = U_c + i V_c
  for (int e = tid; e < 3 * (NH + 1); e += NT) {
    const int c = e / (NH + 1), k = e % (NH + 1);
    C A, B;
    if (k == NH && nyq_scalar) {
      // masked state: the mx = N/2 plane holds only (N/2,0,0); after the y/z inverse
      // transforms it is the constant c_N (and phase(N/2,0,0)*c_N on the shifted grid).
      const C cn = cscale(unyq[(long long)c * g.field + NH], scale);
      A = cn;
      B = cmul(cn, phase[NH + 3 * N / 2]);
    } else {
      A = work[(long long)(2 * c) * g.field + rbase + k];
      B = work[(long long)(2 * c + 1) * g.field + rbase + k];
    }
    C* sq = seq + c * RP;
    C zk, zm;
    pack_pair(A, B, k, NH, N, &zk, &zm);
    sq[k + (k >> 3)] = zk;
    if (k != 0 && k != NH) sq[(N - k) + ((N - k) >> 3)] = zm;
  }
  __syncthreads();
  smem_fft<N, +1, 3, NT, RowTile<RP>>(seq, s_tw, tid);
  double esum = 0.0, vmax2 = 0.0;
  for (int x = tid; x < N; x += NT) {
    const int p = x + (x >> 3);
    const C z0 = seq[p], z1 = seq[RP + p], z2 = seq[2 * RP + p];
    const double a0 = z0.x, a1 = z1.x, a2 = z2.x;
    const double s2 = a0 * a0 + a1 * a1 + a2 * a2;
    esum += 0.5 * s2;
    vmax2 = fmax(vmax2, s2);
    seq[0 * RP + p] = cmk(z0.x * z0.x, z0.y * z0.y);
    seq[1 * RP + p] = cmk(z0.x * z1.x, z0.y * z1.y);
    seq[2 * RP + p] = cmk(z0.x * z2.x, z0.y * z2.y);
    seq[3 * RP + p] = cmk(z1.x * z1.x, z1.y * z1.y);
    seq[4 * RP + p] = cmk(z1.x * z2.x, z1.y * z2.y);
    seq[5 * RP + p] = cmk(z2.x * z2.x, z2.y * z2.y);
  }
  if (partials != nullptr) {
    block_sum_max<NT>(esum, vmax2, red);
    if (tid == 0) {
      partials[2 * row] = esum;
      partials[2 * row + 1] = vmax2;
    }
  }
  __syncthreads();
  smem_fft<N, -1, 6, NT, RowTile<RP>>(seq, s_tw, tid);
  for (int e = tid; e < 6 * (NH + 1); e += NT) {
    const int pr = e / (NH + 1), k = e % (NH + 1);
    const int km = (N - k) % N;
    const C Zk = seq[pr * RP + k + (k >> 3)];
    const C Zm = seq[pr * RP + km + (km >> 3)];
    C A, B;
    unpack_pair(Zk, Zm, &A, &B);
    work[(long long)(2 * pr) * g.field + rbase + k] = A;
    work[(long long)(2 * pr + 1) * g.field + rbase + k] = B;
  }
}


// ------------------------------------------------------------------------------------
// P3 of the FP64 form for N = 256 (16 x 16) and N = 512 (16 x 32; the FP32 form runs
// k_xpass_w below): two-stage FFTs with one shared-memory round trip each.  Persistent CTAs;
// the 6 input rows of the next row group arrive by
// cp.async.bulk into a second staging buffer while the current group is transformed.
//   inverse stage A : radix 16 over stride-M inputs, the packing Z = U + iV (with the
//                     mirror and the real-part rule at mx = 0, N/2) fused into the loads
//   inverse stage B : radix M (M = 32 split over lane pairs, combined by a shuffle);
//                     z_c = u_c + i*u_shifted_c lands in work region 3 + c
//   forward stage A : the products p0 + i*ps fused into the loads, radix 16
//   forward stage B : radix M, then the r2c unpack P0(k), Ps(k) = (Z(k) +- conj Z(N-k))/2
//                     with the mirror fetched from the partner lane by a shuffle, and
//                     128-byte stores straight to HBM
// Both stages of one FFT run on the same warp (half-warp for N = 256), so they meet at a
// __syncwarp; the CTA synchronises twice per row group: before it starts (the previous
// group is done, its staging buffer is refilled) and between the inverse and forward
// FFTs (each product reads two components).
// The (N/2,0,0) sums of the 12 product planes accumulate in registers per CTA.
template <int N, class C>
struct XP {
  static constexpr int M = N / 16;                 // stage-B radix
  static constexpr bool PAIR = (M == 32);          // radix 32 as two radix-16 halves + shuffle
  static constexpr int NH = N / 2;
  // rows per iteration: two where their staging fits the CTA budget at two CTAs per SM
  // (N = 256), so one barrier sequence serves two rows; at N = 512 one (two rows, all six
  // warps busy in the inverse stages but one CTA per SM, measured slower)
  static constexpr int ROWS = (N == 256) ? 2 : 1;
  static constexpr int SP = N + N / 16;            // padded sequence (one slot per 16)
  static constexpr int NT = 192;
  // resident CTAs per SM the register budget is built for
  static constexpr int MINB = 2;
  // staged row of one field: NH + 1 values rounded up to 16 bytes (the bulk-copy unit)
  static constexpr int RS = (int)(((NH + 1) * sizeof(C) + 15) / 16 * 16 / sizeof(C));
  static constexpr int ROWIN = 6 * RS;
  static constexpr int STG = (ROWIN > 3 * SP ? ROWIN : 3 * SP);
  static constexpr uint32_t kRowBytes = RS * sizeof(C);
  static constexpr size_t smem = (size_t)(2 * ROWS * STG + ROWS * 6 * SP + N) * sizeof(C) + 128 +
                                 2 * sizeof(uint64_t);
};

__device__ __forceinline__ int pp16(int e) { return e + (e >> 4); }

// W_32^q = exp(-2*pi*i*q/32), q < 16, as the twiddle table holds it (exp(-2*pi*i*t/512) at
// t = 16 q, rounded from long double; the FP32 form rounds these doubles), so the radix-32
// combine of the two-stage x pass multiplies by immediates instead of loading them.
__host__ __device__ constexpr double w32_cos(int q) {  // cos(pi q / 16), 0 <= q <= 8
  return q == 0 ? 1.0 : q == 1 ? 0.98078528040323043 : q == 2 ? 0.92387953251128674 : q == 3 ? 0.83146961230254524
       : q == 4 ? 0.70710678118654757 : q == 5 ? 0.55557023301960218 : q == 6 ? 0.38268343236508978
       : q == 7 ? 0.19509032201612828 : 0.0;
}
template <class C>
__device__ __forceinline__ C w32(int q) {  // 0 <= q < 16 (unrolled: folds to immediates)
  const double re = q <= 8 ? w32_cos(q) : -w32_cos(16 - q);
  const double im = q <= 8 ? -w32_cos(8 - q) : -w32_cos(q - 8);
  return cmk((real_of<C>)re, (real_of<C>)im);
}

template <class C>
__device__ __forceinline__ C shfl2(C v, int src) {
  return cmk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
template <class C>
__device__ __forceinline__ C shfl2_xor(C v, int m) {
  return cmk(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

template <int N, class C>
__global__ void __launch_bounds__(192, XP<N, C>::MINB)
k_xpass2(C* __restrict__ work, const C* __restrict__ unyq, const C* __restrict__ phase,
         double scale, int nyq_scalar, double* __restrict__ nyq_part, const C* __restrict__ tw2_g, Geom g,
         int* err) {
  using X = XP<N, C>;
  constexpr int M = X::M, NH = X::NH, ROWS = X::ROWS, SP = X::SP, STG = X::STG, RS = X::RS;
  extern __shared__ unsigned char smraw[];
  __shared__ int s_fail;
  __shared__ double s_nyq[2][12];
  const uint32_t pad = (128u - (smem_u32(smraw) & 127u)) & 127u;
  C* stg = reinterpret_cast<C*>(smraw + pad);  // [2][ROWS][STG]
  C* W = stg + 2 * ROWS * STG;                       // [ROWS][6][SP]
  C* tw2 = W + ROWS * 6 * SP;                        // [M][16]: W_N^(r*j)
  uint64_t* bars = reinterpret_cast<uint64_t*>(tw2 + N);
  const int tid = threadIdx.x;
  for (int t = tid; t < N; t += 192) tw2[t] = tw2_g[t];
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    s_fail = 0;
  }
  __syncthreads();
  const long long niter = (long long)N * N / ROWS;
  auto issue = [&](long long it, int b) {
    mbar_arrive_expect_tx(&bars[b], ROWS * 6 * X::kRowBytes);
#pragma unroll
    for (int r = 0; r < ROWS; ++r) {
      const long long row = it * ROWS + r;
#pragma unroll
      for (int f = 0; f < 6; ++f)
        bulk_load(stg + (b * ROWS + r) * STG + f * RS, work + (long long)f * g.field + SNS_IDX(row, (long long)N * N) * g.pitch,
                  X::kRowBytes, &bars[b]);
    }
  };
  if (tid == 0 && blockIdx.x < niter) issue(blockIdx.x, 0);
  // Stage-B twiddles W_N^(j*rr), rr = 2 i + h: the same for every row this thread transforms
  // (inverse and forward stages B share the lane mapping), from the shared table.
  auto stage_b_tw = [&](int i, int j, int h) -> C { return tw2[(2 * i + h) * 16 + j]; };
  double nyq_p0 = 0.0, nyq_ps = 0.0;  // owned by the lane that holds k = N/2 of its pair
  int k = 0;
  for (long long it = blockIdx.x; it < niter; ++k, it += gridDim.x) {
    const int b = k & 1;
    const uint32_t parity = (uint32_t)(k >> 1) & 1u;
    if (tid == 0 && !mbar_wait_bounded(&bars[b], parity)) s_fail = 1;
    __syncthreads();
    if (s_fail) {  // no other copy is in flight: the next row group is issued after this wait
      if (tid == 0) atomicExch(err, kErrTmaTimeout);
      return;
    }
    (void)mbar_try_wait(&bars[b], parity);
    // every thread has finished the previous row group, so its staging buffer takes the next
    if (tid == 0 && it + gridDim.x < niter) issue(it + gridDim.x, b ^ 1);
    C* S = stg + b * ROWS * STG;

    // ---- inverse stage A: (r, c, t), packing fused into the loads
    if (tid < ROWS * 3 * M) {
      const int t = tid % M, c = (tid / M) % 3, r = tid / (3 * M);
      const C* Ur = S + r * STG + (2 * c) * RS;
      const C* Vr = Ur + RS;
      C v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) {
        const int x = t + M * q;
        C z;
        if (x == 0) {
          z = cmk(Ur[0].x, Vr[0].x);
        } else if (x < NH) {
          const C U = Ur[SNS_IDX(x, RS)], V = Vr[SNS_IDX(x, RS)];
          z = cmk(U.x - V.y, U.y + V.x);
        } else if (x == NH) {
          C U, V;
          if (nyq_scalar) {
            U = cscale(unyq[(long long)c * g.field + NH], scale);
            V = cmul(U, phase[NH + 3 * N / 2]);
          } else {
            U = Ur[NH];
            V = Vr[NH];
          }
          z = cmk(U.x, V.x);
        } else {
          const C U = Ur[SNS_IDX(N - x, RS)], V = Vr[SNS_IDX(N - x, RS)];
          z = cmk(U.x + V.y, V.x - U.y);
        }
        v[q] = z;
      }
      dft16<+1>(v);
      C* Wc = W + (r * 6 + c) * SP;
#pragma unroll
      for (int q = 0; q < 16; ++q) Wc[SNS_IDX(pp16(16 * t + q), SP)] = v[q];
    }
    __syncwarp();

    // ---- inverse stage B: z_c into work region 3 + c
    if constexpr (X::PAIR) {
      if (tid < ROWS * 96) {
        const int lane = tid & 31, c = (tid >> 5) % 3, r = tid / 96, j = lane & 15, h = lane >> 4;
        const C* Wc = W + (r * 6 + c) * SP;
        C v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int rr = 2 * i + h;
          v[i] = cmulc(Wc[SNS_IDX(pp16(j + 16 * rr), SP)], stage_b_tw(i, j, h));  // inverse twiddle = conj
        }
        dft16<+1>(v);
        if (h) {
#pragma unroll
          for (int q = 1; q < 16; ++q) v[q] = cmulc(v[q], w32<C>(q));  // conj W32^q
        }
        C* Zc = W + (r * 6 + 3 + c) * SP;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const C o = shfl2_xor(v[q], 16);
          const C z = h ? csub(o, v[q]) : cadd(v[q], o);
          Zc[SNS_IDX(pp16(j + 16 * (q + 16 * h)), SP)] = z;
        }
      }
    } else {
      if (tid < ROWS * 3 * 16) {
        const int j = tid & 15, c = (tid >> 4) % 3, r = tid / 48;
        const C* Wc = W + (r * 6 + c) * SP;
        C v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q)
          v[q] = q == 0 ? Wc[pp16(j)] : cmulc(Wc[SNS_IDX(pp16(j + 16 * q), SP)], tw2[SNS_IDX(q * 16 + j, N)]);
        dft16<+1>(v);
        C* Zc = W + (r * 6 + 3 + c) * SP;
#pragma unroll
        for (int q = 0; q < 16; ++q) Zc[SNS_IDX(pp16(j + 16 * q), SP)] = v[q];
      }
    }
    __syncthreads();

    // ---- forward stages, per row group; the warp (half-warp for N = 256) of product ab
    // runs both stages of its FFT.  Product ab lands in work region ab (ab < 3, free since
    // the inverse stage B) or in the consumed staging rows (ab >= 3).
    constexpr int FWD_ROWS = X::NT / (6 * M);  // rows one pass of the CTA covers
    static_assert(X::PAIR ? FWD_ROWS == 1 : FWD_ROWS == ROWS, "one forward pass per row group");
    auto prod = [&](int r, int ab) { return ab < 3 ? W + (r * 6 + ab) * SP : S + r * STG + (ab - 3) * SP; };
#pragma unroll 1
    for (int r0 = 0; r0 < ROWS; r0 += FWD_ROWS) {
      {
        // forward stage A: products fused into the loads
        const int t = tid % M, ab = (tid / M) % 6, r = r0 + tid / (6 * M);
        // pairs 00 01 02 11 12 22
        const int ca = (ab >= 3) + (ab >= 5), cb = ab < 3 ? ab : (ab < 5 ? ab - 2 : 2);
        const C* Za = W + (r * 6 + 3 + ca) * SP;
        const C* Zb = W + (r * 6 + 3 + cb) * SP;
        C v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int x = SNS_IDX(pp16(t + M * q), SP);
          const C za = Za[x];
          const C zb = ca == cb ? za : Zb[x];  // squares 00, 11, 22: one load
          v[q] = cmk(za.x * zb.x, za.y * zb.y);
        }
        dft16<-1>(v);
        C* Wp = prod(r, ab);
#pragma unroll
        for (int q = 0; q < 16; ++q) Wp[SNS_IDX(pp16(16 * t + q), SP)] = v[q];
      }
      __syncwarp();

      // forward stage B, r2c unpack through the partner lane, stores to HBM
      if constexpr (X::PAIR) {
        const int r = r0;
        const int lane = tid & 31, ab = tid >> 5, j = lane & 15, h = lane >> 4;
        const C* Wp = prod(r, ab);
        C v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int rr = 2 * i + h;
          v[i] = cmul(Wp[SNS_IDX(pp16(j + 16 * rr), SP)], stage_b_tw(i, j, h));
        }
        dft16<-1>(v);
        if (h) {
#pragma unroll
          for (int q = 1; q < 16; ++q) v[q] = cmul(v[q], w32<C>(q));
        }
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const C o = shfl2_xor(v[q], 16);
          v[q] = h ? csub(o, v[q]) : cadd(v[q], o);  // X(j + 16 (q + 16 h))
        }
        const int partner = ((16 - j) & 15) + 16 * (1 - h);
        const long long row = it * ROWS + r;
        C* o0 = work + (long long)(2 * ab) * g.field + row * g.pitch;
        C* o1 = o0 + g.field;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const C send = j == 0 ? v[(16 - i) & 15] : v[15 - i];
          const C recv = shfl2(send, partner);
          const C zm = (j == 0 && i == 0) ? v[0] : recv;
          const int kk = j + 16 * (16 * h + i);
          if (kk <= NH) {
            C A, B;
            unpack_pair(v[i], zm, &A, &B);
            o0[SNS_IDX(kk, g.pitch)] = A;
            o1[SNS_IDX(kk, g.pitch)] = B;
            if (kk == NH) {
              nyq_p0 += A.x;
              nyq_ps += B.x;
            }
          }
        }
      } else {
        const int j = tid & 15, sq = tid >> 4, r = sq / 6, ab = sq % 6;
        const C* Wp = prod(r, ab);
        C v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q)
          v[q] = q == 0 ? Wp[pp16(j)] : cmul(Wp[SNS_IDX(pp16(j + 16 * q), SP)], tw2[SNS_IDX(q * 16 + j, N)]);
        dft16<-1>(v);
        const int lane = tid & 31;
        const int partner = (lane & 16) + ((16 - j) & 15);
        const long long row = it * ROWS + r;
        C* o0 = work + (long long)(2 * ab) * g.field + row * g.pitch;
        C* o1 = o0 + g.field;
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const C recv = shfl2(v[15 - q], partner);
          const C zm = j == 0 ? v[(16 - q) & 15] : recv;
          const int kk = j + 16 * q;
          if (kk <= NH) {
            C A, B;
            unpack_pair(v[q], zm, &A, &B);
            o0[SNS_IDX(kk, g.pitch)] = A;
            o1[SNS_IDX(kk, g.pitch)] = B;
            if (kk == NH) {
              nyq_p0 += A.x;
              nyq_ps += B.x;
            }
          }
        }
      }
    }
    // the staging rows were written through st.shared; order that before the bulk copy
    // that refills them after the next row's barrier
    fence_proxy_async_smem();
  }
  // per-CTA Nyquist partials, fixed order: [field][cta]
  if constexpr (X::PAIR) {
    const int lane = tid & 31, ab = tid >> 5;
    if (lane == 16) {  // j = 0, h = 1 holds k = N/2
      nyq_part[(2 * ab) * gridDim.x + blockIdx.x] = nyq_p0;
      nyq_part[(2 * ab + 1) * gridDim.x + blockIdx.x] = nyq_ps;
    }
  } else {
    const int j = tid & 15, sq = tid >> 4, r = sq / 6, ab = sq % 6;
    if (j == 0) {
      s_nyq[r][2 * ab] = nyq_p0;
      s_nyq[r][2 * ab + 1] = nyq_ps;
    }
    __syncthreads();
    if (tid < 12) nyq_part[tid * gridDim.x + blockIdx.x] = s_nyq[0][tid] + s_nyq[1][tid];
  }
}

// ---------------------------------------------------------------------------------------
// x pass of the FP32 form at N = 128, 256 and 512: one warp owns R = 512 / N rows at a time and
// runs every stage of them alone, so the CTA (eight warps, one CTA per SM) never
// synchronises inside the loop.  The same operation as k_xpass2 (reference: the nonlinear
// term of spectral_solver.cpp:93-158, 169-215 on the r2c layout), reorganised so the three
// inverse transforms meet the products in registers:
//   inverse stage A  lane t (of M = N/16) per row: 16-point DFTs over x = t + M q, packing
//                    z_c = U_c + i V_c fused into the staged-row loads; out to Wc[c][t][k].
//                    The staging buffer is then free: the next row group's bulk copy is
//                    issued into it and lands while the rest of this group is transformed.
//   inverse stage B  lane (j, h): the M-point DFT over t at fixed k = j (four-step twiddle
//                    W_N^(j t) before; at N = 512 two half-warps and one shuffle; at N = 128
//                    8-point DFTs, a lane taking two of the warp's four rows in turn), leaving
//                    z_c(x) for x = j + 16 n, n of the lane, of all three components in
//                    registers
//   products + forward stage A  per product u_a u_b (both grids: real and imaginary part)
//                    the M-point DFT over n at fixed j (at N = 512 split in frequency: one
//                    shuffle, then a 16-point DFT; at N = 128 an 8-point DFT), times
//                    W_N^(j k1) / 2 (the r2c unpack's factor 1/2, exact); out to P[ab][j][k1]
//   forward stage B  lane k1: the 16-point DFT over j, outputs k1 + M k2; r2c unpack of the
//                    two grids through the partner lane (N - k), 128-byte stores to HBM
// The products run in two halves of three (00 01 02, then 11 12 22), each through Wc and its
// forward stage B, so a warp holds one staged row group and one transposition buffer.  Every
// transposition goes through shared memory once, XOR-swizzled (no bank conflicts); the
// products never do.  The kernel is bound by instruction issue, so its complex additions run
// as packed FP32 pairs (padd / psub, dft16<.., true>): the same results in fewer instructions.
template <int N>
struct XW {
  using C = float2;
  static constexpr int M = N / 16;      // inverse stage-A lanes per row, forward stage-B lanes
  static constexpr int R = 512 / N;     // rows per warp (32 lanes = R * M)
  static constexpr int NH = N / 2;
  static constexpr int WARPS = 8;
  static constexpr int RS = (int)(((NH + 1) * sizeof(C) + 15) / 16 * 16 / sizeof(C));  // staged row
  static constexpr int STG = R * 6 * RS;  // the staging buffer: [R][6 fields][RS]
  static constexpr int WC = R * 3 * N;    // transposition buffer [R][3][N]
  static constexpr int PER_WARP = STG + WC;
  static constexpr uint32_t kRowBytes = RS * sizeof(C);
  static constexpr int TWT = 16 * 32;     // four-step twiddles [i][lane], then the same halved
  static constexpr size_t smem = (size_t)(WARPS * PER_WARP + 2 * TWT) * sizeof(C) + 128 +
                                 WARPS * (sizeof(uint64_t) + R * 12 * sizeof(double));
  static_assert(R * M == 32, "a warp covers its rows' lanes");
};

// DIAG: the physical velocity's energy and vmax^2 instead (the inverse stages only): work
// fields 0..2 hold u_0..u_2 on one grid after the inverse z and y passes; the two packed
// sequences u_0 + i u_1 and u_2 meet in registers, each row's sum of |u|^2 / 2 and max of
// |u|^2 are reduced over its lanes, and the CTA's totals (rows in a fixed order per warp,
// warps in order) go to part[2 cta], part[2 cta + 1].
template <int N, bool DIAG = false>
__global__ void __launch_bounds__(32 * XW<N>::WARPS, 1)
k_xpass_w(float2* __restrict__ work, const float2* __restrict__ unyq, const float2* __restrict__ phase, double scale,
          int nyq_scalar, double* __restrict__ nyq_part, const float2* __restrict__ tw2_g, Geom g, int* err) {
  using X = XW<N>;
  using C = float2;
  constexpr int M = X::M, R = X::R, NH = X::NH, RS = X::RS;
  constexpr unsigned kFull = 0xffffffffu;
  extern __shared__ unsigned char smraw[];
  const uint32_t pad = (128u - (smem_u32(smraw) & 127u)) & 127u;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  C* const all = reinterpret_cast<C*>(smraw + pad);
  C* const stg = all + warp * X::PER_WARP;  // [R][6][RS]
  C* const Wc = stg + X::STG;               // [R][3][N], element (t, k) at 16 t + (k ^ (t & 15))
  C* const twt = all + X::WARPS * X::PER_WARP;  // [16][32]
  C* const twh = twt + X::TWT;                   // [16][32], times 1/2
  uint64_t* const bar = reinterpret_cast<uint64_t*>(twh + X::TWT) + warp;
  double* const s_nyq = reinterpret_cast<double*>(reinterpret_cast<uint64_t*>(twh + X::TWT) + X::WARPS);
  double* const my_nyq = s_nyq + warp * R * 12;  // [WARPS][R][12]
  for (int e = lane; e < R * 12; e += 32) my_nyq[e] = 0.0;
  if (lane == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  __syncwarp();
  const long long niter = (long long)N * N / R;
  const long long gw = (long long)blockIdx.x * X::WARPS + warp, nw = (long long)gridDim.x * X::WARPS;
  constexpr int NF = DIAG ? 3 : 6;  // staged fields per row
  constexpr int NC = DIAG ? 2 : 3;  // complex sequences per row (packed pairs of real fields)
  auto issue = [&](long long it) {
    mbar_arrive_expect_tx(bar, R * NF * X::kRowBytes);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const long long row = it * R + r;
#pragma unroll
      for (int f = 0; f < NF; ++f)
        bulk_load(stg + (r * 6 + f) * RS, work + (long long)f * g.field + SNS_IDX(row, (long long)N * N) * g.pitch,
                  X::kRowBytes, bar);
    }
  };
  if (lane == 0 && gw < niter) issue(gw);

  // Four-step twiddles: lane L (j = L & 15, h = L >> 4 at N = 512) visits rr = 2 i + h at
  // N = 512, rr = i at N = 256, and needs W_N^(j rr) = tw2[rr][j]; the CTA keeps them as
  // twt[i][L] (one table for every warp; consecutive lanes, consecutive words).  The forward
  // stage takes them halved (twh, exact): the r2c unpack's factor 1/2 rides on the twiddle
  // multiply that is there anyway, with bitwise the same results.
  constexpr int S2 = (N == 512) ? 2 : 1;
  const int j = lane & 15, hh = (N == 512) ? (lane >> 4) : 0;
  for (int e = tid; e < X::TWT; e += 32 * X::WARPS) {
    const int i = e >> 5, L = e & 31;
    const int rr = S2 * i + ((N == 512) ? (L >> 4) : 0);
    const C w = rr < M ? tw2_g[SNS_IDX(rr * 16 + (L & 15), N)] : cmk(0.f, 0.f);  // (N = 128: i < 8)
    twt[e] = w;
    twh[e] = cmk(0.5f * w.x, 0.5f * w.y);
  }
  __syncthreads();
  auto tw = [&](int i) -> C { return twt[SNS_IDX(i * 32 + lane, X::TWT)]; };
  auto twhalf = [&](int i) -> C { return twh[SNS_IDX(i * 32 + lane, X::TWT)]; };
  // Swizzles.  Wc: element (t, k) of a row at 16 t + (k ^ key); P: element (j, k1) of a row
  // and product at pslot.  At N = 128 a half-warp spans two rows, so the row enters both.
  auto wkey = [](int t, int r) { return N == 128 ? ((t + 8 * (r & 1)) & 15) : (t & 15); };
  auto pslot = [](int jr, int k1, int r) {
    if constexpr (N == 128) {
      const int jj = jr ^ (r & 1);
      return 8 * jj + (k1 ^ ((jj >> 1) & 7));
    } else {
      return M * jr + (k1 ^ jr);
    }
  };

  bool ok = true;
  int k = 0;
  double acc_es = 0.0, acc_vm = 0.0;  // DIAG: running totals of this lane's rows
  for (long long it = gw; it < niter; it += nw, ++k) {
    const bool landed = mbar_wait_bounded(bar, (uint32_t)k & 1u);
    if (!__all_sync(kFull, landed)) {  // the copy of this row group never landed; none other is in flight
      ok = false;
      break;
    }

    // ---- inverse stage A: lane (t, r), the three components in turn
    {
      const int t = lane % M, r = lane / M;
#pragma unroll 1
      for (int c = 0; c < NC; ++c) {
        const C* Ur = stg + (r * 6 + 2 * c) * RS;
        const C* Vr = Ur + RS;
        const bool has_v = !(DIAG && c == 1);  // the diagnostic's second sequence is u_2 alone
        C v[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          // x = t + M q: below N/2 for q < 8, N/2 + t for q = 8, above N/2 for q > 8
          const int x = t + M * q;
          C z;
          const C zero = cmk(0.f, 0.f);
          if (q == 0 && t == 0) {
            z = cmk(Ur[0].x, has_v ? Vr[0].x : 0.f);
          } else if (q < 8) {
            const C U = Ur[SNS_IDX(x, RS)], V = has_v ? Vr[SNS_IDX(x, RS)] : zero;
            z = cmk(U.x - V.y, U.y + V.x);
          } else if (q == 8 && t == 0) {
            C U, V;
            if (nyq_scalar) {
              if constexpr (DIAG) {
                U = cscale(unyq[(long long)(2 * c) * g.field + NH], (float)scale);
                V = has_v ? cscale(unyq[(long long)(2 * c + 1) * g.field + NH], (float)scale) : zero;
              } else {
                U = cscale(unyq[(long long)c * g.field + NH], (float)scale);
                V = cmul(U, phase[NH + 3 * N / 2]);
              }
            } else {
              U = Ur[NH];
              V = has_v ? Vr[NH] : zero;
            }
            z = cmk(U.x, V.x);
          } else {
            const C U = Ur[SNS_IDX(N - x, RS)], V = has_v ? Vr[SNS_IDX(N - x, RS)] : zero;
            z = cmk(U.x + V.y, V.x - U.y);
          }
          v[q] = z;
        }
        dft16<+1, C, true>(v);
        C* W = Wc + (r * 3 + c) * N;
#pragma unroll
        for (int q = 0; q < 16; ++q) W[SNS_IDX(16 * t + (q ^ wkey(t, r)), N)] = v[q];
      }
    }
    // the staged rows are consumed: order those reads before the bulk copy of the next row
    // group into the same buffer, which lands while this group is finished
    fence_proxy_async_smem();
    __syncwarp();
    if (lane == 0 && it + nw < niter) issue(it + nw);

    // ---- inverse stage B: z[p][c][q] = z_c(j + 16 n) of row rB(p), n = q + 16 h (N = 512),
    // n = q (N = 256, 128); at N = 128 (M = 8) a lane takes two rows in turn (p = 0, 1)
    constexpr int MP = (N == 128) ? 2 : 1;
    constexpr int NZ = 16 / MP;  // positions per lane and row
    auto row_b = [&](int p) { return N == 512 ? 0 : (N == 256 ? (lane >> 4) : 2 * p + (lane >> 4)); };
    C z[MP][3][NZ];  // (the diagnostic uses the first two)
#pragma unroll
    for (int p = 0; p < MP; ++p) {
      const int rB = row_b(p);
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const C* W = Wc + (rB * 3 + c) * N;
        C v[NZ];
#pragma unroll
        for (int i = 0; i < NZ; ++i) {
          const int rr = S2 * i + hh;  // the stage-A lane t whose output k = j this is
          v[i] = cmulc(W[SNS_IDX(16 * rr + (j ^ wkey(rr, rB)), N)], tw(i));  // inverse twiddle = conj
        }
        if constexpr (N == 128) {
          dft8<+1>(v);
        } else {
          dft16<+1, C, true>(v);
        }
        if constexpr (N == 512) {
          if (hh) {
#pragma unroll
            for (int q = 1; q < 16; ++q) v[q] = cmulc(v[q], w32<C>(q));  // conj W32^q
          }
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const C o = shfl2_xor(v[q], 16);
            z[p][c][q] = hh ? psub(o, v[q]) : padd(v[q], o);
          }
        } else {
#pragma unroll
          for (int q = 0; q < NZ; ++q) z[p][c][q] = v[q];
        }
      }
    }
    __syncwarp();  // Wc is read; the products overwrite it

    if constexpr (DIAG) {
      // |u|^2 = (u_0 + i u_1) magnitude^2 + u_2^2 per position, in FP64; a row's lanes are
      // the whole warp (N = 512) or one half-warp per row (N = 256, and each pass at 128)
#pragma unroll
      for (int p = 0; p < MP; ++p) {
        double es = 0.0, vm = 0.0;
#pragma unroll
        for (int q = 0; q < NZ; ++q) {
          const double ax = z[p][0][q].x, ay = z[p][0][q].y, bx = z[p][1][q].x;
          const double s2 = ax * ax + ay * ay + bx * bx;
          es += 0.5 * s2;
          vm = fmax(vm, s2);
        }
#pragma unroll
        for (int o = (N == 512 ? 16 : 8); o > 0; o >>= 1) {
          es += __shfl_xor_sync(kFull, es, o);
          vm = fmax(vm, __shfl_xor_sync(kFull, vm, o));
        }
        acc_es += es;  // every lane of the row holds the row's totals
        acc_vm = fmax(acc_vm, vm);
      }
      __syncwarp();  // Wc is read; the next row group's inverse stage A overwrites it
    }

#pragma unroll
    for (int half = 0; half < (DIAG ? 0 : 2); ++half) {
      // ---- products and forward stage A: P[ab % 3][j][k1] in Wc at pslot(j, k1, row)
#pragma unroll
      for (int p = 0; p < MP; ++p) {
        const int rB = row_b(p);
#pragma unroll
        for (int ab = 3 * half; ab < 3 * half + 3; ++ab) {
          // pairs 00 01 02 11 12 22
          const int ca = (ab >= 3) + (ab >= 5), cb = ab < 3 ? ab : (ab < 5 ? ab - 2 : 2);
          C v[NZ];
#pragma unroll
          for (int q = 0; q < NZ; ++q) v[q] = pmul(z[p][ca][q], z[p][cb][q]);
          if constexpr (N == 512) {
            // M = 32 split in frequency: h = 0 takes p(n) + p(n + 16) (even k1), h = 1 takes
            // (p(n) - p(n + 16)) W32^n (odd k1)
#pragma unroll
            for (int q = 0; q < 16; ++q) {
              const C o = shfl2_xor(v[q], 16);
              v[q] = hh ? (q == 0 ? psub(o, v[q]) : cmul(psub(o, v[q]), w32<C>(q))) : padd(v[q], o);
            }
          }
          if constexpr (N == 128) {
            dft8<-1>(v);
          } else {
            dft16<-1, C, true>(v);
          }
          C* Pab = Wc + ((ab % 3) * R + rB) * N;
#pragma unroll
          for (int m = 0; m < NZ; ++m) {
            const int k1 = S2 * m + hh;
            Pab[SNS_IDX(pslot(j, k1, rB), N)] = cmul(v[m], twhalf(m));  // W_N^(j k1) / 2
          }
        }
      }
      __syncwarp();

      // ---- forward stage B, r2c unpack through the partner lane, stores to HBM
      {
        const int k1 = lane % M, r = lane / M;
        const int partner = (N == 512) ? ((32 - lane) & 31) : ((lane & ~(M - 1)) + ((M - k1) & (M - 1)));
        const long long row = it * R + r;
#pragma unroll 1
        for (int ab = 3 * half; ab < 3 * half + 3; ++ab) {
          const C* Pab = Wc + ((ab % 3) * R + r) * N;
          C v[16];
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) v[jj] = Pab[SNS_IDX(pslot(jj, k1, r), N)];
          dft16<-1, C, true>(v);  // v[i] = X(k1 + M i)
          C* o0 = work + (long long)(2 * ab) * g.field + row * g.pitch;
          C* o1 = o0 + g.field;
          // outputs k = k1 + M i <= N/2 only: i <= 8 (i = 8 is the Nyquist column, lane k1 = 0)
#pragma unroll
          for (int i = 0; i <= NH / M; ++i) {
            const C send = k1 == 0 ? v[(16 - i) & 15] : v[15 - i];
            const C zm = shfl2(send, partner);  // X(N - k1 - M i)
            const int kk = k1 + M * i;
            if (kk <= NH) {
              // r2c unpack of the halved transform: A = X(k) + conj X(N-k), B = -i (X(k) - conj X(N-k))
              const C sm = padd(v[i], zm), df = psub(v[i], zm);
              const C A = cmk(sm.x, df.y), B = cmk(sm.y, -df.x);
              o0[SNS_IDX(kk, g.pitch)] = A;
              o1[SNS_IDX(kk, g.pitch)] = B;
              if (kk == NH) {
                my_nyq[r * 12 + 2 * ab] += A.x;
                my_nyq[r * 12 + 2 * ab + 1] += B.x;
              }
            }
          }
        }
      }
      __syncwarp();  // Wc is read; the next half (or the next row group) overwrites it
    }
  }
  if (!ok && lane == 0) atomicExch(err, kErrTmaTimeout);
  if constexpr (DIAG) {
    // one lane per row group: lane 0 (N = 512: the warp is one row), lanes 0 and 16 otherwise
    double w_es = acc_es, w_vm = acc_vm;
    if constexpr (N != 512) {
      w_es = __shfl_sync(kFull, acc_es, 0) + __shfl_sync(kFull, acc_es, 16);
      w_vm = fmax(__shfl_sync(kFull, acc_vm, 0), __shfl_sync(kFull, acc_vm, 16));
    }
    if (lane == 0) {
      s_nyq[2 * warp] = w_es;
      s_nyq[2 * warp + 1] = w_vm;
    }
    __syncthreads();
    if (tid == 0) {
      double es = 0.0, vm = 0.0;
#pragma unroll 1
      for (int w = 0; w < X::WARPS; ++w) {
        es += s_nyq[2 * w];
        vm = fmax(vm, s_nyq[2 * w + 1]);
      }
      nyq_part[2 * blockIdx.x] = es;
      nyq_part[2 * blockIdx.x + 1] = vm;
    }
    return;
  }
  // per-CTA Nyquist partials, fixed order: [field][cta]
  __syncthreads();
  if (tid < 12) {
    double s = 0.0;
#pragma unroll 1
    for (int w = 0; w < X::WARPS * R; ++w) s += s_nyq[w * 12 + tid];
    nyq_part[tid * gridDim.x + blockIdx.x] = s;
  }
}

// Nyquist-plane sums: column N/2 of each of the 12 product fields summed over all rows
// (the (N/2,0,0) output of the y/z forward transforms is the plain sum of the plane).
// grid 12, fixed summation order.
template <class C>
__global__ void __launch_bounds__(256) k_nyq_reduce(const C* __restrict__ work, double* __restrict__ sums,
                                                    Geom g) {
  __shared__ double red[256];
  const C* f = work + (long long)blockIdx.x * g.field + g.nh;
  const long long rows = (long long)g.n * g.n;
  double s = 0.0;
  for (long long r = threadIdx.x; r < rows; r += 256) s += f[r * g.pitch].x;
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) sums[blockIdx.x] = red[0];
}

// ------------------------------------------------------------------------------------
// P5 sweep: per mode, the reference's accumulate (:926-936), add_viscous_project
// (:955-974), RK stage update (:994-1033) and project_truncate (:825-844).
template <class C>
struct ModeIn {
  C p0[6];
  C ps[6];
};

template <class C>
__device__ __forceinline__ C minus_i_k(C a, int k) {
  const real_of<C> rk = (real_of<C>)k;
  return cmk(rk * a.y, -rk * a.x);
}

// Dealiased product value of one pair at one mode (accumulate lambda, :928-931).
template <class C>
__device__ __forceinline__ C pair_value(C p0, C ps, C phase, bool keep, int dealias) {
  C value = dealias ? cscale(cadd(p0, cmulc(ps, phase)), 0.5) : p0;
  if (!keep) value = czero<C>();
  return value;
}

// Viscous term, Leray projection and mask (:955-974), then the RK stage update and the
// projection of u (:994-1039) -- or the RHS itself in modes 1 and 2.
template <class C>
__device__ __forceinline__ void finish_mode(C r[3], int ix, int iy, int iz, int n, C uu[3], C gg[3],
                                            bool load_g, C rr[3], const SweepArgs& a, CompWord lo[3]);

// Compensated state of the FP32 precision form.  The RK update u += b*dt*g adds an
// increment some 1e-3 of |u| at dt = 1e-3; rounding u to FP32 after every stage drops the
// increment's low bits, and over thousands of steps that dominates the form's error.  So u
// is carried as its stored FP32 value hi plus a remainder, and the sweep forms the update
// in FP64 from the two.  The remainder U - hi of each real part is kept as an int8 q, the
// remainder in units of ulp(hi)/255 truncated toward zero (so |q| <= 127 and the decoded
// value never reaches the rounding boundary of hi: round-to-nearest(hi + lo) == hi), and a
// decoded pair encodes back to the same pair, so states round-trip exactly through the host.
// The precision kept is about ulp(hi)/255, 2^-32 relative, against 2^-24 for FP32 alone.
// ulp(hi) = 2^(E - 150) and its inverse, E the biased exponent of hi (at least 1), built from
// the exponent bits: no division anywhere in the encoding.
__device__ __forceinline__ int comp_exp(float hi) {
  const int e = (int)((__float_as_uint(hi) >> 23) & 0xffu);
  return e > 0 ? e : 1;
}
__device__ __forceinline__ double pow2(int k) { return __longlong_as_double((long long)(k + 1023) << 52); }
__device__ __forceinline__ double comp_part(float hi, int q) {
  return (double)q * pow2(comp_exp(hi) - 150) * (1.0 / 255.0);
}
__device__ __forceinline__ int comp_q(double U, float hi) {
  const double r = (U - (double)hi) * pow2(150 - comp_exp(hi)) * 255.0;  // U - hi exact; |r| <= 127.5
  // toward zero, after a nudge of 1e-6 away from it: a decoded remainder (an integer up to
  // FP64 round-off) comes back as the same integer, and the bounds 63.75 (hi a power of two,
  // U below it) and 127.5 are never crossed
  return (int)trunc(r + copysign(1.0e-6, r));
}
__device__ __forceinline__ double2 comp_decode(float2 hi, CompWord lo) {
  const int qr = (int)(int8_t)(lo & 0xffu), qi = (int)(int8_t)(lo >> 8);
  return make_double2((double)hi.x + comp_part(hi.x, qr), (double)hi.y + comp_part(hi.y, qi));
}
__device__ __forceinline__ float2 comp_encode(double2 U, CompWord* lo) {
  const float2 hi = make_float2(__double2float_rn(U.x), __double2float_rn(U.y));
  const int qr = comp_q(U.x, hi.x), qi = comp_q(U.y, hi.y);
  *lo = (CompWord)(((unsigned)(qr & 0xff)) | ((unsigned)(qi & 0xff) << 8));
  return hi;
}

// Per-stage scalars with the step taken from a device clock: the same expressions as the
// host's stage arguments (the reference's Real-typed products, :998, 1014, 1030), on the
// clock's current step size.
__device__ __forceinline__ SweepArgs resolve_step(SweepArgs a) {
  if (a.clock == nullptr) return a;
  const double dt = a.clock[kClockDt];
  a.frozen = a.clock[kClockStopped] != 0.0;
  a.nu = a.clock[kClockNu];
  if (a.stage == 0) {
    a.ub = dt / 3.0;
    a.if_tau = dt / 3.0;
  } else if (a.stage == 1) {
    a.ub = 15.0 * dt / 16.0;
    a.if_tau = 5.0 * dt / 12.0;
  } else {
    a.ub = 8.0 * dt / 15.0;
    a.if_tau = dt / 4.0;
  }
  return a;
}

template <class C>
__device__ __forceinline__ void sweep_mode(const ModeIn<C>& in, int ix, int iy, int iz, int n, C phase,
                                           C uu[3], C gg[3], bool load_g, C rr[3],
                                           const SweepArgs& a, CompWord lo[3]) {
  const int m2 = ix * ix + iy * iy + iz * iz;
  const bool keep = 4LL * m2 <= (long long)n * n;
  const int kv[3] = {ix, iy, iz};
  C r[3] = {czero<C>(), czero<C>(), czero<C>()};
  const int pa[6] = {0, 0, 0, 1, 1, 2};
  const int pb[6] = {0, 1, 2, 1, 2, 2};
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    const C value = pair_value(in.p0[p], in.ps[p], phase, keep, a.dealias);
    r[pa[p]] = cadd(r[pa[p]], minus_i_k(value, kv[pb[p]]));
    if (pa[p] != pb[p]) r[pb[p]] = cadd(r[pb[p]], minus_i_k(value, kv[pa[p]]));
  }
  finish_mode(r, ix, iy, iz, n, uu, gg, load_g, rr, a, lo);
}

template <class C>
__device__ __forceinline__ void finish_mode(C r[3], int ix, int iy, int iz, int n, C uu[3], C gg[3],
                                            bool load_g, C rr[3], const SweepArgs& a, CompWord lo[3]) {
  const int m2 = ix * ix + iy * iy + iz * iz;
  const bool keep = 4LL * m2 <= (long long)n * n;
  const double k2 = (double)m2;
  if (a.mode == 2) {  // nonlinear term only: masked, neither viscous term nor projection
    rr[0] = r[0];
    rr[1] = r[1];
    rr[2] = r[2];
    return;
  }
  if (!a.visc_if) {
#pragma unroll
    for (int c = 0; c < 3; ++c) r[c] = csub(r[c], cscale(uu[c], a.nu * k2));
  }
  if (k2 > 0.0 && keep) {
    const C dot = cadd(cadd(cscale(r[0], (double)ix), cscale(r[1], (double)iy)), cscale(r[2], (double)iz));
    const C factor = cscale(dot, 1.0 / k2);
    r[0] = csub(r[0], cscale(factor, (double)ix));
    r[1] = csub(r[1], cscale(factor, (double)iy));
    r[2] = csub(r[2], cscale(factor, (double)iz));
  } else {
    r[0] = r[1] = r[2] = czero<C>();
  }
  if (a.mode == 1) {
    rr[0] = r[0];
    rr[1] = r[1];
    rr[2] = r[2];
    return;
  }
  if (a.frozen) return;  // the solve's clock reached its horizon: u and g stay as they are
  if constexpr (sizeof(C) == 8) {
    if (a.ulo != nullptr) {
      // FP32 form with the compensated state: u = hi + lo updated and projected in FP64
      double2 U[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        gg[c] = load_g ? cadd(cscale(gg[c], (float)a.ga), r[c]) : r[c];
        U[c] = comp_decode(uu[c], lo[c]);
        U[c] = make_double2(U[c].x + a.ub * (double)gg[c].x, U[c].y + a.ub * (double)gg[c].y);
      }
      if (a.visc_if) {
        const double f = exp(-a.nu * k2 * a.if_tau);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          U[c] = make_double2(U[c].x * f, U[c].y * f);
          gg[c] = cscale(gg[c], (float)f);
        }
      }
      if (k2 > 0.0 && keep) {
        const double2 dot = make_double2((U[0].x * ix + U[1].x * iy) + U[2].x * iz,
                                         (U[0].y * ix + U[1].y * iy) + U[2].y * iz);
        const double2 factor = make_double2(dot.x * (1.0 / k2), dot.y * (1.0 / k2));
        const double kv[3] = {(double)ix, (double)iy, (double)iz};
#pragma unroll
        for (int c = 0; c < 3; ++c) uu[c] = comp_encode(make_double2(U[c].x - factor.x * kv[c],
                                                                     U[c].y - factor.y * kv[c]), &lo[c]);
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          uu[c] = czero<C>();
          lo[c] = 0;
        }
      }
      return;
    }
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    gg[c] = load_g ? cadd(cscale(gg[c], a.ga), r[c]) : r[c];
    uu[c] = cadd(uu[c], cscale(gg[c], a.ub));
  }
  if (a.visc_if) {
    // integrating factor to the next stage time, exponent in FP64 for either precision
    const double f = exp(-a.nu * k2 * a.if_tau);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uu[c] = cscale(uu[c], f);
      gg[c] = cscale(gg[c], f);
    }
  }
  if (k2 > 0.0 && keep) {
    const C dot = cadd(cadd(cscale(uu[0], (double)ix), cscale(uu[1], (double)iy)), cscale(uu[2], (double)iz));
    const C factor = cscale(dot, 1.0 / k2);
    uu[0] = csub(uu[0], cscale(factor, (double)ix));
    uu[1] = csub(uu[1], cscale(factor, (double)iy));
    uu[2] = csub(uu[2], cscale(factor, (double)iz));
  } else {
    uu[0] = uu[1] = uu[2] = czero<C>();
  }
}

template <int N, class C>
__global__ void __launch_bounds__(256)
k_sweep(const C* __restrict__ work, C* __restrict__ u, C* __restrict__ gbuf,
        C* __restrict__ rhs, const double* __restrict__ nyq_part, int nparts, const C* __restrict__ phase,
        SweepArgs a0, Geom g) {
  const SweepArgs a = resolve_step(a0);
  constexpr int NH = N / 2;
  const long long e = (long long)blockIdx.x * 256 + threadIdx.x;
  const long long total = (long long)N * N * NH;
  const bool load_g = a.stage > 0;
  if (e < total) {
    const long long row = e / NH;
    const int mx = (int)(e % NH);
    const int my = signed_mode((int)(row % N), N);
    const int mz = signed_mode((int)(row / N), N);
    const long long idx = row * g.pitch + mx;
    ModeIn<C> in;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      in.p0[p] = work[(long long)(2 * p) * g.field + idx];
      in.ps[p] = work[(long long)(2 * p + 1) * g.field + idx];
    }
    C uu[3], gg[3], rr[3];
    CompWord lo[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uu[c] = u[(long long)c * g.field + idx];
      gg[c] = load_g ? gbuf[(long long)c * g.field + idx] : czero<C>();
      if (a.ulo) lo[c] = a.ulo[(long long)c * g.field + idx];
    }
    sweep_mode(in, mx, my, mz, N, phase[mx + my + mz + 3 * N / 2], uu, gg, load_g, rr, a, lo);
    if (a.mode != 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) rhs[(long long)c * g.field + idx] = rr[c];
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u[(long long)c * g.field + idx] = uu[c];
        gbuf[(long long)c * g.field + idx] = gg[c];
        if (a.ulo) a.ulo[(long long)c * g.field + idx] = lo[c];
      }
    }
    // The plane mx = N/2 is outside the sphere except at (N/2,0,0): the reference's
    // masked RHS, g and projected u are zero there.  Row 0 is written below.
    if (mx == 0 && row != 0) {
      const long long inq = row * g.pitch + NH;
      const C zero = czero<C>();
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (a.mode != 0) {
          rhs[(long long)c * g.field + inq] = zero;
        } else {
          u[(long long)c * g.field + inq] = zero;
          gbuf[(long long)c * g.field + inq] = zero;
          if (a.ulo) a.ulo[(long long)c * g.field + inq] = 0u;
        }
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x < 32) {
    // the self-conjugate Nyquist mode (N/2, 0, 0), column nh of row (0, 0): warp 0 sums
    // the per-CTA plane sums (lane-strided, then a fixed shuffle tree: deterministic)
    double part[12];
#pragma unroll
    for (int f = 0; f < 12; ++f) {
      double acc = 0.0;
      for (int i = threadIdx.x; i < nparts; i += 32) acc += nyq_part[f * nparts + i];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      part[f] = acc;
    }
  if (threadIdx.x == 0) {
    ModeIn<C> in;
#pragma unroll
    for (int p = 0; p < 6; ++p) {
      in.p0[p] = cmk((real_of<C>)part[2 * p], real_of<C>(0));
      in.ps[p] = cmk((real_of<C>)part[2 * p + 1], real_of<C>(0));
    }
    const long long idx = NH;
    C uu[3], gg[3], rr[3];
    CompWord lo[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uu[c] = u[(long long)c * g.field + idx];
      gg[c] = load_g ? gbuf[(long long)c * g.field + idx] : czero<C>();
      if (a.ulo) lo[c] = a.ulo[(long long)c * g.field + idx];
    }
    sweep_mode(in, NH, 0, 0, N, phase[NH + 3 * N / 2], uu, gg, load_g, rr, a, lo);
    if (a.mode != 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) rhs[(long long)c * g.field + idx] = rr[c];
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        u[(long long)c * g.field + idx] = uu[c];
        gbuf[(long long)c * g.field + idx] = gg[c];
        if (a.ulo) a.ulo[(long long)c * g.field + idx] = lo[c];
      }
    }
  }
  }
}



// The self-conjugate mode (N/2, 0, 0) for the fused P5 path: one warp sums the x pass's
// per-CTA plane sums in a fixed order and runs the sweep on that single mode (column N/2
// of row 0, which no P5 tile touches).
template <int N, class C>
__global__ void __launch_bounds__(32) k_nyq_mode(C* __restrict__ u, C* __restrict__ gbuf,
                                                 C* __restrict__ rhs, const double* __restrict__ nyq_part,
                                                 int nparts, const C* __restrict__ phase, SweepArgs a0, Geom g) {
  const SweepArgs a = resolve_step(a0);
  constexpr int NH = N / 2;
  const int tid = threadIdx.x;
  const bool load_g = a.stage > 0;
  double part[12];
#pragma unroll
  for (int f = 0; f < 12; ++f) {
    double acc = 0.0;
    for (int i = tid; i < nparts; i += 32) acc += nyq_part[f * nparts + i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    part[f] = acc;
  }
  if (tid != 0) return;
  ModeIn<C> in;
#pragma unroll
  for (int p = 0; p < 6; ++p) {
    in.p0[p] = cmk((real_of<C>)part[2 * p], real_of<C>(0));
    in.ps[p] = cmk((real_of<C>)part[2 * p + 1], real_of<C>(0));
  }
  C uu[3], gg[3], rr[3];
  CompWord lo[3] = {0, 0, 0};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    uu[c] = u[(long long)c * g.field + NH];
    gg[c] = load_g ? gbuf[(long long)c * g.field + NH] : czero<C>();
    if (a.ulo) lo[c] = a.ulo[(long long)c * g.field + NH];
  }
  sweep_mode(in, NH, 0, 0, N, phase[NH + 3 * N / 2], uu, gg, load_g, rr, a, lo);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    if (a.mode != 0) {
      rhs[(long long)c * g.field + NH] = rr[c];
    } else {
      u[(long long)c * g.field + NH] = uu[c];
      gbuf[(long long)c * g.field + NH] = gg[c];
      if (a.ulo) a.ulo[(long long)c * g.field + NH] = lo[c];
    }
  }
}

// ------------------------------------------------------------------------------------
// Rotational form (selectable; the reference computes only the conservative form).
// omega_hat = i k x u_hat on every stored mode (the wavenumbers of the stored modes, index
// N/2 -> +N/2, as the conservative form's -i k uses them).
template <class C>
__global__ void k_omega_hat(const C* __restrict__ u, C* __restrict__ w, Geom g) {
  const long long total = (long long)g.n * g.n * (g.nh + 1);
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  using RT = real_of<C>;
  const long long row = e / (g.nh + 1);
  const int ix = (int)(e % (g.nh + 1));
  const RT kx = (RT)ix, ky = (RT)signed_mode((int)(row % g.n), g.n), kz = (RT)signed_mode((int)(row / g.n), g.n);
  const long long idx = row * g.pitch + ix;
  const C u0 = u[idx], u1 = u[g.field + idx], u2 = u[2 * g.field + idx];
  // i * (a) = (-a.y, a.x)
  auto i_times = [](RT ax, RT ay) { return cmk(-ay, ax); };
  w[idx] = i_times(ky * u2.x - kz * u1.x, ky * u2.y - kz * u1.y);
  w[g.field + idx] = i_times(kz * u0.x - kx * u2.x, kz * u0.y - kx * u2.y);
  w[2 * g.field + idx] = i_times(kx * u1.x - ky * u0.x, kx * u1.y - ky * u0.y);
}

// Rotational x pass, one row (y, z) per CTA.  Inputs after the inverse y/z passes: work
// fields 2c, 2c+1 = U_c, V_c (velocity on both grids), 6 + 2c, 7 + 2c = Omega_c, Psi_c
// (vorticity on both grids).  Inverse x of the 6 packed pairs, u x omega on both grids,
// forward x of the 3 packed components; outputs: work fields 2c, 2c+1 = A_c, B_c.
template <int N, class C>
__global__ void __launch_bounds__(nt_x<N>())
k_xpass_rot(C* __restrict__ work, const C* __restrict__ unyq, const C* __restrict__ wnyq,
            const C* __restrict__ phase, double scale, int nyq_scalar, const C* __restrict__ tw, Geom g) {
  constexpr int NT = nt_x<N>();
  constexpr int NH = N / 2;
  constexpr int RP = row_pitch(N);
  extern __shared__ __align__(16) unsigned char smraw_x[];
  C* smem = reinterpret_cast<C*>(smraw_x);
  C* s_tw = smem;
  C* seq = smem + N;  // 6 sequences of pitch RP
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const long long rbase = (long long)blockIdx.x * g.pitch;
  for (int e = tid; e < 6 * (NH + 1); e += NT) {
    const int q = e / (NH + 1), k = e % (NH + 1);
    const int c = q % 3, vort = q / 3;
    C A, B;
    if (k == NH && nyq_scalar) {
      // masked state: the plane mx = N/2 holds only (N/2,0,0), a constant after the y/z
      // inverse transforms (times the phase on the shifted grid)
      const C cn = cscale((vort ? wnyq : unyq)[(long long)c * g.field + NH], scale);
      A = cn;
      B = cmul(cn, phase[NH + 3 * N / 2]);
    } else {
      A = work[(long long)(6 * vort + 2 * c) * g.field + rbase + k];
      B = work[(long long)(6 * vort + 2 * c + 1) * g.field + rbase + k];
    }
    C zk, zm;
    pack_pair(A, B, k, NH, N, &zk, &zm);
    C* sq = seq + q * RP;
    sq[k + (k >> 3)] = zk;
    if (k != 0 && k != NH) sq[(N - k) + ((N - k) >> 3)] = zm;
  }
  __syncthreads();
  smem_fft<N, +1, 6, NT, RowTile<RP>>(seq, s_tw, tid);
  for (int x = tid; x < N; x += NT) {
    const int p = x + (x >> 3);
    C uu[3], ww[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      uu[c] = seq[c * RP + p];        // (u_c, u_c shifted)
      ww[c] = seq[(3 + c) * RP + p];  // (omega_c, omega_c shifted)
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int a = (c + 1) % 3, b = (c + 2) % 3;
      seq[c * RP + p] = cmk(uu[a].x * ww[b].x - uu[b].x * ww[a].x, uu[a].y * ww[b].y - uu[b].y * ww[a].y);
    }
  }
  __syncthreads();
  smem_fft<N, -1, 3, NT, RowTile<RP>>(seq, s_tw, tid);
  for (int e = tid; e < 3 * (NH + 1); e += NT) {
    const int c = e / (NH + 1), k = e % (NH + 1);
    const int km = (N - k) % N;
    C A, B;
    unpack_pair(seq[c * RP + k + (k >> 3)], seq[c * RP + km + (km >> 3)], &A, &B);
    work[(long long)(2 * c) * g.field + rbase + k] = A;
    work[(long long)(2 * c + 1) * g.field + rbase + k] = B;
  }
}

// Rotational k-space sweep: r_c = the dealiased, masked (u x omega)_c (no -i k), then the
// shared viscous / integrating-factor, Leray projection and RK3 update of finish_mode.
// The (N/2,0,0) mode takes its two-grid values from the plane sums of the 6 product fields.
template <int N, class C>
__global__ void __launch_bounds__(256)
k_sweep_rot(const C* __restrict__ work, C* __restrict__ u, C* __restrict__ gbuf, C* __restrict__ rhs,
            const double* __restrict__ nyq_sums, const C* __restrict__ phase, SweepArgs a0, Geom g) {
  const SweepArgs a = resolve_step(a0);
  constexpr int NH = N / 2;
  const long long e = (long long)blockIdx.x * 256 + threadIdx.x;
  const long long total = (long long)N * N * NH;
  const bool load_g = a.stage > 0;
  using RT = real_of<C>;
  auto update = [&](long long idx, int mx, int my, int mz, const C* A, const C* B, C ph) {
    const int m2 = mx * mx + my * my + mz * mz;
    const bool keep = 4LL * m2 <= (long long)N * N;
    C r[3], uu[3], gg[3], rr[3];
    CompWord lo[3] = {0, 0, 0};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      r[c] = pair_value(A[c], B[c], ph, keep, a.dealias);
      uu[c] = u[(long long)c * g.field + idx];
      gg[c] = load_g ? gbuf[(long long)c * g.field + idx] : czero<C>();
      if (a.ulo) lo[c] = a.ulo[(long long)c * g.field + idx];
    }
    finish_mode(r, mx, my, mz, N, uu, gg, load_g, rr, a, lo);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (a.mode != 0) {
        rhs[(long long)c * g.field + idx] = rr[c];
      } else {
        u[(long long)c * g.field + idx] = uu[c];
        gbuf[(long long)c * g.field + idx] = gg[c];
        if (a.ulo) a.ulo[(long long)c * g.field + idx] = lo[c];
      }
    }
  };
  if (e < total) {
    const long long row = e / NH;
    const int mx = (int)(e % NH);
    const int my = signed_mode((int)(row % N), N);
    const int mz = signed_mode((int)(row / N), N);
    const long long idx = row * g.pitch + mx;
    C A[3], B[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      A[c] = work[(long long)(2 * c) * g.field + idx];
      B[c] = work[(long long)(2 * c + 1) * g.field + idx];
    }
    update(idx, mx, my, mz, A, B, phase[mx + my + mz + 3 * N / 2]);
    if (mx == 0 && row != 0) {  // the plane mx = N/2 is zero off (N/2,0,0) after the mask
      const long long inq = row * g.pitch + NH;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        if (a.mode != 0) {
          rhs[(long long)c * g.field + inq] = czero<C>();
        } else {
          u[(long long)c * g.field + inq] = czero<C>();
          gbuf[(long long)c * g.field + inq] = czero<C>();
          if (a.ulo) a.ulo[(long long)c * g.field + inq] = 0u;
        }
      }
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    C A[3], B[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      A[c] = cmk((RT)nyq_sums[2 * c], RT(0));
      B[c] = cmk((RT)nyq_sums[2 * c + 1], RT(0));
    }
    update(NH, NH, 0, 0, A, B, phase[NH + 3 * N / 2]);
  }
}

// ------------------------------------------------------------------------------------
// P5 fused (N = 128, 256, 512): forward z pass of the 12 product fields and the whole
// k-space sweep in one persistent kernel, so the transformed products never return to HBM.
// A tile is (TW columns mx, one my, all mz); its 12 field tiles arrive one after another
// through TMA (double-buffered).  The z FFT leaves each thread 8 modes in registers:
//   P0 field of pair p -> parked in tensor memory;
//   Ps field of pair p -> combined with the parked P0 into the dealiased value, whose -i k
//                          contributions accumulate into r_x, r_y, r_z in tensor memory, in
//                          the reference's order (pairs 00 01 02 11 12 22);
//   after the 12th      -> viscous term, Leray projection, RK3 update and projection of u.
// Tensor memory per thread: 4 blocks of CW columns (P0, r_x, r_y, r_z).
template <int N>
constexpr uint32_t p5_cols() { return N == 512 ? 512u : (N == 256 ? 256u : 128u); }
template <int N>
constexpr int nt_p5() { return nt_tma<N>(); }

template <int N, class C>
__global__ void __launch_bounds__(nt_p5<N>(), tma_minb<N>())
k_p5(const __grid_constant__ CUtensorMap map, C* __restrict__ u, C* __restrict__ gbuf,
     C* __restrict__ rhs, const double* __restrict__ nyq_part, int nparts, const C* __restrict__ tw,
     const C* __restrict__ phase, SweepArgs a0, int ncb, const int* __restrict__ live, int nlive, Geom g,
     int* err) {
  const SweepArgs a = resolve_step(a0);
  constexpr int NT = nt_p5<N>();
  constexpr int BR = box_rows<N>();
  constexpr int NBOX = N / BR;
  constexpr int NH = N / 2;
  constexpr int TW = tile_cols<C>();
  constexpr uint32_t kTileBytes = 128u * N;
  constexpr uint32_t COLS = p5_cols<N>();
  using RO = LastStage<N, NT, TW>;
  constexpr int WPC = tmem_words<C>();  // tensor-memory words per complex value
  constexpr int MPT = RO::KB * RO::R;    // modes per thread
  constexpr int CW = WPC * MPT;          // tensor-memory words per field of modes
  static_assert(RO::R == 4 || RO::R == 8, "last radix moves through tensor memory");
  static_assert((NT / 32 + 3) / 4 * 4 * CW <= (int)COLS, "tensor memory budget");
  static_assert((TW * (N / RO::R)) % NT == 0, "every thread owns whole butterflies");
  extern __shared__ unsigned char smraw[];
  __shared__ int s_fail;
  __shared__ uint32_t s_tmem;
  const uint32_t pad = (128u - (smem_u32(smraw) & 127u)) & 127u;
  C* in0 = reinterpret_cast<C*>(smraw + pad);
  C* in1 = in0 + TW * N;
  C* W = in1 + TW * N;
  C* s_tw = W + TW * N;
  uint64_t* bars = reinterpret_cast<uint64_t*>(s_tw + N);
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int t = tid; t < N; t += NT) s_tw[t] = tw[t];
  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    s_fail = 0;
  }
  if (warp == 0) {
    tmem_alloc(&s_tmem, COLS);
    tmem_relinquish();
  }
  __syncthreads();
  const uint32_t tbase = s_tmem;
  // this thread's lane and columns: P0 park [0, CW), r_x, r_y, r_z at CW * (1 + c)
  const uint32_t tq = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)((warp >> 2) * 4 * CW);
  const bool load_g = a.stage > 0;

  // tiles (cb, my), index my * ncb + cb (at most N x (N/16 + 1): 32-bit); with a live list
  // only the listed ones
  const long long ntiles = live ? (long long)nlive : (long long)ncb * N;
  auto tile_of = [&](long long t, int& cb, int& my) {
    const int idx = live ? __ldg(&live[SNS_IDX(t, nlive)]) : (int)t;
    my = idx / ncb;
    cb = idx - my * ncb;
  };
  const long long mytiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const long long nunits = 12 * mytiles;
  auto issue = [&](long long ul, int b) {
    const long long t = blockIdx.x + (ul / 12) * gridDim.x;
    const int f = (int)(ul % 12);
    int cb, my;
    tile_of(t, cb, my);
    C* dst = b ? in1 : in0;
    mbar_arrive_expect_tx(&bars[b], kTileBytes);
#pragma unroll
    for (int k = 0; k < NBOX; ++k) tma_load_4d(dst + k * BR * TW, &map, &bars[b], cb * 2 * TW, my, k * BR, f);
  };
  if (tid == 0) {
    if (nunits > 0) issue(0, 0);
    if (nunits > 1) issue(1, 1);
  }
  for (long long ul = 0; ul < nunits; ++ul) {
    const int b = (int)(ul & 1);
    const uint32_t parity = (uint32_t)(ul >> 1) & 1u;
    if (tid == 0 && !mbar_wait_bounded(&bars[b], parity)) s_fail = 1;
    __syncthreads();
    if (s_fail) {
      if (tid == 0) {
        atomicExch(err, kErrTmaTimeout);
        (void)mbar_wait_bounded(&bars[b ^ 1], (uint32_t)((ul + 1) >> 1) & 1u);
      }
      if (warp == 0) tmem_dealloc(tbase, COLS);
      return;
    }
    (void)mbar_try_wait(&bars[b], parity);
    const C* IN = b ? in1 : in0;
    const long long t = blockIdx.x + (ul / 12) * gridDim.x;
    const int f = (int)(ul % 12);
    int cb, my;
    tile_of(t, cb, my);
    const int mx0 = cb * TW;
    // Each radix butterfly of the last stage hands its R modes to the sink: column
    // s = b % TW (b = tid + i*NT), z index (j/NS)*NS*R + j%NS + r*NS with j = b / TW; mode
    // q = i*R + r of this thread owns tensor-memory columns [WPC*q, WPC*(q + 1)) of every block.
    const int iy = signed_mode(my, N);
    const int p = f >> 1;
    const int ca = (p >= 3) + (p >= 5), cbp = p < 3 ? p : (p < 5 ? p - 2 : 2);
    auto sink = [&](int i, C* v) {
      constexpr int R = RO::R, NS = RO::NS;
      const int bb = tid + i * NT, s_ = bb % TW, j = bb / TW;
      const uint32_t col = (uint32_t)(WPC * R * i);
      // tensor-memory columns of this thread's blocks stay inside the allocation
      (void)SNS_IDX((warp >> 2) * 4 * CW + 4 * CW - 1, (long long)COLS);
      (void)SNS_IDX(col + WPC * R - 1, (long long)CW);
      if ((f & 1) == 0) {
        tmem_st<R>(tq + col, v);  // park P0 of this pair
        return;
      }
      const int ix = mx0 + s_;
      int izs[R];
      {
        C p0[R];
        tmem_ld<R>(tq + col, p0);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          izs[r] = signed_mode((j / NS) * NS * R + (j % NS) + r * NS, N);
          const bool keep = 4LL * (ix * ix + iy * iy + izs[r] * izs[r]) <= (long long)N * N;
          v[r] = pair_value(p0[r], v[r], __ldg(&phase[SNS_IDX(ix + iy + izs[r] + 3 * N / 2, 3 * N + 1)]), keep,
                            a.dealias);
        }
      }
      // r_a += -i k_b value; r_b += -i k_a value (a != b); the first touch starts the sum
#pragma unroll
      for (int side = 0; side < 2; ++side) {
        if (side == 1 && ca == cbp) break;
        const int dst = side == 0 ? ca : cbp, kc = side == 0 ? cbp : ca;
        const bool first = side == 0 ? (p == 0) : (p == 1 || p == 2);  // r_x at 00, r_y at 01, r_z at 02
        const uint32_t ta = tq + (uint32_t)(CW * (1 + dst)) + col;
        C r[R];
        if (!first) tmem_ld<R>(ta, r);
#pragma unroll
        for (int rr = 0; rr < R; ++rr) {
          const int kk = kc == 0 ? ix : (kc == 1 ? iy : izs[rr]);
          const C c = minus_i_k(v[rr], kk);
          r[rr] = first ? c : cadd(r[rr], c);
        }
        tmem_st<R>(ta, r);
      }
    };
    tile_fft_sink<N, -1, NT, TW>([&](int s_, int e_) { return IN[SNS_IDX(e_ * TW + s_, TW * N)]; }, W, s_tw, tid,
                                 sink);
    tmem_wait_st();
    __syncthreads();  // IN[b] and W are free again
    if (tid == 0 && ul + 2 < nunits) issue(ul + 2, b);
    auto mode_s = [&](int q) { return (tid + (q / RO::R) * NT) % TW; };
    auto mode_e = [&](int q) {
      const int j = (tid + (q / RO::R) * NT) / TW, r = q % RO::R;
      return (j / RO::NS) * RO::NS * RO::R + (j % RO::NS) + r * RO::NS;
    };
    if (f == 11) {
      // Two-deep software pipeline over this thread's modes: the u, g loads of mode q + 1
      // are in flight while mode q is combined and stored (different modes, no aliasing).
      C uu_n[3], gg_n[3];
      CompWord lo_n[3] = {0, 0, 0};
      auto load_mode = [&](int q, C* uu, C* gg, CompWord* lo) {
        const long long idx = SNS_IDX(((long long)mode_e(q) * N + my) * g.pitch + mx0 + mode_s(q), g.field);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          uu[c] = u[(long long)c * g.field + idx];
          gg[c] = load_g ? gbuf[(long long)c * g.field + idx] : czero<C>();
          if (a.ulo) lo[c] = a.ulo[(long long)c * g.field + idx];
        }
      };
      load_mode(0, uu_n, gg_n, lo_n);
#pragma unroll 1
      for (int q = 0; q < MPT; ++q) {
        C uu[3], gg[3], rr[3];
        CompWord lo[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          uu[c] = uu_n[c];
          gg[c] = gg_n[c];
          lo[c] = lo_n[c];
        }
        if (q + 1 < MPT) load_mode(q + 1, uu_n, gg_n, lo_n);
        C r3[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) r3[c] = tmem_ld1<C>(tq + CW * (1 + c) + WPC * q);
        const int ix = mx0 + mode_s(q);
        if (ix >= NH) continue;
        const int ez = mode_e(q);
        const int iz = signed_mode(ez, N);
        const long long row = (long long)ez * N + my;
        const long long idx = SNS_IDX(row * g.pitch + ix, g.field);
        finish_mode(r3, ix, iy, iz, N, uu, gg, load_g, rr, a, lo);
        const bool nyq_zero = ix == 0 && row != 0;  // plane mx = N/2 is zero off (N/2,0,0)
        const long long inq = SNS_IDX(row * g.pitch + NH, g.field);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (a.mode != 0) {
            rhs[(long long)c * g.field + idx] = rr[c];
            if (nyq_zero) rhs[(long long)c * g.field + inq] = czero<C>();
          } else {
            u[(long long)c * g.field + idx] = uu[c];
            gbuf[(long long)c * g.field + idx] = gg[c];
            if (a.ulo) a.ulo[(long long)c * g.field + idx] = lo[c];
            if (nyq_zero) {
              u[(long long)c * g.field + inq] = czero<C>();
              gbuf[(long long)c * g.field + inq] = czero<C>();
              if (a.ulo) a.ulo[(long long)c * g.field + inq] = 0u;
            }
          }
        }
      }
    }
  }
  __syncthreads();
  if (warp == 0) tmem_dealloc(tbase, COLS);
}

// ------------------------------------------------------------------------------------
// Generic x transforms (FFT-backend contract and initialisation).  Two rows of one field
// share a complex FFT.  grid (N*N/2, nf).
template <int N, class C>
__global__ void __launch_bounds__(nt_x<N>())
k_xpass_r2c(const double* __restrict__ in, C* __restrict__ out, const C* __restrict__ tw, Geom g) {
  constexpr int NT = nt_x<N>();
  constexpr int NH = N / 2;
  constexpr int RP = row_pitch(N);
  extern __shared__ __align__(16) unsigned char smraw_x[];
  C* smem = reinterpret_cast<C*>(smraw_x);
  C* s_tw = smem;
  C* seq = smem + N;
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const long long r0 = 2LL * blockIdx.x;
  const double* fin = in + (long long)blockIdx.y * N * N * N;
  C* fout = out + (long long)blockIdx.y * g.field;
  using RT = real_of<C>;
  for (int x = tid; x < N; x += NT) seq[x + (x >> 3)] = cmk((RT)fin[r0 * N + x], (RT)fin[(r0 + 1) * N + x]);
  __syncthreads();
  smem_fft<N, -1, 1, NT, RowTile<RP>>(seq, s_tw, tid);
  for (int k = tid; k <= NH; k += NT) {
    const int km = (N - k) % N;
    C A, B;
    unpack_pair(seq[k + (k >> 3)], seq[km + (km >> 3)], &A, &B);
    fout[r0 * g.pitch + k] = A;
    fout[(r0 + 1) * g.pitch + k] = B;
  }
}

template <int N, class C>
__global__ void __launch_bounds__(nt_x<N>())
k_xpass_c2r(const C* __restrict__ in, double* __restrict__ out, const C* __restrict__ tw, Geom g) {
  constexpr int NT = nt_x<N>();
  constexpr int NH = N / 2;
  constexpr int RP = row_pitch(N);
  extern __shared__ __align__(16) unsigned char smraw_x[];
  C* smem = reinterpret_cast<C*>(smraw_x);
  C* s_tw = smem;
  C* seq = smem + N;
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const long long r0 = 2LL * blockIdx.x;
  const C* fin = in + (long long)blockIdx.y * g.field;
  double* fout = out + (long long)blockIdx.y * N * N * N;
  for (int k = tid; k <= NH; k += NT) {
    C zk, zm;
    pack_pair(fin[r0 * g.pitch + k], fin[(r0 + 1) * g.pitch + k], k, NH, N, &zk, &zm);
    seq[k + (k >> 3)] = zk;
    if (k != 0 && k != NH) seq[(N - k) + ((N - k) >> 3)] = zm;
  }
  __syncthreads();
  smem_fft<N, +1, 1, NT, RowTile<RP>>(seq, s_tw, tid);
  for (int x = tid; x < N; x += NT) {
    const C v = seq[x + (x >> 3)];
    fout[r0 * N + x] = v.x;
    fout[(r0 + 1) * N + x] = v.y;
  }
}

// Energy / vmax partials of the physical velocity (work fields 0,1,2 after the inverse
// z and y passes of u_hat without phase shift).  One row per CTA.
template <int N, class C>
__global__ void __launch_bounds__(nt_x<N>())
k_xpass_diag(const C* __restrict__ work, const C* __restrict__ unyq, double scale, int nyq_scalar,
             double* __restrict__ partials, const C* __restrict__ tw, Geom g) {
  constexpr int NT = nt_x<N>();
  constexpr int NH = N / 2;
  constexpr int RP = row_pitch(N);
  extern __shared__ __align__(16) unsigned char smraw_x[];
  C* smem = reinterpret_cast<C*>(smraw_x);
  C* s_tw = smem;
  C* seq = smem + N;  // 2 sequences: u0 + i u1, u2
  __shared__ double red[2 * (NT / 32)];
  const int tid = threadIdx.x;
  load_twiddles<N>(s_tw, tw, tid, NT);
  const long long row = blockIdx.x;
  const long long rbase = row * g.pitch;
  for (int k = tid; k <= NH; k += NT) {
    C U[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      if (k == NH && nyq_scalar) U[c] = cscale(unyq[(long long)c * g.field + NH], scale);
      else U[c] = work[(long long)c * g.field + rbase + k];
    }
    C zk, zm;
    pack_pair(U[0], U[1], k, NH, N, &zk, &zm);
    seq[k + (k >> 3)] = zk;
    if (k != 0 && k != NH) seq[(N - k) + ((N - k) >> 3)] = zm;
    pack_pair(U[2], czero<C>(), k, NH, N, &zk, &zm);
    seq[RP + k + (k >> 3)] = zk;
    if (k != 0 && k != NH) seq[RP + (N - k) + ((N - k) >> 3)] = zm;
  }
  __syncthreads();
  smem_fft<N, +1, 2, NT, RowTile<RP>>(seq, s_tw, tid);
  double esum = 0.0, vmax2 = 0.0;
  for (int x = tid; x < N; x += NT) {
    const int p = x + (x >> 3);
    const C a = seq[p], b = seq[RP + p];
    const double ax = a.x, ay = a.y, bx = b.x;
    const double s2 = ax * ax + ay * ay + bx * bx;
    esum += 0.5 * s2;
    vmax2 = fmax(vmax2, s2);
  }
  block_sum_max<NT>(esum, vmax2, red);
  if (tid == 0) {
    partials[2 * row] = esum;
    partials[2 * row + 1] = vmax2;
  }
}

// ------------------------------------------------------------------------------------
// Size-independent kernels.

// Taylor-Green field at cell centres (ava_taylor_green_impl.hpp:805-812), x fastest.
__global__ void k_tgv_init(double* __restrict__ phys, int n) {
  const long long np = (long long)n * n * n;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= np) return;
  constexpr double kPi = 3.141592653589793238462643383279502884;
  const int ix = (int)(id % n), iy = (int)((id / n) % n), iz = (int)(id / ((long long)n * n));
  const double x = ((double)ix + 0.5) * 2.0 * kPi / (double)n;
  const double y = ((double)iy + 0.5) * 2.0 * kPi / (double)n;
  const double z = ((double)iz + 0.5) * 2.0 * kPi / (double)n;
  phys[id] = sin(x) * cos(y) * cos(z);
  phys[np + id] = -cos(x) * sin(y) * cos(z);
  phys[2 * np + id] = 0.0;
}

// project_truncate over every stored mode, Nyquist column included (:825-844).
template <class C>
__global__ void k_project_truncate(C* __restrict__ u, Geom g) {
  const long long total = (long long)g.n * g.n * (g.nh + 1);
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const long long row = e / (g.nh + 1);
  const int ix = (int)(e % (g.nh + 1));
  const int iy = signed_mode((int)(row % g.n), g.n);
  const int iz = signed_mode((int)(row / g.n), g.n);
  const long long idx = row * g.pitch + ix;
  const int m2 = ix * ix + iy * iy + iz * iz;
  const bool keep = 4LL * m2 <= (long long)g.n * g.n;
  const double k2 = (double)m2;
  C ux = u[idx], uy = u[g.field + idx], uz = u[2 * g.field + idx];
  if (k2 > 0.0 && keep) {
    const C dot = cadd(cadd(cscale(ux, (double)ix), cscale(uy, (double)iy)), cscale(uz, (double)iz));
    const C factor = cscale(dot, 1.0 / k2);
    ux = csub(ux, cscale(factor, (double)ix));
    uy = csub(uy, cscale(factor, (double)iy));
    uz = csub(uz, cscale(factor, (double)iz));
  } else {
    ux = uy = uz = czero<C>();
  }
  u[idx] = ux;
  u[g.field + idx] = uy;
  u[2 * g.field + idx] = uz;
}

template <class C>
__global__ void k_add_sparse(C* __restrict__ u, const long long* __restrict__ idx,
                             const double2* __restrict__ val, int count) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const long long at = idx[i];
  using RT = real_of<C>;
  u[at] = cadd(u[at], cmk((RT)val[i].x, (RT)val[i].y));
}

// half -> reference full layout (mx < 0 from the conjugate mirror), widened to double.
__device__ __forceinline__ double2 widen(double2 v) { return v; }
__device__ __forceinline__ double2 widen(float2 v) { return make_double2(v.x, v.y); }

template <class C>
__device__ __forceinline__ double2 widen_comp(const C* half, const CompWord* lo, long long i) {
  if constexpr (sizeof(C) == 8) {
    if (lo) return comp_decode(half[i], lo[i]);
  }
  return widen(half[i]);
}

template <class C>
__global__ void k_half_to_full(const C* __restrict__ half, double2* __restrict__ full, Geom g,
                               const CompWord* __restrict__ lo) {
  const long long n = g.n;
  const long long total = n * n * n;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= total) return;
  const int x = (int)(id % n);
  const long long y = (id / n) % n, z = id / (n * n);
  if (x <= g.nh) {
    full[id] = widen_comp(half, lo, (z * n + y) * g.pitch + x);
  } else {
    const long long ym = (n - y) % n, zm = (n - z) % n;
    full[id] = cconj(widen_comp(half, lo, (zm * n + ym) * g.pitch + (n - x)));
  }
}

// reference full layout -> half; with hermitian_part the Hermitian part
// (c_m + conj(c_-m))/2 is stored, so a c2r of the result equals Re(IDFT(c)).
template <class C>
__global__ void k_full_to_half(const double2* __restrict__ full, C* __restrict__ half, int hermitian_part,
                               long long src_pitch, Geom g, CompWord* __restrict__ lo) {
  const long long n = g.n;
  const long long total = n * n * (g.nh + 1);
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= total) return;
  const long long row = e / (g.nh + 1);
  const int x = (int)(e % (g.nh + 1));
  const long long y = row % n, z = row / n;
  double2 v = full[row * src_pitch + x];  // src_pitch n: the full layout; nh + 1: its left half
  if (hermitian_part) {  // (full layout only)
    const long long ym = (n - y) % n, zm = (n - z) % n, xm = (n - x) % n;
    const double2 w = full[(zm * n + ym) * n + xm];
    v = make_double2(0.5 * (v.x + w.x), 0.5 * (v.y - w.y));
  }
  if constexpr (sizeof(C) == 8) {
    if (lo) {  // FP32 form, compensated: the remainder the FP32 value drops goes to lo
      half[row * g.pitch + x] = comp_encode(v, &lo[row * g.pitch + x]);
      return;
    }
  }
  using RT = real_of<C>;
  half[row * g.pitch + x] = cmk((RT)v.x, (RT)v.y);
}

// Parseval enstrophy and max spectral divergence of the (masked) state, in FP64 for
// either storage precision.
// Enstrophy = 0.5/N^6 * sum_m |H(omega_hat)_m|^2 over the full spectrum, with
// omega_hat = i k x u_hat as the reference forms it (:1147-1157).  Planes mx = 0 and
// mx = N/2 are their own x-mirror: weight 1 and the in-plane Hermitian part; other
// columns stand for themselves and their conjugate mirror: weight 2.
template <class C>
__device__ __forceinline__ void omega_hat(const C* u, long long field, long long idx, int ix, int iy, int iz,
                                          double2 w[3]) {
  const double2 u0 = widen(u[idx]), u1 = widen(u[field + idx]), u2 = widen(u[2 * field + idx]);
  const double rx = ix, ry = iy, rz = iz;
  w[0] = make_double2(-(ry * u2.y - rz * u1.y), ry * u2.x - rz * u1.x);
  w[1] = make_double2(-(rz * u0.y - rx * u2.y), rz * u0.x - rx * u2.x);
  w[2] = make_double2(-(rx * u1.y - ry * u0.y), rx * u1.x - ry * u0.x);
}

template <class C>
__global__ void __launch_bounds__(256) k_spectral_diag(const C* __restrict__ u, double* __restrict__ partials,
                                                       Geom g) {
  __shared__ double red_s[256];
  __shared__ double red_m[256];
  const long long total = (long long)g.n * g.n * (g.nh + 1);
  double s = 0.0, m = 0.0;
  for (long long e = (long long)blockIdx.x * 256 + threadIdx.x; e < total; e += (long long)gridDim.x * 256) {
    const long long row = e / (g.nh + 1);
    const int ix = (int)(e % (g.nh + 1));
    const int yi = (int)(row % g.n), zi = (int)(row / g.n);
    const int iy = signed_mode(yi, g.n), iz = signed_mode(zi, g.n);
    const long long idx = row * g.pitch + ix;
    double2 w[3];
    omega_hat(u, g.field, idx, ix, iy, iz, w);
    double contrib;
    if (ix == 0 || ix == g.nh) {
      const int ym = (g.n - yi) % g.n, zm = (g.n - zi) % g.n;
      const long long idm = ((long long)zm * g.n + ym) * g.pitch + ix;
      double2 wm[3];
      omega_hat(u, g.field, idm, ix, signed_mode(ym, g.n), signed_mode(zm, g.n), wm);
      contrib = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double hx = 0.5 * (w[c].x + wm[c].x), hy = 0.5 * (w[c].y - wm[c].y);
        contrib += hx * hx + hy * hy;
      }
    } else if (yi == g.n / 2 || zi == g.n / 2) {
      // mirror -m is not stored; its value is conj(u_m) but its wavenumber keeps +N/2 on the
      // Nyquist axis, so omega_hat(-m) is not conj(omega_hat(m)): form H explicitly.
      const int my2 = yi == g.n / 2 ? iy : -iy, mz2 = zi == g.n / 2 ? iz : -iz;
      const double2 u0 = widen(u[idx]), u1 = widen(u[g.field + idx]), u2 = widen(u[2 * g.field + idx]);
      const double2 c0 = cconj(u0), c1 = cconj(u1), c2 = cconj(u2);
      const double rx = -ix, ry = my2, rz = mz2;
      double2 wm[3];
      wm[0] = cmk(-(ry * c2.y - rz * c1.y), ry * c2.x - rz * c1.x);
      wm[1] = cmk(-(rz * c0.y - rx * c2.y), rz * c0.x - rx * c2.x);
      wm[2] = cmk(-(rx * c1.y - ry * c0.y), rx * c1.x - ry * c0.x);
      contrib = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double hx = 0.5 * (w[c].x + wm[c].x), hy = 0.5 * (w[c].y - wm[c].y);
        contrib += 2.0 * (hx * hx + hy * hy);
      }
      const double2 dm = cadd(cadd(cscale(c0, rx), cscale(c1, ry)), cscale(c2, rz));
      m = fmax(m, sqrt(dm.x * dm.x + dm.y * dm.y));
    } else {
      contrib = 0.0;
#pragma unroll
      for (int c = 0; c < 3; ++c) contrib += 2.0 * (w[c].x * w[c].x + w[c].y * w[c].y);
    }
    s += contrib;
    const double2 u0 = widen(u[idx]), u1 = widen(u[g.field + idx]), u2 = widen(u[2 * g.field + idx]);
    const double2 div = cadd(cadd(cscale(u0, (double)ix), cscale(u1, (double)iy)), cscale(u2, (double)iz));
    m = fmax(m, sqrt(div.x * div.x + div.y * div.y));
  }
  red_s[threadIdx.x] = s;
  red_m[threadIdx.x] = m;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      red_s[threadIdx.x] += red_s[threadIdx.x + o];
      red_m[threadIdx.x] = fmax(red_m[threadIdx.x], red_m[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = red_s[0];
    partials[2 * blockIdx.x + 1] = red_m[0];
  }
}

// Fixed-order reduction of `count` partials at stride `stride` (one CTA).
// One CTA of 1024 threads; four independent loads in flight per thread (the partials are
// read once, a few MB at most), then a fixed-order tree: the result does not depend on timing.
__global__ void __launch_bounds__(1024) k_reduce(const double* __restrict__ partials, int count, int stride,
                                                 int op_max, double* __restrict__ out) {
  __shared__ double red[1024];
  const int tid = threadIdx.x;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i0 = tid; i0 < count; i0 += 4 * 1024) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * 1024;
      if (i < count) {
        const double v = partials[(long long)i * stride];
        s[u] = op_max ? fmax(s[u], v) : s[u] + v;
      }
    }
  }
  red[tid] = op_max ? fmax(fmax(s[0], s[1]), fmax(s[2], s[3])) : (s[0] + s[1]) + (s[2] + s[3]);
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (tid < o) red[tid] = op_max ? fmax(red[tid], red[tid + o]) : red[tid] + red[tid + o];
    __syncthreads();
  }
  if (tid == 0) *out = red[0];
}

// ------------------------------------------------------------------------------------
// Host launchers.
template <class K>
static void set_smem(K kernel, size_t bytes) {
  if (bytes > 48 * 1024) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    // prefer the largest shared-memory carveout so the occupancy the launch shapes are
    // computed from (and get) is bounded by the real budget, not a smaller default split
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, (int)cudaSharedmemCarveoutMaxShared);
  }
}

template <int N, class C>
struct Launch {
  static constexpr int kT = tile_cols<C>();
  static constexpr size_t yz_smem() { return (size_t)(N + kT * N) * sizeof(C); }
  static constexpr size_t x_smem(int nseq) { return (size_t)(N + nseq * row_pitch(N)) * sizeof(C); }
  static C* F(void* p) { return static_cast<C*>(p); }
  static const C* F(const void* p) { return static_cast<const C*>(p); }

  static void zpass_inv_phase(const void* u, void* work, const void* tw, const void* phase, double scale,
                              int ntiles, Geom g, cudaStream_t st) {
    dim3 grid(ntiles, N, 3);
    k_zpass_inv_phase<N, C><<<grid, nt_yz<N>(), yz_smem(), st>>>(F(u), F(work), F(tw), F(phase), scale, g);
  }
  static void ypass(void* f, int nf, int dir, int ntiles, const void* tw, Geom g, cudaStream_t st) {
    dim3 grid(ntiles, N, nf);
    if (dir < 0) {
      k_ypass<N, -1, C><<<grid, nt_yz<N>(), yz_smem(), st>>>(F(f), F(tw), g);
    } else {
      k_ypass<N, +1, C><<<grid, nt_yz<N>(), yz_smem(), st>>>(F(f), F(tw), g);
    }
  }
  static void zpass(const void* src, void* dst, int nf, int dir, int ntiles, double scale, const void* tw, Geom g,
                    cudaStream_t st) {
    dim3 grid(ntiles, N, nf);
    if (dir < 0) {
      k_zpass<N, -1, C><<<grid, nt_yz<N>(), yz_smem(), st>>>(F(src), F(dst), scale, F(tw), g);
    } else {
      k_zpass<N, +1, C><<<grid, nt_yz<N>(), yz_smem(), st>>>(F(src), F(dst), scale, F(tw), g);
    }
  }
  static void xpass_products(void* work, const void* unyq, const void* phase, double scale, int nyq_scalar,
                             double* partials, const void* tw, Geom g, cudaStream_t st) {
    k_xpass_products<N, C><<<N * N, nt_x<N>(), x_smem(6), st>>>(F(work), F(unyq), F(phase), scale, nyq_scalar,
                                                                  partials, F(tw), g);
  }
  static void nyq_reduce(const void* work, double* sums, Geom g, cudaStream_t st) {
    k_nyq_reduce<C><<<12, 256, 0, st>>>(F(work), sums, g);
  }
  static void sweep(const void* work, void* u, void* gbuf, void* rhs, const double* nyq_part, int nparts,
                    const void* phase, SweepArgs a, Geom g, cudaStream_t st) {
    const long long total = (long long)N * N * (N / 2);
    k_sweep<N, C><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(F(work), F(u), F(gbuf), F(rhs), nyq_part, nparts,
                                                                   F(phase), a, g);
  }
  static void xpass2(void* work, const void* unyq, const void* phase, double scale, int nyq_scalar, double* nyq_part,
                     const void* tw2, Geom g, int grid, int* err, cudaStream_t st) {
    if constexpr ((N == 128 || N == 256 || N == 512) && std::is_same_v<C, float2>) {
      k_xpass_w<N><<<grid, 32 * XW<N>::WARPS, XW<N>::smem, st>>>(F(work), F(unyq), F(phase), scale, nyq_scalar,
                                                                 nyq_part, F(tw2), g, err);
    } else if constexpr (N == 256 || N == 512) {
      k_xpass2<N, C><<<grid, XP<N, C>::NT, XP<N, C>::smem, st>>>(F(work), F(unyq), F(phase), scale, nyq_scalar,
                                                                  nyq_part, F(tw2), g, err);
    }
  }
  static void p5(const CUtensorMap& map, void* u, void* gbuf, void* rhs, const double* nyq_part, int nparts,
                 const void* tw, const void* phase, SweepArgs a, int ncb, const int* live, int nlive, Geom g,
                 int grid, int* err, cudaStream_t st) {
    if constexpr (N == 128 || N == 256 || N == 512) {
      k_nyq_mode<N, C><<<1, 32, 0, st>>>(F(u), F(gbuf), F(rhs), nyq_part, nparts, F(phase), a, g);
      k_p5<N, C><<<grid, nt_p5<N>(), tma_smem<N, C>(), st>>>(map, F(u), F(gbuf), F(rhs), nyq_part, nparts, F(tw),
                                                              F(phase), a, ncb, live, nlive, g, err);
    }
  }
  // Persistent grid of the fused P5 (0: this size runs forward z + sweep as two kernels).
  // The runtime's occupancy query reports one CTA per SM for this tensor-memory kernel
  // whatever its allocation, so residency is computed from the kernel's own limits: shared
  // memory, registers, threads, and its tensor-memory columns (512 per SM).
  static int p5_grid(int nsm) {
    if constexpr (N == 128 || N == 256 || N == 512) {
      int dev = 0, smem_sm = 0, smem_rsv = 0, regs_sm = 0, thr_sm = 0;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
      cudaDeviceGetAttribute(&smem_rsv, cudaDevAttrReservedSharedMemoryPerBlock, dev);
      cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev);
      cudaDeviceGetAttribute(&thr_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev);
      cudaFuncAttributes fa{};
      cudaFuncGetAttributes(&fa, k_p5<N, C>);
      const long long smem_cta = (long long)tma_smem<N, C>() + fa.sharedSizeBytes + smem_rsv;
      const long long regs_cta = (long long)((fa.numRegs + 7) / 8 * 8) * nt_p5<N>();
      int nb = 512 / (int)p5_cols<N>();
      if (smem_cta > 0) nb = (int)std::min<long long>(nb, smem_sm / smem_cta);
      if (regs_cta > 0) nb = (int)std::min<long long>(nb, regs_sm / regs_cta);
      nb = std::min(nb, thr_sm / nt_p5<N>());
      return nsm * (nb < 1 ? 1 : nb);
    } else {
      (void)nsm;
      return 0;
    }
  }
  // Persistent grid of the two-stage x pass (0: this size uses the generic x pass).
  static int xpass2_grid(int nsm) {
    if constexpr ((N == 128 || N == 256 || N == 512) && std::is_same_v<C, float2>) {
      int nb = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_xpass_w<N>, 32 * XW<N>::WARPS, XW<N>::smem);
      // every warp owns row groups: no CTA beyond one per XW::WARPS row groups
      const long long ncta = ((long long)N * N / XW<N>::R + XW<N>::WARPS - 1) / XW<N>::WARPS;
      long long grid = (long long)nsm * (nb > 0 ? nb : 1);
      return (int)(grid < ncta ? grid : ncta);
    } else if constexpr (N == 256 || N == 512) {
      int nb = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_xpass2<N, C>, XP<N, C>::NT, XP<N, C>::smem);
      const long long niter = (long long)N * N / XP<N, C>::ROWS;
      long long grid = (long long)nsm * (nb > 0 ? nb : 1);
      return (int)(grid < niter ? grid : niter);
    } else {
      (void)nsm;
      return 0;
    }
  }
  // physical energy / vmax^2 per row: the warp-per-row kernel where it exists (FP32, N = 128,
  // 256, 512; grid as the x pass's), else the generic one-row-per-CTA kernel
  static int xpass_diag2(const void* work, const void* unyq, double scale, int nyq_scalar, double* partials,
                         const void* tw, const void* tw2, Geom g, int grid, int* err, cudaStream_t st) {
    if constexpr ((N == 128 || N == 256 || N == 512) && std::is_same_v<C, float2>) {
      if (grid > 0) {
        k_xpass_w<N, true><<<grid, 32 * XW<N>::WARPS, XW<N>::smem, st>>>(
            static_cast<float2*>(const_cast<void*>(work)), F(unyq), nullptr, scale, nyq_scalar, partials, F(tw2), g,
            err);
        return grid;  // one (energy, vmax^2) pair per CTA
      }
    }
    (void)tw2;
    (void)grid;
    (void)err;
    xpass_diag(work, unyq, scale, nyq_scalar, partials, tw, g, st);
    return N * N;  // one pair per row
  }
  static void omega_hat(const void* u, void* w, Geom g, cudaStream_t st) {
    const long long total = (long long)N * N * (N / 2 + 1);
    k_omega_hat<C><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(F(u), F(w), g);
  }
  static void xpass_rot(void* work, const void* unyq, const void* wnyq, const void* phase, double scale,
                        int nyq_scalar, const void* tw, Geom g, cudaStream_t st) {
    k_xpass_rot<N, C><<<N * N, nt_x<N>(), x_smem(6), st>>>(F(work), F(unyq), F(wnyq), F(phase), scale, nyq_scalar,
                                                           F(tw), g);
  }
  static void sweep_rot(const void* work, void* u, void* gbuf, void* rhs, const double* nyq_sums, const void* phase,
                        SweepArgs a, Geom g, cudaStream_t st) {
    const long long total = (long long)N * N * (N / 2);
    k_sweep_rot<N, C><<<(unsigned)((total + 255) / 256), 256, 0, st>>>(F(work), F(u), F(gbuf), F(rhs), nyq_sums,
                                                                       F(phase), a, g);
  }
  static void xpass_r2c(const double* in, void* out, int nf, const void* tw, Geom g, cudaStream_t st) {
    k_xpass_r2c<N, C><<<dim3(N * N / 2, nf), nt_x<N>(), x_smem(1), st>>>(in, F(out), F(tw), g);
  }
  static void xpass_c2r(const void* in, double* out, int nf, const void* tw, Geom g, cudaStream_t st) {
    k_xpass_c2r<N, C><<<dim3(N * N / 2, nf), nt_x<N>(), x_smem(1), st>>>(F(in), out, F(tw), g);
  }
  static void xpass_diag(const void* work, const void* unyq, double scale, int nyq_scalar, double* partials,
                         const void* tw, Geom g, cudaStream_t st) {
    k_xpass_diag<N, C><<<N * N, nt_x<N>(), x_smem(2), st>>>(F(work), F(unyq), scale, nyq_scalar, partials, F(tw), g);
  }
  template <int AXIS, int DIR, int VARIANT>
  static void yz_tma_launch(const CUtensorMap& map, TmaArgs a, const void* tw, const void* phase, Geom g, int grid,
                            cudaStream_t st) {
    k_yz_tma<N, AXIS, DIR, VARIANT, C><<<grid, nt_tma<N>(), tma_smem<N, C>(), st>>>(map, a, F(tw), F(phase), g);
  }
  static void yz_tma(const CUtensorMap& map, int axis, int dir, int variant, TmaArgs a, const void* tw,
                     const void* phase, Geom g, int grid, cudaStream_t st) {
    if (variant == 1) yz_tma_launch<2, +1, 1>(map, a, tw, phase, g, grid, st);
    else if (axis == 1 && dir < 0) yz_tma_launch<1, -1, 0>(map, a, tw, phase, g, grid, st);
    else if (axis == 1) yz_tma_launch<1, +1, 0>(map, a, tw, phase, g, grid, st);
    else if (dir < 0) yz_tma_launch<2, -1, 0>(map, a, tw, phase, g, grid, st);
    else yz_tma_launch<2, +1, 0>(map, a, tw, phase, g, grid, st);
  }
  // Resident CTAs per SM of the TMA pass (all its instantiations share one footprint).
  static int tma_blocks_per_sm() {
    int lo = 1 << 30;
    auto occ = [&](auto kernel) {
      int nb = 0;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, nt_tma<N>(), tma_smem<N, C>());
      lo = nb < lo ? nb : lo;
    };
    occ(k_yz_tma<N, 2, +1, 1, C>);
    occ(k_yz_tma<N, 1, -1, 0, C>);
    occ(k_yz_tma<N, 1, +1, 0, C>);
    occ(k_yz_tma<N, 2, -1, 0, C>);
    occ(k_yz_tma<N, 2, +1, 0, C>);
    return lo > 0 && lo < (1 << 30) ? lo : 1;
  }
  // Opt every kernel of this size into its dynamic shared memory (once per process).
  static void init() {
    if constexpr ((N == 128 || N == 256 || N == 512) && std::is_same_v<C, float2>) {
      set_smem(k_xpass_w<N>, XW<N>::smem);
      set_smem(k_xpass_w<N, true>, XW<N>::smem);
    }
    else if constexpr (N == 256 || N == 512) set_smem(k_xpass2<N, C>, XP<N, C>::smem);
    if constexpr (N == 128 || N == 256 || N == 512) set_smem(k_p5<N, C>, tma_smem<N, C>());
    set_smem(k_yz_tma<N, 2, +1, 1, C>, tma_smem<N, C>());
    set_smem(k_yz_tma<N, 1, -1, 0, C>, tma_smem<N, C>());
    set_smem(k_yz_tma<N, 1, +1, 0, C>, tma_smem<N, C>());
    set_smem(k_yz_tma<N, 2, -1, 0, C>, tma_smem<N, C>());
    set_smem(k_yz_tma<N, 2, +1, 0, C>, tma_smem<N, C>());
    set_smem(k_zpass_inv_phase<N, C>, yz_smem());
    set_smem(k_ypass<N, -1, C>, yz_smem());
    set_smem(k_ypass<N, +1, C>, yz_smem());
    set_smem(k_zpass<N, -1, C>, yz_smem());
    set_smem(k_zpass<N, +1, C>, yz_smem());
    set_smem(k_xpass_products<N, C>, x_smem(6));
    set_smem(k_xpass_r2c<N, C>, x_smem(1));
    set_smem(k_xpass_c2r<N, C>, x_smem(1));
    set_smem(k_xpass_diag<N, C>, x_smem(2));
    set_smem(k_xpass_rot<N, C>, x_smem(6));
  }
  static const Ops* table() {
    static const Ops ops = {N,  (int)sizeof(C), kT, init, zpass_inv_phase, ypass, zpass, xpass_products, nyq_reduce,
                            sweep, xpass_r2c, xpass_c2r, xpass_diag, yz_tma, tma_blocks_per_sm, xpass2, xpass2_grid,
                            p5, p5_grid, omega_hat, xpass_rot, sweep_rot, xpass_diag2};
    return &ops;
  }
};

template <class C>
const Ops* ops_for_type(int n) {
  switch (n) {
    case 8: return Launch<8, C>::table();
    case 12: return Launch<12, C>::table();
    case 16: return Launch<16, C>::table();
    case 24: return Launch<24, C>::table();
    case 32: return Launch<32, C>::table();
    case 48: return Launch<48, C>::table();
    case 64: return Launch<64, C>::table();
    case 96: return Launch<96, C>::table();
    case 128: return Launch<128, C>::table();
    case 256: return Launch<256, C>::table();
    case 512: return Launch<512, C>::table();
    default: return nullptr;
  }
}

const Ops* ops_for(int n, int precision) {
  if (precision == 0) return ops_for_type<double2>(n);
  if (precision == 1) return ops_for_type<float2>(n);
  return nullptr;
}

static unsigned blocks_for(long long total, int bs) { return (unsigned)((total + bs - 1) / bs); }

template <class C>
static C* FC(void* p) { return static_cast<C*>(p); }
template <class C>
static const C* FC(const void* p) { return static_cast<const C*>(p); }

void launch_tgv_init(double* phys, Geom g, cudaStream_t st) {
  const long long np = (long long)g.n * g.n * g.n;
  k_tgv_init<<<blocks_for(np, 256), 256, 0, st>>>(phys, g.n);
}
void launch_project_truncate(void* u, int precision, Geom g, cudaStream_t st) {
  const long long total = (long long)g.n * g.n * (g.nh + 1);
  if (precision == 0) k_project_truncate<double2><<<blocks_for(total, 256), 256, 0, st>>>(FC<double2>(u), g);
  else k_project_truncate<float2><<<blocks_for(total, 256), 256, 0, st>>>(FC<float2>(u), g);
}
void launch_add_sparse(void* u, int precision, const long long* idx, const double2* val, int count,
                       cudaStream_t st) {
  if (count <= 0) return;
  if (precision == 0) k_add_sparse<double2><<<blocks_for(count, 256), 256, 0, st>>>(FC<double2>(u), idx, val, count);
  else k_add_sparse<float2><<<blocks_for(count, 256), 256, 0, st>>>(FC<float2>(u), idx, val, count);
}
void launch_half_to_full(const void* half, int precision, double2* full, Geom g, cudaStream_t st,
                         const CompWord* lo) {
  const long long total = (long long)g.n * g.n * g.n;
  if (precision == 0)
    k_half_to_full<double2><<<blocks_for(total, 256), 256, 0, st>>>(FC<double2>(half), full, g, nullptr);
  else k_half_to_full<float2><<<blocks_for(total, 256), 256, 0, st>>>(FC<float2>(half), full, g, lo);
}
void launch_full_to_half(const double2* full, void* half, int precision, int hermitian_part, Geom g,
                         cudaStream_t st, CompWord* lo, long long src_pitch) {
  const long long total = (long long)g.n * g.n * (g.nh + 1);
  if (src_pitch <= 0 || hermitian_part) src_pitch = g.n;
  if (precision == 0)
    k_full_to_half<double2><<<blocks_for(total, 256), 256, 0, st>>>(full, FC<double2>(half), hermitian_part,
                                                                      src_pitch, g, nullptr);
  else
    k_full_to_half<float2><<<blocks_for(total, 256), 256, 0, st>>>(full, FC<float2>(half), hermitian_part,
                                                                    src_pitch, g, lo);
}
void launch_spectral_diag(const void* u, int precision, double* partials, int nblocks, Geom g, cudaStream_t st) {
  if (precision == 0) k_spectral_diag<double2><<<nblocks, 256, 0, st>>>(FC<double2>(u), partials, g);
  else k_spectral_diag<float2><<<nblocks, 256, 0, st>>>(FC<float2>(u), partials, g);
}
// One thread: the reference's adaptive step (run_taylor_green, ava_taylor_green_impl.hpp:
// 1363-1378) on the device, with the horizon in place of the output times.
__device__ void clock_advance(const double* __restrict__ vmax2, double* __restrict__ c) {
  const double t = c[kClockT], t_end = c[kClockTEnd];
  if (c[kClockStopped] != 0.0 || !(t < t_end - 1.0e-14)) {
    c[kClockStopped] = 1.0;
    c[kClockDt] = 0.0;
    return;
  }
  const double vmax = sqrt(*vmax2);
  double main_dt = c[kClockDtMax];
  if (vmax > 1.0e-14) main_dt = fmin(main_dt, c[kClockCfl] * c[kClockDx] / vmax);
  const double dt = fmin(main_dt, t_end - t);
  c[kClockDt] = dt;
  c[kClockT] = t + dt;
  c[kClockSteps] += 1.0;
}
__global__ void k_clock_step(const double* __restrict__ vmax2, double* __restrict__ c) {
  if (threadIdx.x == 0 && blockIdx.x == 0) clock_advance(vmax2, c);
}

// The index-check record of the debug build: {count, first line, first index}; count -1 in
// the normal build, which has no checks.
int bounds_record(long long* out3) {
#ifdef SNS_BOUNDS_CHECK
  BoundsRecord r{};
  const cudaError_t e = cudaMemcpyFromSymbol(&r, g_bounds, sizeof r);
  if (e != cudaSuccess) return (int)e;
  out3[0] = (long long)r.count;
  out3[1] = r.line;
  out3[2] = r.index;
#else
  out3[0] = -1;
  out3[1] = 0;
  out3[2] = 0;
#endif
  return 0;
}

void launch_clock_step(const double* vmax2, double* clock, cudaStream_t st) {
  k_clock_step<<<1, 32, 0, st>>>(vmax2, clock);
}

// The max of the per-row vmax^2 partials (as k_reduce: max is exact in any order) and the
// clock's step from it in one launch, for the device CFL step.
__global__ void __launch_bounds__(1024) k_clock_step_partials(const double* __restrict__ partials, int count,
                                                              int stride, double* __restrict__ c) {
  __shared__ double red[1024];
  const int tid = threadIdx.x;
  double m[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i0 = tid; i0 < count; i0 += 4 * 1024) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int i = i0 + u * 1024;
      if (i < count) m[u] = fmax(m[u], partials[(long long)i * stride]);
    }
  }
  red[tid] = fmax(fmax(m[0], m[1]), fmax(m[2], m[3]));
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (tid < o) red[tid] = fmax(red[tid], red[tid + o]);
    __syncthreads();
  }
  if (tid == 0) clock_advance(red, c);
}

void launch_clock_step_partials(const double* partials, int count, int stride, double* clock, cudaStream_t st) {
  k_clock_step_partials<<<1, 1024, 0, st>>>(partials, count, stride, clock);
}

void launch_reduce(const double* partials, int count, int stride, int op_max, double* out, cudaStream_t st) {
  k_reduce<<<1, 1024, 0, st>>>(partials, count, stride, op_max, out);
}

}  // namespace sns
