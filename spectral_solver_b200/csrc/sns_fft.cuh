// Shared-memory Stockham FFT engine for sm_100a, generic over the complex type
// (double2 for the FP64 plain form, float2 for the FP32 precision form).
//
// A CTA transforms NSEQ independent sequences of length L that sit in shared memory.
// Each radix-R stage is the Stockham autosort step (Stockham 1966; the GPU form of
// Govindaraju et al., SC'08): butterfly j of a sequence reads elements j + r*L/R,
// multiplies by W_{Ns*R}^{r*(j mod Ns)}, runs an R-point DFT in registers and writes
// elements (j/Ns)*Ns*R + (j mod Ns) + r*Ns.  Output comes out in natural order, so no
// bit reversal pass is needed.  Radices 2, 3, 4 and 8 are written out as register
// butterflies; each length has a compile-time plan.
//
// Twiddles come from a per-CTA shared-memory table tw[t] = exp(-2*pi*i*t/L), t < L,
// filled from a host-computed global table (no sin/cos on the device).
//
// Addressing is a policy: ColTile (y/z passes: element e of sequence s at e*NSEQ + s,
// one 128-byte row of 8 sequences per element, conflict-free) or RowTile (x pass:
// element e of sequence s at s*PITCH + e + e/8; the one-slot-per-8 padding keeps the
// stride-R stores of the first stages free of bank conflicts).
#pragma once

#include <cuda_runtime.h>

#include "sns_check.cuh"

namespace sns {

// Complex type traits and helpers (double2 / float2).
template <class C>
struct CplxT;
template <>
struct CplxT<double2> {
  using R = double;
};
template <>
struct CplxT<float2> {
  using R = float;
};
template <class T>
struct RealT;
template <>
struct RealT<double> {
  using C = double2;
};
template <>
struct RealT<float> {
  using C = float2;
};
template <class C>
using real_of = typename CplxT<C>::R;
template <class T>
using cplx_of = typename RealT<T>::C;

__host__ __device__ __forceinline__ double2 cmk(double x, double y) { return make_double2(x, y); }
__host__ __device__ __forceinline__ float2 cmk(float x, float y) { return make_float2(x, y); }
template <class C>
__host__ __device__ __forceinline__ C czero() {
  return cmk(real_of<C>(0), real_of<C>(0));
}
template <class C>
__host__ __device__ __forceinline__ C cadd(C a, C b) {
  return cmk(a.x + b.x, a.y + b.y);
}
template <class C>
__host__ __device__ __forceinline__ C csub(C a, C b) {
  return cmk(a.x - b.x, a.y - b.y);
}
template <class C>
__host__ __device__ __forceinline__ C cmul(C a, C b) {
  return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// FP32 complex add and subtract as one packed instruction on the register pair (sm_100's
// add.f32x2 / sub.f32x2: two IEEE single-precision operations, round to nearest, the same
// results as two scalar ones).  Opt-in: the two-stage x pass is bound by instruction issue
// and most of its arithmetic is butterfly additions, so it takes them; in the y/z passes and
// the fused sweep they cost 2-3 % (additions there often absorb a product into an FFMA,
// which a packed add prevents), so those keep the scalar forms.
__device__ __forceinline__ unsigned long long f2_pack(float2 a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ float2 f2_unpack(unsigned long long r) {
  float2 a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ float2 padd(float2 a, float2 b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pack(a)), "l"(f2_pack(b)));
  return f2_unpack(d);
}
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pack(a)), "l"(f2_pack(b)));
  return f2_unpack(d);
}
// (a.x * b.x, a.y * b.y) in one packed instruction
__device__ __forceinline__ float2 pmul(float2 a, float2 b) {
  unsigned long long d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f2_pack(a)), "l"(f2_pack(b)));
  return f2_unpack(d);
}

// a * conj(b)
template <class C>
__host__ __device__ __forceinline__ C cmulc(C a, C b) {
  return cmk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <class C>
__host__ __device__ __forceinline__ C cscale(C a, real_of<C> s) {
  return cmk(s * a.x, s * a.y);
}
template <class C>
__host__ __device__ __forceinline__ C cconj(C a) {
  return cmk(a.x, -a.y);
}
// multiply by -i (DIR=-1) or +i (DIR=+1)
template <int DIR, class C>
__host__ __device__ __forceinline__ C mul_dir_i(C a) {
  if constexpr (DIR < 0) return cmk(a.y, -a.x);
  else return cmk(-a.y, a.x);
}

// ------------------------------------------------------------------------------------
// R-point DFTs in registers, sign DIR (-1 forward, +1 inverse), unnormalised.
template <int DIR, class C>
__host__ __device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int DIR, class C>
__host__ __device__ __forceinline__ void dft3(C* v) {
  using RT = real_of<C>;
  constexpr RT kS3 = RT(0.86602540378443864676372317075293618);  // sin(pi/3)
  constexpr RT kHalf = RT(0.5);
  C a = v[0], b = v[1], c = v[2];
  C t1 = cadd(b, c);
  C t2 = cmk(a.x - kHalf * t1.x, a.y - kHalf * t1.y);
  C d = csub(b, c);
  // DIR*i*sin(pi/3)*(b-c) with forward sign -1: y1 = t2 - i*s*d, y2 = t2 + i*s*d
  C t3 = mul_dir_i<DIR>(cmk(kS3 * d.x, kS3 * d.y));
  v[0] = cadd(a, t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}

template <int DIR, class C>
__host__ __device__ __forceinline__ void dft4(C* v) {
  C a = v[0], b = v[1], c = v[2], d = v[3];
  C s0 = cadd(a, c), s1 = csub(a, c);
  C s2 = cadd(b, d), s3 = mul_dir_i<DIR>(csub(b, d));
  v[0] = cadd(s0, s2);
  v[2] = csub(s0, s2);
  v[1] = cadd(s1, s3);
  v[3] = csub(s1, s3);
}
// FP32 with packed additions: the six plain additions packed; the two that take +-i (b - d)
// stay scalar, so the swapped pair is never formed.  Same results as dft4<DIR, float2>.
template <int DIR>
__device__ __forceinline__ void dft4p(float2* v) {
  const float2 a = v[0], b = v[1], c = v[2], d = v[3];
  const float2 s0 = padd(a, c), s1 = psub(a, c), s2 = padd(b, d), t = psub(b, d);
  v[0] = padd(s0, s2);
  v[2] = psub(s0, s2);
  if constexpr (DIR < 0) {  // s3 = -i t
    v[1] = make_float2(s1.x + t.y, s1.y - t.x);
    v[3] = make_float2(s1.x - t.y, s1.y + t.x);
  } else {  // s3 = +i t
    v[1] = make_float2(s1.x - t.y, s1.y + t.x);
    v[3] = make_float2(s1.x + t.y, s1.y - t.x);
  }
}

template <int DIR, class C>
__host__ __device__ __forceinline__ void dft8(C* v) {
  using RT = real_of<C>;
  constexpr RT kH = RT(0.70710678118654752440084436210484904);  // sqrt(2)/2
  // radix-2 split into even/odd 4-point DFTs, then combine with W8^k
  C e[4] = {v[0], v[2], v[4], v[6]};
  C o[4] = {v[1], v[3], v[5], v[7]};
  dft4<DIR>(e);
  dft4<DIR>(o);
  // W8^1 = (1 + DIR*i)/sqrt2 * ... : exp(DIR*i*pi/4) = kH*(1 + DIR*i)
  C o1 = cmk(kH * (o[1].x - DIR * o[1].y), kH * (o[1].y + DIR * o[1].x));
  C o2 = mul_dir_i<DIR>(o[2]);
  // W8^3 = exp(DIR*3i*pi/4) = kH*(-1 + DIR*i)
  C o3 = cmk(kH * (-o[3].x - DIR * o[3].y), kH * (-o[3].y + DIR * o[3].x));
  v[0] = cadd(e[0], o[0]);
  v[4] = csub(e[0], o[0]);
  v[1] = cadd(e[1], o1);
  v[5] = csub(e[1], o1);
  v[2] = cadd(e[2], o2);
  v[6] = csub(e[2], o2);
  v[3] = cadd(e[3], o3);
  v[7] = csub(e[3], o3);
}


// 16-point DFT in registers, natural order in and out: 4 x 4 Cooley-Tukey
// (inner 4-point DFTs over stride-4 inputs, twiddles W16^(n2*k1), outer 4-point DFTs).
// PK: the 4-point DFTs with packed FP32 additions (C = float2, device code only).
template <int DIR, class C, bool PK = false>
__host__ __device__ __forceinline__ void dft16(C* v) {
  using RT = real_of<C>;
  constexpr RT c1 = RT(0.92387953251128675612818318939678829);  // cos(pi/8)
  constexpr RT s1 = RT(0.38268343236508977172845998403039887);  // sin(pi/8)
  constexpr RT h = RT(0.70710678118654752440084436210484904);   // cos(pi/4)
  C a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    C t[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
    if constexpr (PK) dft4p<DIR>(t);
    else dft4<DIR>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
  }
  // twiddles W16^m, m = n2*k1, W16 = exp(DIR*2*pi*i/16): (cos, DIR*sin) of pi*m/8
  auto tw = [](C x, RT c, RT s) {  // x * (c + DIR*i*s)
    return cmk(x.x * c - DIR * x.y * s, x.y * c + DIR * x.x * s);
  };
  a[1][1] = tw(a[1][1], c1, s1);
  a[1][2] = tw(a[1][2], h, h);
  a[1][3] = tw(a[1][3], s1, c1);
  a[2][1] = tw(a[2][1], h, h);
  a[2][2] = mul_dir_i<DIR>(a[2][2]);
  a[2][3] = tw(a[2][3], -h, h);
  a[3][1] = tw(a[3][1], s1, c1);
  a[3][2] = tw(a[3][2], -h, h);
  a[3][3] = tw(a[3][3], -c1, -s1);
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    if constexpr (PK) dft4p<DIR>(t);
    else dft4<DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
  }
}

template <int R, int DIR, class C>
__host__ __device__ __forceinline__ void dftR(C* v) {
  if constexpr (R == 2) dft2<DIR>(v);
  else if constexpr (R == 3) dft3<DIR>(v);
  else if constexpr (R == 4) dft4<DIR>(v);
  else if constexpr (R == 8) dft8<DIR>(v);
  else if constexpr (R == 16) dft16<DIR>(v);
  else static_assert(R == 2, "unsupported radix");
}

// ------------------------------------------------------------------------------------
// Plans: radices in application order.  Ns grows as the product of earlier radices.
template <int... Rs>
struct Radices {};

template <int L>
struct Plan;
template <> struct Plan<2> { using type = Radices<2>; };
template <> struct Plan<4> { using type = Radices<4>; };
template <> struct Plan<6> { using type = Radices<3, 2>; };
template <> struct Plan<8> { using type = Radices<8>; };
template <> struct Plan<12> { using type = Radices<4, 3>; };
template <> struct Plan<16> { using type = Radices<4, 4>; };
template <> struct Plan<24> { using type = Radices<8, 3>; };
template <> struct Plan<32> { using type = Radices<8, 4>; };
template <> struct Plan<48> { using type = Radices<4, 4, 3>; };
template <> struct Plan<64> { using type = Radices<8, 8>; };
template <> struct Plan<96> { using type = Radices<8, 4, 3>; };
template <> struct Plan<128> { using type = Radices<8, 4, 4>; };
template <> struct Plan<256> { using type = Radices<8, 8, 4>; };
template <> struct Plan<512> { using type = Radices<8, 8, 8>; };
template <> struct Plan<1024> { using type = Radices<8, 8, 4, 4>; };

// Addressing policies -----------------------------------------------------------------
template <int NSEQ>
struct ColTile {  // element e of sequence s -> e*NSEQ + s
  static __device__ __forceinline__ int at(int s, int e) { return e * NSEQ + s; }
  static constexpr bool kSeqFast = true;
};

template <int PITCH>
struct RowTile {  // element e of sequence s -> s*PITCH + e + e/8
  static __device__ __forceinline__ int at(int s, int e) { return s * PITCH + e + (e >> 3); }
  static constexpr bool kSeqFast = false;
};

// Row pitch (in complex elements) of a padded RowTile sequence of length L.
__host__ __device__ constexpr int row_pitch(int L) { return L + (L + 7) / 8; }

// Twiddle of a stage: tw[t] = exp(-2*pi*i*t/L); the inverse uses its conjugate.
template <int DIR, class C>
__device__ __forceinline__ C stage_twiddle(const C* tw, int t) {
  C w = tw[t];
  if constexpr (DIR > 0) w.y = -w.y;
  return w;
}

// One Stockham stage for all NSEQ sequences, NT threads.
template <int L, int DIR, int NSEQ, int NT, class Addr, int Ns, int R, class C>
__device__ __forceinline__ void fft_stage(C* buf, const C* tw, int tid) {
  constexpr int kBf = L / R;               // butterflies per sequence
  constexpr int kTot = NSEQ * kBf;          // butterflies in the tile
  constexpr int kBpt = (kTot + NT - 1) / NT;
  constexpr int kTwStep = L / (Ns * R);
  C v[kBpt][R];
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      int s, j;
      if constexpr (Addr::kSeqFast) { s = b % NSEQ; j = b / NSEQ; }
      else { j = b % kBf; s = b / kBf; }
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = buf[Addr::at(s, j + r * kBf)];
      if constexpr (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) v[i][r] = cmul(v[i][r], stage_twiddle<DIR>(tw, r * k * kTwStep));
      }
      dftR<R, DIR>(v[i]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      int s, j;
      if constexpr (Addr::kSeqFast) { s = b % NSEQ; j = b / NSEQ; }
      else { j = b % kBf; s = b / kBf; }
      const int k = j % Ns;
      const int base = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) buf[Addr::at(s, base + r * Ns)] = v[i][r];
    }
  }
  __syncthreads();
}

template <int L, int DIR, int NSEQ, int NT, class Addr, int Ns, int R, int... Rest, class C>
__device__ __forceinline__ void fft_stages(C* buf, const C* tw, int tid) {
  fft_stage<L, DIR, NSEQ, NT, Addr, Ns, R>(buf, tw, tid);
  if constexpr (sizeof...(Rest) > 0) fft_stages<L, DIR, NSEQ, NT, Addr, Ns * R, Rest...>(buf, tw, tid);
}

template <int L, int DIR, int NSEQ, int NT, class Addr, class C, int... Rs>
__device__ __forceinline__ void fft_run(C* buf, const C* tw, int tid, Radices<Rs...>) {
  fft_stages<L, DIR, NSEQ, NT, Addr, 1, Rs...>(buf, tw, tid);
}

// Transform NSEQ sequences of length L in place.  Caller must __syncthreads() before
// (data written) — the engine syncs after every stage, so the result is visible on return.
template <int L, int DIR, int NSEQ, int NT, class Addr, class C>
__device__ __forceinline__ void smem_fft(C* buf, const C* tw, int tid) {
  fft_run<L, DIR, NSEQ, NT, Addr>(buf, tw, tid, typename Plan<L>::type{});
}


// ------------------------------------------------------------------------------------
// Tile FFT for the streaming y/z passes: TW sequences (columns) of length L, element e of
// column s at e*TW + s (TW = 8 complex doubles or 16 complex floats: one 128-byte row
// segment per element).  The first stage reads a source policy (the TMA-filled input
// buffer, with any pre-multiplier fused into the load) and writes the work buffer W; the
// middle stages run in place in W; the last stage writes a destination policy (global
// memory, so the result never makes a second trip through shared memory).
template <int L, int DIR, int NT, int TW, int Ns, int R, bool FIRST, bool LAST, class Src, class Dst, class C>
__device__ __forceinline__ void tstage(const Src& src, const Dst& dst, const C* tw, int tid) {
  constexpr int kBf = L / R;
  constexpr int kTot = TW * kBf;
  constexpr int kBpt = (kTot + NT - 1) / NT;
  constexpr int kTwStep = L / (Ns * R);
  C v[kBpt][R];
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      const int s = b % TW, j = b / TW;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = src(s, j + r * kBf);
      if constexpr (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) v[i][r] = cmul(v[i][r], stage_twiddle<DIR>(tw, SNS_IDX(r * k * kTwStep, L)));
      }
      dftR<R, DIR>(v[i]);
    }
  }
  if constexpr (!FIRST && !LAST) __syncthreads();  // in place in W
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      const int s = b % TW, j = b / TW;
      const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
      for (int r = 0; r < R; ++r) dst(s, base + r * Ns, v[i][r]);
    }
  }
  if constexpr (!LAST) __syncthreads();
}

template <int TW, class C>
struct WLoad {
  const C* w;
  int n;  // elements of the work buffer (the index check of the debug build)
  __device__ __forceinline__ C operator()(int s, int e) const { return w[SNS_IDX(e * TW + s, n)]; }
};
template <int TW, class C>
struct WStore {
  C* w;
  int n;
  __device__ __forceinline__ void operator()(int s, int e, C v) const { w[SNS_IDX(e * TW + s, n)] = v; }
};

template <int L, int DIR, int NT, int TW, int Ns, bool FIRST, class Src0, class DstG, class C, int R, int... Rest>
__device__ __forceinline__ void tfft_rec(const Src0& src0, C* W, const DstG& dstg, const C* tw, int tid) {
  constexpr bool LAST = sizeof...(Rest) == 0;
  using WL = WLoad<TW, C>;
  using WS = WStore<TW, C>;
  if constexpr (FIRST && LAST) {
    tstage<L, DIR, NT, TW, Ns, R, true, true>(src0, dstg, tw, tid);
  } else if constexpr (FIRST) {
    tstage<L, DIR, NT, TW, Ns, R, true, false>(src0, WS{W, L * TW}, tw, tid);
  } else if constexpr (LAST) {
    tstage<L, DIR, NT, TW, Ns, R, false, true>(WL{W, L * TW}, dstg, tw, tid);
  } else {
    tstage<L, DIR, NT, TW, Ns, R, false, false>(WL{W, L * TW}, WS{W, L * TW}, tw, tid);
  }
  if constexpr (!LAST) tfft_rec<L, DIR, NT, TW, Ns * R, false, Src0, DstG, C, Rest...>(src0, W, dstg, tw, tid);
}

template <int L, int DIR, int NT, int TW, class Src0, class DstG, class C, int... Rs>
__device__ __forceinline__ void tfft_run(const Src0& src0, C* W, const DstG& dstg, const C* tw, int tid,
                                         Radices<Rs...>) {
  tfft_rec<L, DIR, NT, TW, 1, true, Src0, DstG, C, Rs...>(src0, W, dstg, tw, tid);
}

// Transform the TW columns read through src0; results go to dstg(s, e, value).  No barrier
// is issued after the last stage: the caller syncs before reusing W or the source buffer.
template <int L, int DIR, int NT, int TW, class Src0, class DstG, class C>
__device__ __forceinline__ void tile_fft(const Src0& src0, C* W, const DstG& dstg, const C* tw, int tid) {
  tfft_run<L, DIR, NT, TW>(src0, W, dstg, tw, tid, typename Plan<L>::type{});
}

// ------------------------------------------------------------------------------------
// Tile FFT whose last stage hands each butterfly's R outputs to sink(i, v) as soon as they
// are computed (i = the thread's butterfly index; output r of butterfly i sits at column
// b % TW and element (j/NS)*NS*R + j%NS + r*NS, b = tid + i*NT, j = b / TW), so only R
// values are live at a time.  Requires every thread to own whole butterflies.
template <class P>
struct LastRadix;
template <int R>
struct LastRadix<Radices<R>> {
  static constexpr int value = R;
};
template <int R0, int R1, int... Rs>
struct LastRadix<Radices<R0, R1, Rs...>> {
  static constexpr int value = LastRadix<Radices<R1, Rs...>>::value;
};

// Shape of the last stage of a TW-column tile FFT of length L on NT threads.
template <int L, int NT, int TW>
struct LastStage {
  static constexpr int R = LastRadix<typename Plan<L>::type>::value;
  static constexpr int NS = L / R;                        // Ns of the last stage
  static constexpr int KB = (TW * (L / R) + NT - 1) / NT;  // butterflies per thread
};

template <int L, int DIR, int NT, int TW, int Ns, int R, class Src, class Sink, class C>
__device__ __forceinline__ void tstage_sink(const Src& src, const C* tw, int tid, Sink& sink) {
  constexpr int kBf = L / R;
  constexpr int kTot = TW * kBf;
  static_assert(kTot % NT == 0, "whole butterflies per thread");
  constexpr int kBpt = kTot / NT;
  constexpr int kTwStep = L / (Ns * R);
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    const int s = b % TW, j = b / TW;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src(s, j + r * kBf);
    if constexpr (Ns > 1) {
      const int k = j % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], stage_twiddle<DIR>(tw, r * k * kTwStep));
    }
    dftR<R, DIR>(v);
    sink(i, v);
  }
}

template <int L, int DIR, int NT, int TW, int Ns, bool FIRST, class Src0, class Sink, class C, int R, int... Rest>
__device__ __forceinline__ void tfft_sink_rec(const Src0& src0, C* W, const C* tw, int tid, Sink& sink) {
  using WL = WLoad<TW, C>;
  using WS = WStore<TW, C>;
  if constexpr (sizeof...(Rest) == 0) {
    if constexpr (FIRST) tstage_sink<L, DIR, NT, TW, Ns, R>(src0, tw, tid, sink);
    else tstage_sink<L, DIR, NT, TW, Ns, R>(WL{W, L * TW}, tw, tid, sink);
  } else {
    if constexpr (FIRST) tstage<L, DIR, NT, TW, Ns, R, true, false>(src0, WS{W, L * TW}, tw, tid);
    else tstage<L, DIR, NT, TW, Ns, R, false, false>(WL{W, L * TW}, WS{W, L * TW}, tw, tid);
    tfft_sink_rec<L, DIR, NT, TW, Ns * R, false, Src0, Sink, C, Rest...>(src0, W, tw, tid, sink);
  }
}

template <int L, int DIR, int NT, int TW, class Src0, class Sink, class C, int... Rs>
__device__ __forceinline__ void tfft_sink_run(const Src0& src0, C* W, const C* tw, int tid, Sink& sink,
                                              Radices<Rs...>) {
  tfft_sink_rec<L, DIR, NT, TW, 1, true, Src0, Sink, C, Rs...>(src0, W, tw, tid, sink);
}

template <int L, int DIR, int NT, int TW, class Src0, class Sink, class C>
__device__ __forceinline__ void tile_fft_sink(const Src0& src0, C* W, const C* tw, int tid, Sink& sink) {
  tfft_sink_run<L, DIR, NT, TW>(src0, W, tw, tid, sink, typename Plan<L>::type{});
}

}  // namespace sns
