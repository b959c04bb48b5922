// Shared-memory Stockham FFT engine for sm_100a (FP64 complex).
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

namespace sns {

__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by -i (DIR=-1) or +i (DIR=+1)
template <int DIR>
__host__ __device__ __forceinline__ double2 mul_dir_i(double2 a) {
  if constexpr (DIR < 0) return make_double2(a.y, -a.x);
  else return make_double2(-a.y, a.x);
}

// ------------------------------------------------------------------------------------
// R-point DFTs in registers, sign DIR (-1 forward, +1 inverse), unnormalised.
template <int DIR>
__host__ __device__ __forceinline__ void dft2(double2* v) {
  double2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int DIR>
__host__ __device__ __forceinline__ void dft3(double2* v) {
  constexpr double kS3 = 0.86602540378443864676372317075293618;  // sin(pi/3)
  double2 a = v[0], b = v[1], c = v[2];
  double2 t1 = cadd(b, c);
  double2 t2 = make_double2(a.x - 0.5 * t1.x, a.y - 0.5 * t1.y);
  double2 d = csub(b, c);
  // DIR*i*sin(pi/3)*(b-c) with forward sign -1: y1 = t2 - i*s*d, y2 = t2 + i*s*d
  double2 t3 = mul_dir_i<DIR>(make_double2(kS3 * d.x, kS3 * d.y));
  v[0] = cadd(a, t1);
  v[1] = cadd(t2, t3);
  v[2] = csub(t2, t3);
}

template <int DIR>
__host__ __device__ __forceinline__ void dft4(double2* v) {
  double2 a = v[0], b = v[1], c = v[2], d = v[3];
  double2 s0 = cadd(a, c), s1 = csub(a, c);
  double2 s2 = cadd(b, d), s3 = mul_dir_i<DIR>(csub(b, d));
  v[0] = cadd(s0, s2);
  v[2] = csub(s0, s2);
  v[1] = cadd(s1, s3);
  v[3] = csub(s1, s3);
}

template <int DIR>
__host__ __device__ __forceinline__ void dft8(double2* v) {
  constexpr double kH = 0.70710678118654752440084436210484904;  // sqrt(2)/2
  // radix-2 split into even/odd 4-point DFTs, then combine with W8^k
  double2 e[4] = {v[0], v[2], v[4], v[6]};
  double2 o[4] = {v[1], v[3], v[5], v[7]};
  dft4<DIR>(e);
  dft4<DIR>(o);
  // W8^1 = (1 + DIR*i)/sqrt2 * ... : exp(DIR*i*pi/4) = kH*(1 + DIR*i)
  double2 o1 = make_double2(kH * (o[1].x - DIR * o[1].y), kH * (o[1].y + DIR * o[1].x));
  double2 o2 = mul_dir_i<DIR>(o[2]);
  // W8^3 = exp(DIR*3i*pi/4) = kH*(-1 + DIR*i)
  double2 o3 = make_double2(kH * (-o[3].x - DIR * o[3].y), kH * (-o[3].y + DIR * o[3].x));
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
template <int DIR>
__host__ __device__ __forceinline__ void dft16(double2* v) {
  constexpr double c1 = 0.92387953251128675612818318939678829;  // cos(pi/8)
  constexpr double s1 = 0.38268343236508977172845998403039887;  // sin(pi/8)
  constexpr double h = 0.70710678118654752440084436210484904;   // cos(pi/4)
  double2 a[4][4];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    double2 t[4] = {v[n2], v[n2 + 4], v[n2 + 8], v[n2 + 12]};
    dft4<DIR>(t);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) a[n2][k1] = t[k1];
  }
  // twiddles W16^m, m = n2*k1, W16 = exp(DIR*2*pi*i/16): (cos, DIR*sin) of pi*m/8
  auto tw = [](double2 x, double c, double s) {  // x * (c + DIR*i*s)
    return make_double2(x.x * c - DIR * x.y * s, x.y * c + DIR * x.x * s);
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
    double2 t[4] = {a[0][k1], a[1][k1], a[2][k1], a[3][k1]};
    dft4<DIR>(t);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) v[k1 + 4 * k2] = t[k2];
  }
}

template <int R, int DIR>
__host__ __device__ __forceinline__ void dftR(double2* v) {
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

// Row pitch (in double2) of a padded RowTile sequence of length L.
__host__ __device__ constexpr int row_pitch(int L) { return L + (L + 7) / 8; }

// One Stockham stage for all NSEQ sequences, NT threads.
template <int L, int DIR, int NSEQ, int NT, class Addr, int Ns, int R>
__device__ __forceinline__ void fft_stage(double2* buf, const double2* tw, int tid) {
  constexpr int kBf = L / R;               // butterflies per sequence
  constexpr int kTot = NSEQ * kBf;          // butterflies in the tile
  constexpr int kBpt = (kTot + NT - 1) / NT;
  constexpr int kTwStep = L / (Ns * R);
  double2 v[kBpt][R];
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
        for (int r = 1; r < R; ++r) {
          double2 w = tw[r * k * kTwStep];
          if constexpr (DIR > 0) w.y = -w.y;
          v[i][r] = cmul(v[i][r], w);
        }
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

template <int L, int DIR, int NSEQ, int NT, class Addr, int Ns, int R, int... Rest>
__device__ __forceinline__ void fft_stages(double2* buf, const double2* tw, int tid) {
  fft_stage<L, DIR, NSEQ, NT, Addr, Ns, R>(buf, tw, tid);
  if constexpr (sizeof...(Rest) > 0) fft_stages<L, DIR, NSEQ, NT, Addr, Ns * R, Rest...>(buf, tw, tid);
}

template <int L, int DIR, int NSEQ, int NT, class Addr, int... Rs>
__device__ __forceinline__ void fft_run(double2* buf, const double2* tw, int tid, Radices<Rs...>) {
  fft_stages<L, DIR, NSEQ, NT, Addr, 1, Rs...>(buf, tw, tid);
}

// Transform NSEQ sequences of length L in place.  Caller must __syncthreads() before
// (data written) — the engine syncs after every stage, so the result is visible on return.
template <int L, int DIR, int NSEQ, int NT, class Addr>
__device__ __forceinline__ void smem_fft(double2* buf, const double2* tw, int tid) {
  fft_run<L, DIR, NSEQ, NT, Addr>(buf, tw, tid, typename Plan<L>::type{});
}


// ------------------------------------------------------------------------------------
// Tile FFT for the streaming y/z passes: 8 sequences (columns) of length L, element e of
// column s at e*8 + s.  The first stage reads a source policy (the TMA-filled input
// buffer, with any pre-multiplier fused into the load) and writes the work buffer W; the
// middle stages run in place in W; the last stage writes a destination policy (global
// memory, so the result never makes a second trip through shared memory).
template <int L, int DIR, int NT, int Ns, int R, bool FIRST, bool LAST, class Src, class Dst>
__device__ __forceinline__ void tstage(const Src& src, const Dst& dst, const double2* tw, int tid) {
  constexpr int kBf = L / R;
  constexpr int kTot = 8 * kBf;
  constexpr int kBpt = (kTot + NT - 1) / NT;
  constexpr int kTwStep = L / (Ns * R);
  double2 v[kBpt][R];
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      const int s = b & 7, j = b >> 3;
#pragma unroll
      for (int r = 0; r < R; ++r) v[i][r] = src(s, j + r * kBf);
      if constexpr (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          double2 w = tw[r * k * kTwStep];
          if constexpr (DIR > 0) w.y = -w.y;
          v[i][r] = cmul(v[i][r], w);
        }
      }
      dftR<R, DIR>(v[i]);
    }
  }
  if constexpr (!FIRST && !LAST) __syncthreads();  // in place in W
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      const int s = b & 7, j = b >> 3;
      const int base = (j / Ns) * Ns * R + (j % Ns);
#pragma unroll
      for (int r = 0; r < R; ++r) dst(s, base + r * Ns, v[i][r]);
    }
  }
  if constexpr (!LAST) __syncthreads();
}

struct WLoad {
  const double2* w;
  __device__ __forceinline__ double2 operator()(int s, int e) const { return w[e * 8 + s]; }
};
struct WStore {
  double2* w;
  __device__ __forceinline__ void operator()(int s, int e, double2 v) const { w[e * 8 + s] = v; }
};

template <int L, int DIR, int NT, int Ns, bool FIRST, class Src0, class DstG, int R, int... Rest>
__device__ __forceinline__ void tfft_rec(const Src0& src0, double2* W, const DstG& dstg, const double2* tw, int tid) {
  constexpr bool LAST = sizeof...(Rest) == 0;
  if constexpr (FIRST && LAST) {
    tstage<L, DIR, NT, Ns, R, true, true>(src0, dstg, tw, tid);
  } else if constexpr (FIRST) {
    tstage<L, DIR, NT, Ns, R, true, false>(src0, WStore{W}, tw, tid);
  } else if constexpr (LAST) {
    tstage<L, DIR, NT, Ns, R, false, true>(WLoad{W}, dstg, tw, tid);
  } else {
    tstage<L, DIR, NT, Ns, R, false, false>(WLoad{W}, WStore{W}, tw, tid);
  }
  if constexpr (!LAST) tfft_rec<L, DIR, NT, Ns * R, false, Src0, DstG, Rest...>(src0, W, dstg, tw, tid);
}

template <int L, int DIR, int NT, class Src0, class DstG, int... Rs>
__device__ __forceinline__ void tfft_run(const Src0& src0, double2* W, const DstG& dstg, const double2* tw, int tid,
                                         Radices<Rs...>) {
  tfft_rec<L, DIR, NT, 1, true, Src0, DstG, Rs...>(src0, W, dstg, tw, tid);
}

// Transform the 8 columns read through src0; results go to dstg(s, e, value).  No barrier
// is issued after the last stage: the caller syncs before reusing W or the source buffer.
template <int L, int DIR, int NT, class Src0, class DstG>
__device__ __forceinline__ void tile_fft(const Src0& src0, double2* W, const DstG& dstg, const double2* tw, int tid) {
  tfft_run<L, DIR, NT>(src0, W, dstg, tw, tid, typename Plan<L>::type{});
}

// ------------------------------------------------------------------------------------
// Tile FFT whose last stage leaves its outputs in registers: out.v[i][r] is output r of the
// thread's butterfly i, i.e. column s = b & 7 and element (j/Ns)*Ns*R + j%Ns + r*Ns of that
// column, with b = tid + i*NT, j = b >> 3 and Ns, R those of the last radix.
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

template <int L, int NT>
struct RegOut {
  static constexpr int R = LastRadix<typename Plan<L>::type>::value;
  static constexpr int NS = L / R;                       // Ns of the last stage
  static constexpr int KB = (8 * (L / R) + NT - 1) / NT;  // butterflies per thread
  double2 v[KB][R];
};

template <int L, int DIR, int NT, int Ns, int R, class Src, class Out>
__device__ __forceinline__ void tstage_regs(const Src& src, const double2* tw, int tid, Out& out) {
  constexpr int kBf = L / R;
  constexpr int kTot = 8 * kBf;
  constexpr int kTwStep = L / (Ns * R);
#pragma unroll
  for (int i = 0; i < Out::KB; ++i) {
    const int b = tid + i * NT;
    if (kTot % NT == 0 || b < kTot) {
      const int s = b & 7, j = b >> 3;
#pragma unroll
      for (int r = 0; r < R; ++r) out.v[i][r] = src(s, j + r * kBf);
      if constexpr (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) {
          double2 w = tw[r * k * kTwStep];
          if constexpr (DIR > 0) w.y = -w.y;
          out.v[i][r] = cmul(out.v[i][r], w);
        }
      }
      dftR<R, DIR>(out.v[i]);
    }
  }
}

template <int L, int DIR, int NT, int Ns, bool FIRST, class Src0, class Out, int R, int... Rest>
__device__ __forceinline__ void tfft_regs_rec(const Src0& src0, double2* W, const double2* tw, int tid, Out& out) {
  if constexpr (sizeof...(Rest) == 0) {
    if constexpr (FIRST) tstage_regs<L, DIR, NT, Ns, R>(src0, tw, tid, out);
    else tstage_regs<L, DIR, NT, Ns, R>(WLoad{W}, tw, tid, out);
  } else {
    if constexpr (FIRST) tstage<L, DIR, NT, Ns, R, true, false>(src0, WStore{W}, tw, tid);
    else tstage<L, DIR, NT, Ns, R, false, false>(WLoad{W}, WStore{W}, tw, tid);
    tfft_regs_rec<L, DIR, NT, Ns * R, false, Src0, Out, Rest...>(src0, W, tw, tid, out);
  }
}

template <int L, int DIR, int NT, class Src0, class Out, int... Rs>
__device__ __forceinline__ void tfft_regs_run(const Src0& src0, double2* W, const double2* tw, int tid, Out& out,
                                              Radices<Rs...>) {
  tfft_regs_rec<L, DIR, NT, 1, true, Src0, Out, Rs...>(src0, W, tw, tid, out);
}

template <int L, int DIR, int NT, class Src0>
__device__ __forceinline__ void tile_fft_regs(const Src0& src0, double2* W, const double2* tw, int tid,
                                              RegOut<L, NT>& out) {
  tfft_regs_run<L, DIR, NT>(src0, W, tw, tid, out, typename Plan<L>::type{});
}

// ------------------------------------------------------------------------------------
// Tile FFT whose last stage hands each butterfly's R outputs to sink(i, v) as soon as they
// are computed (i = the thread's butterfly index; output r of butterfly i sits at column
// b & 7 and element (j/NS)*NS*R + j%NS + r*NS, b = tid + i*NT, j = b >> 3), so only R
// values are live at a time.  Requires every thread to own whole butterflies.
template <int L, int DIR, int NT, int Ns, int R, class Src, class Sink>
__device__ __forceinline__ void tstage_sink(const Src& src, const double2* tw, int tid, Sink& sink) {
  constexpr int kBf = L / R;
  constexpr int kTot = 8 * kBf;
  static_assert(kTot % NT == 0, "whole butterflies per thread");
  constexpr int kBpt = kTot / NT;
  constexpr int kTwStep = L / (Ns * R);
#pragma unroll
  for (int i = 0; i < kBpt; ++i) {
    const int b = tid + i * NT;
    const int s = b & 7, j = b >> 3;
    double2 v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src(s, j + r * kBf);
    if constexpr (Ns > 1) {
      const int k = j % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        double2 w = tw[r * k * kTwStep];
        if constexpr (DIR > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dftR<R, DIR>(v);
    sink(i, v);
  }
}

template <int L, int DIR, int NT, int Ns, bool FIRST, class Src0, class Sink, int R, int... Rest>
__device__ __forceinline__ void tfft_sink_rec(const Src0& src0, double2* W, const double2* tw, int tid, Sink& sink) {
  if constexpr (sizeof...(Rest) == 0) {
    if constexpr (FIRST) tstage_sink<L, DIR, NT, Ns, R>(src0, tw, tid, sink);
    else tstage_sink<L, DIR, NT, Ns, R>(WLoad{W}, tw, tid, sink);
  } else {
    if constexpr (FIRST) tstage<L, DIR, NT, Ns, R, true, false>(src0, WStore{W}, tw, tid);
    else tstage<L, DIR, NT, Ns, R, false, false>(WLoad{W}, WStore{W}, tw, tid);
    tfft_sink_rec<L, DIR, NT, Ns * R, false, Src0, Sink, Rest...>(src0, W, tw, tid, sink);
  }
}

template <int L, int DIR, int NT, class Src0, class Sink, int... Rs>
__device__ __forceinline__ void tfft_sink_run(const Src0& src0, double2* W, const double2* tw, int tid, Sink& sink,
                                              Radices<Rs...>) {
  tfft_sink_rec<L, DIR, NT, 1, true, Src0, Sink, Rs...>(src0, W, tw, tid, sink);
}

template <int L, int DIR, int NT, class Src0, class Sink>
__device__ __forceinline__ void tile_fft_sink(const Src0& src0, double2* W, const double2* tw, int tid, Sink& sink) {
  tfft_sink_run<L, DIR, NT>(src0, W, tw, tid, sink, typename Plan<L>::type{});
}

}  // namespace sns
