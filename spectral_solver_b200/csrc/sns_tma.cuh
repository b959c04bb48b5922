// TMA and mbarrier helpers for sm_100a (inline PTX; no cluster multicast anywhere).
//
// Every wait is bounded: a CTA that does not see its tile land within the limit records an
// error code in a device word the host checks after the launch, and returns, instead of
// spinning forever on a shared GPU.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace sns {

enum : int { kErrNone = 0, kErrTmaTimeout = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Orders this thread's generic-proxy shared-memory accesses before later async-proxy
// (bulk copy / TMA) accesses to the same bytes.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Poll with a bounded number of tries (about a second at worst with the default limit);
// true when the phase landed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit = 1u << 22) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(128);
  }
  return false;
}

// Invalidate a barrier before its shared memory is left (or reused for other data).
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// 4-D tiled TMA load global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int c0, int c1, int c2,
                                            int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// 1-D bulk copy global -> shared (size and both addresses multiples of 16 bytes).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}


// ------------------------------------------------------------------------------------
// Tensor memory (TMEM) as per-thread scratch: 128 lanes x 512 columns of 32-bit words per
// SM.  Warp w reaches lanes 32*(w%4) .. +31 (thread t of the warp: its own lane); the
// address is (lane << 16) | column.  Allocation is by one full warp, in powers of two
// >= 32 columns, and must be released before the CTA exits.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
  asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot_smem)),
               "r"(ncols)
               : "memory");
}
__device__ __forceinline__ void tmem_relinquish() {
  asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
  asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Words of this thread's lane: NW 32-bit words at columns [col, col + NW) (32x32b shape).
#define SNS_R2(i) "r"(w[i]), "r"(w[i + 1])
#define SNS_R4(i) SNS_R2(i), SNS_R2(i + 2)
#define SNS_R8(i) SNS_R4(i), SNS_R4(i + 4)
#define SNS_R16(i) SNS_R8(i), SNS_R8(i + 8)
#define SNS_R32(i) SNS_R16(i), SNS_R16(i + 16)
#define SNS_W2(i) "=r"(w[i]), "=r"(w[i + 1])
#define SNS_W4(i) SNS_W2(i), SNS_W2(i + 2)
#define SNS_W8(i) SNS_W4(i), SNS_W4(i + 4)
#define SNS_W16(i) SNS_W8(i), SNS_W8(i + 8)
#define SNS_W32(i) SNS_W16(i), SNS_W16(i + 16)

template <int NW>
__device__ __forceinline__ void tmem_st_words(uint32_t taddr, const uint32_t* w) {
  if constexpr (NW == 2) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(taddr), SNS_R2(0) : "memory");
  } else if constexpr (NW == 4) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr), SNS_R4(0)
                 : "memory");
  } else if constexpr (NW == 8) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
                 SNS_R8(0)
                 : "memory");
  } else if constexpr (NW == 16) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        SNS_R16(0)
        : "memory");
  } else {
    static_assert(NW == 32, "2, 4, 8, 16 or 32 words");
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        SNS_R32(0)
        : "memory");
  }
}

template <int NW>
__device__ __forceinline__ void tmem_ld_words(uint32_t taddr, uint32_t* w) {
  if constexpr (NW == 2) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];" : SNS_W2(0) : "r"(taddr) : "memory");
  } else if constexpr (NW == 4) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];" : SNS_W4(0) : "r"(taddr)
                 : "memory");
  } else if constexpr (NW == 8) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : SNS_W8(0)
                 : "r"(taddr)
                 : "memory");
  } else if constexpr (NW == 16) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : SNS_W16(0)
        : "r"(taddr)
        : "memory");
  } else {
    static_assert(NW == 32, "2, 4, 8, 16 or 32 words");
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : SNS_W32(0)
        : "r"(taddr)
        : "memory");
  }
  tmem_wait_ld();
}

#undef SNS_R2
#undef SNS_R4
#undef SNS_R8
#undef SNS_R16
#undef SNS_R32
#undef SNS_W2
#undef SNS_W4
#undef SNS_W8
#undef SNS_W16
#undef SNS_W32

// Complex values <-> 32-bit words (4 per complex double, 2 per complex float).
template <class C>
constexpr int tmem_words() { return (int)(sizeof(C) / 4); }

__device__ __forceinline__ void to_words(double2 v, uint32_t* w) {
  const unsigned long long a = __double_as_longlong(v.x), b = __double_as_longlong(v.y);
  w[0] = (uint32_t)a;
  w[1] = (uint32_t)(a >> 32);
  w[2] = (uint32_t)b;
  w[3] = (uint32_t)(b >> 32);
}
__device__ __forceinline__ void to_words(float2 v, uint32_t* w) {
  w[0] = __float_as_uint(v.x);
  w[1] = __float_as_uint(v.y);
}
__device__ __forceinline__ void from_words(const uint32_t* w, double2* v) {
  v->x = __longlong_as_double((long long)(((unsigned long long)w[1] << 32) | w[0]));
  v->y = __longlong_as_double((long long)(((unsigned long long)w[3] << 32) | w[2]));
}
__device__ __forceinline__ void from_words(const uint32_t* w, float2* v) {
  v->x = __uint_as_float(w[0]);
  v->y = __uint_as_float(w[1]);
}

// K complex values of this thread's lane at columns [col, col + K * words).
template <int K, class C>
__device__ __forceinline__ void tmem_st(uint32_t taddr, const C* v) {
  constexpr int WPC = tmem_words<C>();
  uint32_t w[K * WPC];
#pragma unroll
  for (int i = 0; i < K; ++i) to_words(v[i], w + WPC * i);
  tmem_st_words<K * WPC>(taddr, w);
}

template <int K, class C>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, C* v) {
  constexpr int WPC = tmem_words<C>();
  uint32_t w[K * WPC];
  tmem_ld_words<K * WPC>(taddr, w);
#pragma unroll
  for (int i = 0; i < K; ++i) from_words(w + WPC * i, v + i);
}

// One complex value of this thread's lane at columns [col, col + words).
template <class C>
__device__ __forceinline__ C tmem_ld1(uint32_t taddr) {
  C v;
  tmem_ld<1>(taddr, &v);
  return v;
}

}  // namespace sns
