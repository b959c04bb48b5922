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

// Poll with a bounded number of tries (about a second at worst); true when the phase landed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (uint32_t i = 0; i < (1u << 22); ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(128);
  }
  return false;
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

// 8 complex doubles (32 words) of this thread's lane, columns [col, col + 32).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const double2* v) {
  uint32_t w[32];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const unsigned long long a = __double_as_longlong(v[i].x), b = __double_as_longlong(v[i].y);
    w[4 * i + 0] = (uint32_t)a;
    w[4 * i + 1] = (uint32_t)(a >> 32);
    w[4 * i + 2] = (uint32_t)b;
    w[4 * i + 3] = (uint32_t)(b >> 32);
  }
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
      "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]), "r"(w[9]),
      "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15]), "r"(w[16]), "r"(w[17]), "r"(w[18]),
      "r"(w[19]), "r"(w[20]), "r"(w[21]), "r"(w[22]), "r"(w[23]), "r"(w[24]), "r"(w[25]), "r"(w[26]), "r"(w[27]),
      "r"(w[28]), "r"(w[29]), "r"(w[30]), "r"(w[31])
      : "memory");
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, double2* v) {
  uint32_t w[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
      : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7]), "=r"(w[8]),
        "=r"(w[9]), "=r"(w[10]), "=r"(w[11]), "=r"(w[12]), "=r"(w[13]), "=r"(w[14]), "=r"(w[15]), "=r"(w[16]),
        "=r"(w[17]), "=r"(w[18]), "=r"(w[19]), "=r"(w[20]), "=r"(w[21]), "=r"(w[22]), "=r"(w[23]), "=r"(w[24]),
        "=r"(w[25]), "=r"(w[26]), "=r"(w[27]), "=r"(w[28]), "=r"(w[29]), "=r"(w[30]), "=r"(w[31])
      : "r"(taddr)
      : "memory");
  tmem_wait_ld();
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    v[i].x = __longlong_as_double((long long)(((unsigned long long)w[4 * i + 1] << 32) | w[4 * i + 0]));
    v[i].y = __longlong_as_double((long long)(((unsigned long long)w[4 * i + 3] << 32) | w[4 * i + 2]));
  }
}

// One complex double (4 words) of this thread's lane at columns [col, col + 4).
__device__ __forceinline__ double2 tmem_ld1(uint32_t taddr) {
  uint32_t w0, w1, w2, w3;
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(w0), "=r"(w1), "=r"(w2), "=r"(w3)
               : "r"(taddr)
               : "memory");
  tmem_wait_ld();
  return make_double2(__longlong_as_double((long long)(((unsigned long long)w1 << 32) | w0)),
                      __longlong_as_double((long long)(((unsigned long long)w3 << 32) | w2)));
}

// K complex doubles (4K words, K = 4 or 8) of this thread's lane at columns [col, col + 4K).
template <int K>
__device__ __forceinline__ void tmem_st(uint32_t taddr, const double2* v) {
  if constexpr (K == 8) {
    tmem_st8(taddr, v);
  } else {
    static_assert(K == 4, "4 or 8 complex values");
    uint32_t w[16];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const unsigned long long a = __double_as_longlong(v[i].x), b = __double_as_longlong(v[i].y);
      w[4 * i + 0] = (uint32_t)a;
      w[4 * i + 1] = (uint32_t)(a >> 32);
      w[4 * i + 2] = (uint32_t)b;
      w[4 * i + 3] = (uint32_t)(b >> 32);
    }
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16};" ::"r"(taddr),
        "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7]), "r"(w[8]),
        "r"(w[9]), "r"(w[10]), "r"(w[11]), "r"(w[12]), "r"(w[13]), "r"(w[14]), "r"(w[15])
        : "memory");
  }
}

template <int K>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, double2* v) {
  if constexpr (K == 8) {
    tmem_ld8(taddr, v);
  } else {
    static_assert(K == 4, "4 or 8 complex values");
    uint32_t w[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]), "=r"(w[7]),
          "=r"(w[8]), "=r"(w[9]), "=r"(w[10]), "=r"(w[11]), "=r"(w[12]), "=r"(w[13]), "=r"(w[14]), "=r"(w[15])
        : "r"(taddr)
        : "memory");
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      v[i].x = __longlong_as_double((long long)(((unsigned long long)w[4 * i + 1] << 32) | w[4 * i + 0]));
      v[i].y = __longlong_as_double((long long)(((unsigned long long)w[4 * i + 3] << 32) | w[4 * i + 2]));
    }
  }
}

}  // namespace sns
