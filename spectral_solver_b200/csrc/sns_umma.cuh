// tcgen05 tensor-core MMA helpers for sm_100a (inline PTX; one CTA, no cluster, no multicast).
//
// Operands come from shared memory through 64-bit matrix descriptors; the accumulator lives
// in tensor memory.  Layout used here: K-major, no swizzle ("interleave"): a core matrix is 8
// rows x 16 bytes (8 rows x 4 FP32/TF32 values) stored contiguously in 128 bytes; the
// descriptor's leading byte offset (LBO) steps between the core matrices that are adjacent
// along K, its stride byte offset (SBO) between the 8-row groups.  One kind::tf32 MMA consumes
// K = 8 values per row (two core-matrix columns), so successive K steps advance the start
// address by 2 * LBO.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "sns_tma.cuh"

namespace sns {

// Byte offset of element (row, k) of a K-major no-swizzle operand with K values per row
// (K a multiple of 4), LBO = 128 bytes (the K core matrices of a row group adjacent) and
// SBO = K/4 * 128 bytes (row groups one after another).
__host__ __device__ constexpr uint32_t umma_kmajor_offset(int row, int k, int K) {
  return (uint32_t)((row >> 3) * (K / 4) * 128 + (k >> 2) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

// Shared-memory matrix descriptor (sm_100 layout: start >> 4 at bit 0, LBO >> 4 at bit 16,
// SBO >> 4 at bit 32, version 1 at bit 46, layout type at bits 61-63 = 0 for no swizzle).
__device__ __forceinline__ uint64_t umma_desc(uint32_t smem_addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((smem_addr >> 4) & 0x3fffu) | ((uint64_t)((lbo >> 4) & 0x3fffu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3fffu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::tf32 with an FP32 accumulator, both operands K-major:
// D format F32 (bits 4-5 = 1), A and B format TF32 (bits 7-9, 10-12 = 2), N >> 3 at bit 17,
// M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_tf32(int M, int N) {
  return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void umma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          bool accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(d_tmem), "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1u : 0u)
      : "memory");
}

// Arrive on `bar` once every MMA this thread issued before has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// TF32 split of an FP32 value: hi keeps the 10 explicit mantissa bits the tensor core reads
// (the low 13 cleared), lo = x - hi (exact in FP32) carries the next bits.  hi*b + lo*b with
// b = b_hi + b_lo, dropping lo*b_lo, gives about 21 bits: the 3xTF32 product.
__device__ __forceinline__ void tf32_split(float x, float* hi, float* lo) {
  const float h = __uint_as_float(__float_as_uint(x) & 0xffffe000u);
  *hi = h;
  *lo = x - h;
}

}  // namespace sns
