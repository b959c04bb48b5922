// Tensor-core DFT sub-block: batched 16-point complex DFTs as tcgen05.mma kind::tf32 with the
// 3xTF32 split (no counterpart in the reference, which has no tensor-core code).
//
// A DFT of length 16 on complex values is a real GEMM: with x packed as 32 reals (re, im
// interleaved), y = B x with B[2p][2q] = c, B[2p][2q+1] = -s, B[2p+1][2q] = s,
// B[2p+1][2q+1] = c, (c, s) = (cos, sin) of -2 pi p q / 16.  A tile of 128 sequences is the
// M = 128 operand A (K = 32, K-major in shared memory), B is the N = 32 operand, and the
// accumulator is 128 lanes x 32 columns of tensor memory.  FP32 accuracy comes from the
// 3xTF32 split: A = A_hi + A_lo and B = B_hi + B_lo (hi = the 10 mantissa bits the tensor core
// reads), D = A_hi B_hi + A_hi B_lo + A_lo B_hi, twelve MMAs of K = 8 per tile.
//
// The register butterflies (dft16 in sns_fft.cuh) run the same batch for comparison.  This
// block is not on the solver's path: the x pass that would host it is bound by its
// shared-memory pipe, and the MMA operands need a hi/lo copy of every input in shared memory
// (the measured figures are in the design notes).
#include "sns_fft.cuh"
#include "sns_kernels.cuh"
#include "sns_umma.cuh"
#include "../../include/sns_b200.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <vector>

namespace {

constexpr int kL = 16;        // DFT length
constexpr int kK = 2 * kL;    // real K
constexpr int kTile = 128;    // sequences per MMA tile (M)
constexpr int kABytes = kTile * kK * 4;  // one TF32 copy of A
constexpr int kBBytes = kK * kK * 4;     // one TF32 copy of B
constexpr size_t kSmem = 2 * kABytes + 2 * kBBytes + 1024;

// out[s] = DFT16(in[s]) (sign -1) for count sequences (count a multiple of 128); bmat: the
// 32 x 32 real DFT matrix, row n = output component, K contiguous.  err: bounded-wait expiry.
__global__ void __launch_bounds__(128) k_dft16_tc(const float* __restrict__ in, float* __restrict__ out,
                                                   const float* __restrict__ bmat, int tiles, int* err) {
  extern __shared__ unsigned char smraw[];
  __shared__ uint64_t bar;
  __shared__ uint32_t s_tmem;
  __shared__ int s_fail;
  const uint32_t pad = (1024u - (sns::smem_u32(smraw) & 1023u)) & 1023u;
  unsigned char* Ahi = smraw + pad;
  unsigned char* Alo = Ahi + kABytes;
  unsigned char* Bhi = Alo + kABytes;
  unsigned char* Blo = Bhi + kBBytes;
  const int tid = threadIdx.x, warp = tid >> 5;
  for (int i = tid; i < kK * kK; i += kTile) {
    const int n = i / kK, k = i % kK;
    float h, l;
    sns::tf32_split(bmat[i], &h, &l);
    *reinterpret_cast<float*>(Bhi + sns::umma_kmajor_offset(n, k, kK)) = h;
    *reinterpret_cast<float*>(Blo + sns::umma_kmajor_offset(n, k, kK)) = l;
  }
  if (tid == 0) {
    sns::mbar_init(&bar, 1);
    sns::fence_mbar_init();
    s_fail = 0;
  }
  if (warp == 0) {
    sns::tmem_alloc(&s_tmem, 32);
    sns::tmem_relinquish();
  }
  sns::tc_fence_before();
  __syncthreads();
  sns::tc_fence_after();
  const uint32_t d = s_tmem;
  const uint32_t idesc = sns::umma_idesc_tf32(kTile, kK);
  const uint32_t a_hi = sns::smem_u32(Ahi), a_lo = sns::smem_u32(Alo);
  const uint32_t b_hi = sns::smem_u32(Bhi), b_lo = sns::smem_u32(Blo);
  constexpr uint32_t kSbo = (kK / 4) * 128;
  int k = 0;
  for (int t = blockIdx.x; t < tiles; t += gridDim.x, ++k) {
    const long long s = (long long)t * kTile + tid;  // this thread's sequence and A row
    const float4* src = reinterpret_cast<const float4*>(in + s * kK);
#pragma unroll
    for (int v = 0; v < kK / 4; ++v) {
      const float4 q = src[v];
      const float e[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float h, l;
        sns::tf32_split(e[j], &h, &l);
        *reinterpret_cast<float*>(Ahi + sns::umma_kmajor_offset(tid, 4 * v + j, kK)) = h;
        *reinterpret_cast<float*>(Alo + sns::umma_kmajor_offset(tid, 4 * v + j, kK)) = l;
      }
    }
    sns::fence_proxy_async_smem();  // the generic-proxy writes of A before the MMAs read it
    sns::tc_fence_before();
    __syncthreads();
    if (tid == 0) {
      sns::tc_fence_after();
#pragma unroll
      for (int kk = 0; kk < kK / 8; ++kk) {
        const uint32_t off = (uint32_t)kk * 2 * 128;
        sns::umma_tf32(d, sns::umma_desc(a_hi + off, 128, kSbo), sns::umma_desc(b_hi + off, 128, kSbo), idesc, kk > 0);
        sns::umma_tf32(d, sns::umma_desc(a_hi + off, 128, kSbo), sns::umma_desc(b_lo + off, 128, kSbo), idesc, true);
        sns::umma_tf32(d, sns::umma_desc(a_lo + off, 128, kSbo), sns::umma_desc(b_hi + off, 128, kSbo), idesc, true);
      }
      sns::umma_commit(&bar);
    }
    if (tid == 0 && !sns::mbar_wait_bounded(&bar, (uint32_t)(k & 1))) s_fail = 1;
    __syncthreads();
    if (s_fail) break;
    (void)sns::mbar_try_wait(&bar, (uint32_t)(k & 1));
    sns::tc_fence_after();
    uint32_t w[kK];
    sns::tmem_ld_words<kK>(d + ((uint32_t)(32 * warp) << 16), w);
    float4* dst = reinterpret_cast<float4*>(out + s * kK);
#pragma unroll
    for (int v = 0; v < kK / 4; ++v)
      dst[v] = make_float4(__uint_as_float(w[4 * v]), __uint_as_float(w[4 * v + 1]), __uint_as_float(w[4 * v + 2]),
                           __uint_as_float(w[4 * v + 3]));
    sns::tc_fence_before();
    __syncthreads();  // every lane read its row before the next tile's MMAs overwrite it
  }
  if (s_fail && tid == 0) {
    atomicExch(err, sns::kErrTmaTimeout);
    // let MMAs still in flight finish before the tensor memory is released
    (void)sns::mbar_wait_bounded(&bar, (uint32_t)(k & 1));
  }
  __syncthreads();
  if (warp == 0) sns::tmem_dealloc(d, 32);
}

// The same batch on the register butterflies (one sequence per thread).
__global__ void __launch_bounds__(128) k_dft16_simt(const float* __restrict__ in, float* __restrict__ out, long long count) {
  for (long long s = (long long)blockIdx.x * 128 + threadIdx.x; s < count; s += (long long)gridDim.x * 128) {
    const float4* src = reinterpret_cast<const float4*>(in + s * kK);
    float2 v[kL];
#pragma unroll
    for (int i = 0; i < kK / 4; ++i) {
      const float4 q = src[i];
      v[2 * i] = make_float2(q.x, q.y);
      v[2 * i + 1] = make_float2(q.z, q.w);
    }
    sns::dft16<-1>(v);
    float4* dst = reinterpret_cast<float4*>(out + s * kK);
#pragma unroll
    for (int i = 0; i < kK / 4; ++i) dst[i] = make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
  }
}

int fail(int code, const char* msg) {
  sns::set_handleless_error(msg);
  return code;
}

}  // namespace

extern "C" int sns_dft16_batch(const float* dev_in, float* dev_out, long long count, int use_tensor_cores,
                               void* stream, double* elapsed_ms) {
  if (!dev_in || !dev_out || count <= 0 || count % kTile != 0 || (use_tensor_cores != 0 && use_tensor_cores != 1))
    return fail(SNS_ERR_INVALID, "sns_dft16_batch: device buffers, count a positive multiple of 128, method 0 or 1");
  if ((reinterpret_cast<uintptr_t>(dev_in) | reinterpret_cast<uintptr_t>(dev_out)) % 16 != 0)
    return fail(SNS_ERR_INVALID, "sns_dft16_batch: buffers must be 16-byte aligned");
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) !=
                                                 cudaSuccess) {
    cudaGetLastError();
    return fail(SNS_ERR_NO_DEVICE, "no CUDA device visible");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the real 32 x 32 DFT matrix, rounded from the exact twiddles
  std::vector<double2> tw(kL);
  sns::fill_twiddles(kL, tw.data());
  std::vector<float> b(kK * kK);
  for (int p = 0; p < kL; ++p)
    for (int q = 0; q < kL; ++q) {
      const double2 w = tw[(p * q) % kL];  // exp(-2 pi i p q / 16)
      b[(2 * p) * kK + 2 * q] = (float)w.x;
      b[(2 * p) * kK + 2 * q + 1] = (float)-w.y;
      b[(2 * p + 1) * kK + 2 * q] = (float)w.y;
      b[(2 * p + 1) * kK + 2 * q + 1] = (float)w.x;
    }
  float* d_b = nullptr;
  int* d_err = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaMalloc((void**)&d_b, b.size() * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc((void**)&d_err, sizeof(int));
  if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, sizeof(int), st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(d_b, b.data(), b.size() * sizeof(float), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_dft16_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmem);
  if (e == cudaSuccess) e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  const int tiles = (int)(count / kTile);
  if (e == cudaSuccess) e = cudaEventRecord(e0, st);
  if (e == cudaSuccess) {
    if (use_tensor_cores) {
      const int grid = tiles < 4 * nsm ? tiles : 4 * nsm;
      k_dft16_tc<<<grid, kTile, kSmem, st>>>(dev_in, dev_out, d_b, tiles, d_err);
    } else {
      const long long blocks = (count + 127) / 128;
      k_dft16_simt<<<(unsigned)(blocks < 16LL * nsm ? blocks : 16LL * nsm), 128, 0, st>>>(dev_in, dev_out, count);
    }
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  int werr = 0;
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaMemcpy(&werr, d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaFree(d_b);
  cudaFree(d_err);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (e != cudaSuccess) {
    char buf[200];
    std::snprintf(buf, sizeof buf, "sns_dft16_batch: %s", cudaGetErrorString(e));
    return fail(SNS_ERR_CUDA, buf);
  }
  if (werr != 0) return fail(SNS_ERR_CUDA, "sns_dft16_batch: a tile's MMAs did not complete within the wait limit");
  if (elapsed_ms) *elapsed_ms = ms;
  return SNS_OK;
}
