// Test hooks of the failure paths (no counterpart in the reference).  They exercise the
// bounded device waits and the device error word without faulting, trapping or hanging a
// GPU: the wait that runs out is on a barrier that nothing will complete, with a short
// poll limit, and the error word is written by the host.
#include "sns_kernels.cuh"
#include "sns_tma.cuh"
#include "../../include/sns_b200.h"

#include <cuda_runtime.h>

#include <cstdio>

namespace {

// One thread arms a shared-memory barrier for 16 bytes that no copy will deliver (nothing is
// in flight), polls it `limit` times as the pass kernels poll their TMA tiles, and records
// whether the wait ran out; the barrier is invalidated before the CTA leaves.
__global__ void k_bounded_wait_probe(uint32_t limit, int* status) {
  __shared__ uint64_t bar;
  if (threadIdx.x != 0) return;
  sns::mbar_init(&bar, 1);
  sns::fence_mbar_init();
  sns::mbar_arrive_expect_tx(&bar, 16);
  const bool landed = sns::mbar_wait_bounded(&bar, 0, limit);
  *status = landed ? sns::kErrNone : sns::kErrTmaTimeout;
  sns::mbar_inval(&bar);
}

}  // namespace

extern "C" int sns_debug_bounded_wait(unsigned polls, int* status) {
  if (status == nullptr || polls == 0 || polls > (1u << 22)) {
    sns::set_handleless_error("sns_debug_bounded_wait: status must be non-null and polls in [1, 2^22]");
    return SNS_ERR_INVALID;
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    sns::set_handleless_error("no CUDA device visible");
    return SNS_ERR_NO_DEVICE;
  }
  int* d = nullptr;
  cudaError_t e = cudaMalloc((void**)&d, sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(d, 0xff, sizeof(int));
  if (e == cudaSuccess) {
    k_bounded_wait_probe<<<1, 32>>>(polls, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(status, d, sizeof(int), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) {
    char buf[200];
    std::snprintf(buf, sizeof buf, "sns_debug_bounded_wait: %s", cudaGetErrorString(e));
    sns::set_handleless_error(buf);
    return SNS_ERR_CUDA;
  }
  return SNS_OK;
}

extern "C" int sns_debug_bounds(long long* count, int* line, long long* index) {
  if (count == nullptr) {
    sns::set_handleless_error("sns_debug_bounds: count must be non-null");
    return SNS_ERR_INVALID;
  }
  long long r[3] = {0, 0, 0};
  const int e = sns::bounds_record(r);
  if (e != 0) {
    char buf[200];
    std::snprintf(buf, sizeof buf, "sns_debug_bounds: %s", cudaGetErrorString((cudaError_t)e));
    sns::set_handleless_error(buf);
    return SNS_ERR_CUDA;
  }
  *count = r[0];
  if (line) *line = (int)r[1];
  if (index) *index = r[2];
  return SNS_OK;
}
