// Index checks of the debug build (compiled with -DSNS_BOUNDS_CHECK into
// libsns_b200_check.so).  In the TMA / tensor-memory pass kernels every shared-memory,
// tensor-memory and global index of a field, tile or table goes through SNS_IDX(i, n): an
// index outside [0, n) is recorded (the count, and the first one's source line and value, in
// device words the host reads with sns_debug_bounds) and replaced by 0, so the access stays
// inside its buffer.  The normal build compiles SNS_IDX(i, n) to i.
#pragma once

#include <cuda_runtime.h>

namespace sns {

#ifdef SNS_BOUNDS_CHECK
struct BoundsRecord {
  unsigned long long count;
  long long index;
  int line;
};
// one record per translation unit; the pass kernels and sns_debug_bounds share sns_kernels.cu's
static __device__ BoundsRecord g_bounds;
__device__ __forceinline__ long long bounds_checked(long long i, long long n, int line) {
  if (i >= 0 && i < n) return i;
  if (atomicAdd(&g_bounds.count, 1ull) == 0ull) {
    g_bounds.index = i;
    g_bounds.line = line;
  }
  return 0;
}
#define SNS_IDX(i, n) (::sns::bounds_checked((long long)(i), (long long)(n), __LINE__))
#else
#define SNS_IDX(i, n) (i)
#endif

}  // namespace sns
