// Allocation-free forward transform: sns_forward_r2c_noalloc.
//
// The same three passes as sns_forward_r2c (x r2c, y, z on the half spectrum, then the
// expansion to the reference's full layout), for callers that must not have a library
// allocate device memory behind their back: applications that reserve the GPU's memory
// up front and hand it out from their own pool, codes that run close to the HBM limit,
// and loops that cannot afford the device-wide synchronisation cudaMalloc / cudaFree may
// cause.  The caller passes device input and output; the intermediate half spectrum and
// the twiddle tables live in one file-scope __device__ array of fixed size, so every
// GPU that loads the library holds that array (about 2.5 MiB) until the process exits.
//
// Limits and sharing:
//   * grids up to N = kMaxN (64); larger N is rejected with SNS_ERR_UNSUPPORTED;
//   * the array is shared by every call on a device and keeps the previous call's
//     contents; each call clears its work region before use.  Calls whose GPU work
//     overlaps (other host threads, or other streams) race on it;
//   * the first call on a device does the set-up (symbol address, twiddle upload,
//     kernel attributes) with that device current;
//   * every call returns only after its work on the stream finished (it synchronises the
//     stream), so a call on a stream that is being captured is refused with
//     SNS_ERR_INVALID before anything is enqueued.
#include "sns_kernels.cuh"
#include "../../include/sns_b200.h"

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

namespace {

constexpr int kMaxN = SNS_NOALLOC_MAX_N;
constexpr int kSizes[] = {8, 12, 16, 24, 32, 48, 64};  // FFT plans with N <= kMaxN
constexpr int kNumSizes = sizeof(kSizes) / sizeof(kSizes[0]);
constexpr int kMaxDevices = 64;

constexpr long long field_elems(int n) { return (long long)n * n * ((n / 2 + 1 + 7) / 8 * 8); }
constexpr int twiddle_total() {
  int t = 0;
  for (int i = 0; i < kNumSizes; ++i) t += kSizes[i];
  return t;
}
// Layout of the array (double2 elements): [half-spectrum work field][twiddles of each N].
constexpr long long kFieldElems = field_elems(kMaxN);
constexpr long long kScratchElems = kFieldElems + twiddle_total();

static_assert(kFieldElems % 16 == 0, "twiddle region stays 256-byte aligned");

static __device__ __align__(256) double2 g_noalloc_scratch[kScratchElems];

struct DeviceSlot {
  bool ready = false;
  double2* base = nullptr;  // device address of g_noalloc_scratch on this device
};

std::mutex g_setup_mu;
DeviceSlot g_slots[kMaxDevices];

int twiddle_offset(int n) {
  int off = 0;
  for (int i = 0; i < kNumSizes; ++i) {
    if (kSizes[i] == n) return off;
    off += kSizes[i];
  }
  return -1;
}

int fail(int code, const char* msg) {
  sns::set_handleless_error(msg);
  return code;
}

int fail_cuda(const char* what, cudaError_t e) {
  char buf[256];
  std::snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
  sns::set_handleless_error(buf);
  return SNS_ERR_CUDA;
}

// Once per device, with that device current: look up the array's device address (its
// name in host code is only a host-side stand-in), upload the twiddle tables and set the
// kernel attributes of every plan that fits.
int setup_device(int dev, double2** base) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceSlot& s = g_slots[dev];
  if (!s.ready) {
    double2* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress((void**)&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda("cudaGetSymbolAddress", e);
    double2 tw[twiddle_total()];
    int off = 0;
    for (int i = 0; i < kNumSizes; ++i) {
      sns::fill_twiddles(kSizes[i], tw + off);
      off += kSizes[i];
      sns::ops_for(kSizes[i])->init();
    }
    const cudaError_t c = cudaMemcpy(p + kFieldElems, tw, sizeof tw, cudaMemcpyHostToDevice);
    if (c != cudaSuccess) return fail_cuda("twiddle upload", c);
    s.base = p;
    s.ready = true;
  }
  *base = s.base;
  return SNS_OK;
}

using GetAddressRange = PFN_cuMemGetAddressRange_v3020;

// The driver's cuMemGetAddressRange, looked up once (a function-local static: its
// initialisation is thread-safe); null when the driver does not export it.
GetAddressRange address_range_fn() {
  static const GetAddressRange fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess) {
      cudaGetLastError();
      return GetAddressRange(nullptr);
    }
    return reinterpret_cast<GetAddressRange>(p);
  }();
  return fn;
}

// A caller's buffer must be device (or managed) memory of the current device, with
// `bytes` inside one allocation, before any kernel touches it.
int check_device_buffer(const void* ptr, size_t bytes, size_t align, int dev, const char* name) {
  char buf[256];
  if (reinterpret_cast<uintptr_t>(ptr) % align != 0) {
    std::snprintf(buf, sizeof buf, "%s: must be %zu-byte aligned", name, align);
    return fail(SNS_ERR_INVALID, buf);
  }
  cudaPointerAttributes a{};
  const cudaError_t e = cudaPointerGetAttributes(&a, ptr);
  if (e != cudaSuccess) {
    cudaGetLastError();
    std::snprintf(buf, sizeof buf, "%s: not a CUDA pointer (%s)", name, cudaGetErrorString(e));
    return fail(SNS_ERR_INVALID, buf);
  }
  if ((a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) || a.device != dev) {
    std::snprintf(buf, sizeof buf, "%s: must be device memory of the current device %d", name, dev);
    return fail(SNS_ERR_INVALID, buf);
  }
  // without the size check the kernels could write past the caller's allocation: refuse
  GetAddressRange range = address_range_fn();
  if (range == nullptr)
    return fail(SNS_ERR_UNSUPPORTED, "cuMemGetAddressRange is not available from the driver: buffer sizes "
                                     "cannot be checked");
  CUdeviceptr base = 0;
  size_t size = 0;
  if (range(&base, &size, (CUdeviceptr)ptr) != CUDA_SUCCESS) {
    std::snprintf(buf, sizeof buf, "%s: cuMemGetAddressRange failed", name);
    return fail(SNS_ERR_INVALID, buf);
  }
  if ((CUdeviceptr)ptr + bytes > base + size) {
    std::snprintf(buf, sizeof buf, "%s: allocation holds %zu bytes from this pointer, %zu needed", name,
                  (size_t)(base + size - (CUdeviceptr)ptr), bytes);
    return fail(SNS_ERR_INVALID, buf);
  }
  return SNS_OK;
}

}  // namespace

extern "C" int sns_forward_r2c_noalloc(int n, const double* dev_physical, double* dev_spectral, void* stream) {
  if (n <= 0 || dev_physical == nullptr || dev_spectral == nullptr)
    return fail(SNS_ERR_INVALID, "sns_forward_r2c_noalloc: n must be positive and both buffers non-null");
  if (n > kMaxN || twiddle_offset(n) < 0) {
    char buf[160];
    std::snprintf(buf, sizeof buf,
                  "sns_forward_r2c_noalloc: grid size %d is not supported (static scratch holds N <= %d; "
                  "sizes 8 12 16 24 32 48 64)", n, kMaxN);
    return fail(SNS_ERR_UNSUPPORTED, buf);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(SNS_ERR_NO_DEVICE, "no CUDA device visible");
  }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_cuda("cudaGetDevice", e);
  if (dev < 0 || dev >= kMaxDevices) return fail(SNS_ERR_UNSUPPORTED, "device ordinal beyond the static slots");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  {
    // the call ends with a stream synchronisation, which a capturing stream cannot take
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cs);
    if (e != cudaSuccess) return fail_cuda("sns_forward_r2c_noalloc: stream", e);
    if (cs != cudaStreamCaptureStatusNone)
      return fail(SNS_ERR_INVALID, "sns_forward_r2c_noalloc: the stream is being captured; the call synchronises "
                                   "its stream and cannot be recorded into a graph");
    // a caller's stream must belong to the current device, like the buffers
    if (st != nullptr) {
      int sdev = -1;
      e = cudaStreamGetDevice(st, &sdev);
      if (e != cudaSuccess) return fail_cuda("sns_forward_r2c_noalloc: stream", e);
      if (sdev != dev) return fail(SNS_ERR_INVALID, "sns_forward_r2c_noalloc: the stream belongs to another device");
    }
  }
  const size_t np = (size_t)n * n * n;
  int rc = check_device_buffer(dev_physical, np * sizeof(double), sizeof(double), dev, "dev_physical");
  if (rc != SNS_OK) return rc;
  rc = check_device_buffer(dev_spectral, 2 * np * sizeof(double), sizeof(double2), dev, "dev_spectral");
  if (rc != SNS_OK) return rc;
  double2* base = nullptr;
  rc = setup_device(dev, &base);
  if (rc != SNS_OK) return rc;

  const sns::Ops* ops = sns::ops_for(n);
  const sns::Geom g{n, n / 2, sns::pitch_for(n), (long long)n * n * sns::pitch_for(n)};
  double2* work = base;
  const double2* tw = base + kFieldElems + twiddle_offset(n);
  const int tiles = g.pitch / 8;  // Nyquist column and padding included, as sns_forward_r2c
  e = cudaMemsetAsync(work, 0, (size_t)g.field * sizeof(double2), st);
  if (e != cudaSuccess) return fail_cuda("sns_forward_r2c_noalloc: clear", e);
  ops->xpass_r2c(dev_physical, work, 1, tw, g, st);
  ops->ypass(work, 1, -1, tiles, tw, g, st);
  ops->zpass(work, work, 1, -1, tiles, 1.0, tw, g, st);
  sns::launch_half_to_full(work, SNS_PRECISION_FP64, reinterpret_cast<double2*>(dev_spectral), g, st);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_cuda("sns_forward_r2c_noalloc: launch", e);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return fail_cuda("sns_forward_r2c_noalloc", e);
  return SNS_OK;
}
