// The initial placement's BiCGSTAB solve for callers that cannot allocate device memory.
//
// gpl_kernel_bicgstab allocates its scratch vectors with cudaMalloc on every call. Some callers
// cannot do that: code whose device memory is budgeted up front by a pool it must not bypass,
// plug-in hosts that forbid a library from growing the device heap behind their back, and code
// that shares the GPU with latency-critical streams, where cudaMalloc and cudaFree may wait for
// the whole device. This entry point gives them the same solve with
// its scratch in one fixed array of this library's own: a file-scope device array. The CUDA
// driver reserves it when it loads this library's device code on a device: at the first use of
// the library's kernels there under lazy module loading (CUDA's default since 12.2; possibly
// inside the first call below, at cudaGetSymbolAddress), or when the context is made with
// CUDA_MODULE_LOADING=EAGER. It is held on that device until the process exits. A caller that
// budgets device memory or captures streams makes one call (or any launch of this library) on
// each device first.
#include <cstdint>
#include <mutex>

#include "../../../include/gpl.h"
#include "../kernels/bicgstab.h"

namespace {

// The largest system the fixed scratch holds: seven vectors of this many floats (each
// rounded up to 256 bytes), the reduction partials and the solver's scalars.
constexpr int64_t kMaxRows = GPL_BICGSTAB_NOALLOC_MAX_ROWS;
constexpr size_t kVecBytes = ((size_t)kMaxRows * sizeof(float) + 255) / 256 * 256;
constexpr size_t kScratchBytes = 7 * kVecBytes + (size_t)gpl::kBicgBlocks * 3 * sizeof(double) + 64 * sizeof(double);

// In host code this name is only a host-side stand-in for the device array: its address is
// looked up per device with cudaGetSymbolAddress before a kernel is given it.
static __device__ __align__(256) unsigned char g_bicgstab_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
void *g_addr[kMaxDevices] = {};

// The scratch's device address on the current device, looked up once per device, by the first
// call made with that device current; that first call should come before any stream capture.
// The address is kept for the process: after cudaDeviceReset on a device it names freed memory,
// so a caller that resets a device must not call this entry point on it again.
cudaError_t scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_bicgstab_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int gpl_kernel_bicgstab_noalloc(int64_t n, const int64_t *row_start, const int32_t *cols, const float *vals, const float *rhs, float *x, int32_t max_iters, int32_t *iterations, float *error, void *stream) {
  if (n < 0) return (int)cudaErrorInvalidValue;
  if (n > kMaxRows) return GPL_NOALLOC_TOO_LARGE;
  if (gpl::bicgstab_scratch_bytes(n) > kScratchBytes) return GPL_NOALLOC_TOO_LARGE;
  void *scratch = nullptr;
  cudaError_t e = scratch_address(&scratch);
  if (e != cudaSuccess) return (int)e;
  cudaStream_t s = (cudaStream_t)stream;
  gpl::CsrDev A{n, row_start, cols, vals};
  gpl::BicgResult r{};
  // the solve clears the vectors that must start at zero (p and v) itself; every other word
  // of the scratch is written before it is read
  e = gpl::bicgstab_solve(A, rhs, x, max_iters, scratch, s, &r);
  cudaError_t e2 = cudaStreamSynchronize(s);
  *iterations = r.iterations;
  *error = r.error;
  return (int)(e != cudaSuccess ? e : e2);
}
