// qmcrt_smooth_static: the trimmed-mean smoother without any device
// allocation, for callers that cannot call cudaMalloc.
//
// qmcrt_smooth needs a copy of the image it overwrites and allocates that
// copy (cudaMallocAsync) on every call.  Some callers may not allocate device
// memory at all: code that runs under a fixed device-memory budget because a
// framework's caching allocator has already reserved the memory, or a
// real-time loop in which the latency or the possible failure of an
// allocation is not acceptable.  This entry point keeps the copy in a
// statically sized device array instead, g_smooth_scratch below: 4,194,304
// floats (16 MiB), which every GPU that loads the library holds until the
// process exits.
//
// The kernel needs the array's device address.  In host code the symbol
// g_smooth_scratch is only a host-side stand-in, not a device address, so it
// must not be passed to a kernel; the address is obtained with
// cudaGetSymbolAddress, once per device, with that device current, on the
// first call made on that device, and cached.  Make that first call before
// any stream capture begins.
//
// Every call shares the one array and leaves its copy of the last image in
// it.  Nothing in it needs to start at zero: each call first copies its
// whole input image into it.  Calls whose work overlaps on the GPU (different
// streams, or different host threads) race on the array; order them.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "qmcrt.h"
#include "smooth.h"

namespace qm {
// Sets the message qmcrt_last_error() returns on this thread (capi.cpp).
void set_last_error(const std::string& msg);
}  // namespace qm

// The scratch array: file scope, 4,194,304 floats (16 MiB) per GPU.
static __device__ __align__(256) float g_smooth_scratch[4194304];

namespace {

constexpr long long kStaticSmoothPixels = 4194304;

constexpr int kMaxDevices = 64;
std::mutex g_addr_mutex;
float* g_addr[kMaxDevices] = {nullptr};

int fail(int code, const std::string& msg) {
  qm::set_last_error(msg);
  return code;
}

}  // namespace

extern "C" int qmcrt_smooth_static(float* device_image, int width, int height, int radius, float trim_ratio,
                                   void* stream) {
  if (!device_image) return fail(QMCRT_ERR_INVALID, "image is NULL");
  if (width <= 0 || height <= 0) return fail(QMCRT_ERR_INVALID, "image size must be positive");
  if (radius < 0 || radius > 64) return fail(QMCRT_ERR_INVALID, "radius must be in [0, 64]");
  if (!(trim_ratio >= 0.0f && trim_ratio < 0.5f)) return fail(QMCRT_ERR_INVALID, "trim ratio must be in [0, 0.5)");
  const long long pixels = (long long)width * height;
  if (pixels > kStaticSmoothPixels)
    return fail(QMCRT_ERR_INVALID, "image of " + std::to_string(pixels) +
                                       " pixels exceeds the static scratch of 4194304 pixels (16 MiB)");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(QMCRT_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(QMCRT_ERR_INVALID, "device index beyond 63");
  float* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_addr_mutex);
    if (!g_addr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_smooth_scratch);
      if (e != cudaSuccess)
        return fail(QMCRT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_addr[dev] = static_cast<float*>(p);
    }
    scratch = g_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = cudaMemcpyAsync(scratch, device_image, (size_t)pixels * sizeof(float), cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess) e = qm::launch_trimmed_mean(scratch, device_image, width, height, radius, trim_ratio, st);
  if (e != cudaSuccess) return fail(QMCRT_ERR_CUDA, std::string("trimmed mean: ") + cudaGetErrorString(e));
  qm::set_last_error(std::string());
  return QMCRT_OK;
}
