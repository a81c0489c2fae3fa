// ontc_lanczos_down_noalloc: the Lanczos-3 2x mip reduction (the kernels of mips.cu, the
// reduction upstream runs per mip in ntc_kernel.cu:533-620) on a caller's DEVICE image,
// allocating nothing.
//
// Who needs it: callers that must not allocate device memory where they reduce a mip.
//  * A host application whose device memory is owned by its own pool (a framework's caching
//    allocator, a texture streamer with a fixed budget): a cudaMalloc outside the pool can
//    fail or fragment what the pool has reserved.
//  * A caller that must not stall its other streams: cudaFree synchronises the whole device,
//    and the allocating entry point (ontc_debug_lanczos_down) allocates and frees its
//    buffers on every call.
//
// How: the x pass's fp32 intermediate, [dim][dim/2][ch] floats, lives in one file-scope
// device array per device (8 MiB).  The x pass writes every element the y pass reads, so
// the array needs no initial contents.  The caller owns source and destination.
#include <mutex>

#include "common.cuh"
#include "kernels.h"
#include "ontc.h"

namespace {

static __device__ __align__(256) float g_lanczos_scratch[ONTC_NOALLOC_SCRATCH_FLOATS];

constexpr int kMaxDevices = 64;

// Device address of the scratch array on the current device, looked up once per device
// (cudaGetSymbolAddress with that device current).
cudaError_t scratch_address(float** out)
{
  static std::mutex mu;
  static float* addr[kMaxDevices] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_lanczos_scratch);
    if (e != cudaSuccess) return e;
    addr[dev] = static_cast<float*>(p);
  }
  *out = addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" int ontc_lanczos_down_noalloc(const uint8_t* d_src, int32_t dim, int32_t ch, uint8_t* d_dst, void* stream)
{
  if (!d_src || !d_dst || dim < 2 || ch < 1 || ch > 4) return ONTC_INVALID_DIMENSION;
  // the intermediate must fit the fixed scratch: refuse before touching the device
  if ((unsigned long long)dim * (unsigned long long)(dim / 2) * (unsigned long long)ch > ONTC_NOALLOC_SCRATCH_FLOATS)
    return ONTC_INVALID_DIMENSION;
  float* tmp = nullptr;
  if (scratch_address(&tmp) != cudaSuccess) return ONTC_CUDA_FAILURE;
  // clear a launch error left by earlier, unrelated work, so the status below is this call's
  // (a sticky error from a faulted context cannot be cleared and is still reported)
  (void)cudaGetLastError();
  cudaError_t e = ontc::launch_lanczos_down(d_src, dim, ch, tmp, d_dst, static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? ONTC_SUCCESS : ONTC_CUDA_FAILURE;
}
