// Filter-bank adjoint that allocates nothing: the scratch the adjoint needs
// (running gradient, reverse-time filter output, per-tile partial sums) lives
// in a fixed array compiled into this library instead of a caller buffer.
//
// Who needs this: callers that must not allocate device memory while they run.
// A processing thread with a per-block deadline cannot afford cudaMalloc or
// cudaFree (both can take milliseconds, and cudaFree waits for the whole device
// to go idle); a deployment that reserves all device memory at start-up has no
// allocator to ask; and a caller holding memory through an allocator it does not
// own (a framework's caching pool) may have no way to hand out an extra buffer
// of the right size at that point.  They get the adjoint without any buffer
// beyond its inputs and outputs, within a fixed size limit.
//
// Rules of use:
//   * The scratch is one array per device, shared by every call on that device.
//     Two calls whose executions overlap in time (different streams, or different
//     host threads without ordering) overwrite each other's intermediate results:
//     serialise them (one stream, or event dependencies).
//   * Nothing in the array needs to start at zero: every word the adjoint reads is
//     written earlier in the same call.
//   * The first call on a device looks up the array's device address (one-time
//     set-up, done with that device current); make that first call before any
//     stream capture begins.
//   * Plans whose scratch exceeds the array (DSPLIB_GPU_STATIC_SCRATCH_FLOATS
//     floats) are rejected with DSPLIB_ERR_BUFFER_TOO_SMALL before any work is queued.
#include <cuda_runtime.h>

#include <mutex>

#include "dsplib_internal.h"

namespace dsplib {
namespace {

constexpr int kMaxDevices = 64;

static __device__ __align__(256) float g_staticScratch[DSPLIB_GPU_STATIC_SCRATCH_FLOATS];

std::mutex g_scratchMutex;
float *g_scratchAddr[kMaxDevices]; // device address of g_staticScratch, per device (null until looked up)

// Address of this device's scratch array; looked up once per device (the device must be current).
cudaError_t staticScratch(float **out)
{
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) return e;
   if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
   std::lock_guard<std::mutex> lock(g_scratchMutex);
   if (!g_scratchAddr[dev]) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_staticScratch);
      if (e != cudaSuccess) return e;
      g_scratchAddr[dev] = (float *) p;
   }
   *out = g_scratchAddr[dev];
   return cudaSuccess;
}

} // namespace
} // namespace dsplib

extern "C" DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_bwdStaticScratch(DSPLIB_gpu_raggedPlan plan, const float *x,
                                                                      const float *taps, const float *coefs,
                                                                      const float *work, const float *gy, float *gx,
                                                                      float *gtaps, float *gcoefs, void *stream)
{
   if (!plan) return DSPLIB_ERR_NULL_POINTER;
   const int64_t need = DSPLIB_gpu_raggedPlanSize(plan, DSPLIB_GPU_RAGGED_SCRATCH);
   if (need < 0) return DSPLIB_ERR_FAILURE;
   if (need > (int64_t) DSPLIB_GPU_STATIC_SCRATCH_FLOATS) return DSPLIB_ERR_BUFFER_TOO_SMALL;
   float *scratch = nullptr;
   if (dsplib::staticScratch(&scratch) != cudaSuccess) return DSPLIB_ERR_FAILURE;
   return DSPLIB_gpu_firBiquadBatched_bwd(plan, x, taps, coefs, work, gy, gx, gtaps, gcoefs, scratch, stream);
}
