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
//   * The array's device address is looked up (cudaGetSymbolAddress, with the
//     plan's device current) on every call made outside stream capture, so it stays
//     valid after a cudaDeviceReset; a call made while its stream is being captured
//     uses the address the last call outside capture found.  So the first call on a
//     device must come before any stream capture begins.
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
float *g_scratchAddr[kMaxDevices]; // device address of g_staticScratch per device, from the last lookup

// Device address of the scratch array on `dev` (the current device).  Looked up on
// every call outside stream capture; a captured call reuses the last lookup.
cudaError_t staticScratch(int dev, cudaStream_t stream, float **out)
{
   if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
   cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
   cudaError_t e = cudaStreamIsCapturing(stream, &cs);
   if (e != cudaSuccess) return e;
   std::lock_guard<std::mutex> lock(g_scratchMutex);
   if (cs == cudaStreamCaptureStatusNone) {
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_staticScratch);
      if (e != cudaSuccess) return e;
      g_scratchAddr[dev] = (float *) p;
   }
   else if (!g_scratchAddr[dev])
      return cudaErrorStreamCaptureUnsupported; // first call on this device made under capture
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
   // the lookup needs the plan's device current: switch to it for the call
   const int dev = dsplib::raggedPlanDevice(plan);
   int prev = 0;
   if (cudaGetDevice(&prev) != cudaSuccess) return DSPLIB_ERR_FAILURE;
   if (prev != dev && cudaSetDevice(dev) != cudaSuccess) return DSPLIB_ERR_FAILURE;
   float *scratch = nullptr;
   DSPLIB_STATUS st = DSPLIB_ERR_FAILURE;
   if (dsplib::staticScratch(dev, (cudaStream_t) stream, &scratch) == cudaSuccess)
      st = DSPLIB_gpu_firBiquadBatched_bwd(plan, x, taps, coefs, work, gy, gx, gtaps, gcoefs, scratch, stream);
   if (prev != dev) (void) cudaSetDevice(prev);
   return st;
}
