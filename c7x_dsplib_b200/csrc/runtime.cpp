// Runtime plumbing shared by the FIR and biquad entry points: error text on the
// handle, device/host pointer classification, staging of host buffers through
// per-thread device scratch, and the DSPLIB_gpu_* extension functions.
#include <atomic>
#include <cstdarg>
#include <cstring>

#include "dsplib_internal.h"

namespace dsplib {

static std::atomic<int64_t> g_launches{0};

void countLaunch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void setError(HandleCommon *h, const char *fmt, ...)
{
   if (!h) return;
   va_list ap;
   va_start(ap, fmt);
   vsnprintf(h->err, sizeof(h->err), fmt, ap);
   va_end(ap);
}

DSPLIB_STATUS cudaFail(HandleCommon *h, cudaError_t e, const char *what)
{
   setError(h, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
   return DSPLIB_ERR_FAILURE;
}

bool isDevicePtr(const void *p)
{
   cudaPointerAttributes attr;
   cudaError_t e = cudaPointerGetAttributes(&attr, p);
   if (e != cudaSuccess) {
      (void) cudaGetLastError();
      return false;
   }
   return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
}

// Device-side address of page-locked (pinned) host memory, nullptr otherwise.
static void *pinnedDevicePtr(const void *p)
{
   cudaPointerAttributes attr;
   if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
      (void) cudaGetLastError();
      return nullptr;
   }
   return attr.type == cudaMemoryTypeHost ? attr.devicePointer : nullptr;
}

void *mappedHostPtr(const void *p) { return pinnedDevicePtr(p); }

namespace {
constexpr int kMaxDevices = 16;
constexpr int kSlots = 6;
struct Scratch {
   void *ptr[kMaxDevices][kSlots] = {};
   size_t cap[kMaxDevices][kSlots] = {};
};
thread_local Scratch t_scratch;
} // namespace

void *stagingBuffer(int slot, size_t bytes)
{
   int dev = 0;
   if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices || slot < 0 || slot >= kSlots)
      return nullptr;
   if (bytes == 0) bytes = 16;
   if (t_scratch.cap[dev][slot] < bytes) {
      if (t_scratch.ptr[dev][slot]) cudaFree(t_scratch.ptr[dev][slot]);
      t_scratch.ptr[dev][slot] = nullptr;
      t_scratch.cap[dev][slot] = 0;
      size_t want = bytes + bytes / 4; // grow with headroom
      void *p = nullptr;
      if (cudaMalloc(&p, want) != cudaSuccess) {
         (void) cudaGetLastError();
         return nullptr;
      }
      t_scratch.ptr[dev][slot] = p;
      t_scratch.cap[dev][slot] = want;
   }
   return t_scratch.ptr[dev][slot];
}

cudaError_t regionIn(Region &r, int slot, bool copyIn, cudaStream_t s)
{
   r.staged = false;
   r.onHost = false;
   r.dev = r.host;
   if (r.height == 0 || r.width == 0) return cudaSuccess;
   if (isDevicePtr(r.host)) return cudaSuccess;
   r.onHost = true;
   // Small pinned buffers (coefficients, states, taps) are read and written in place by
   // the kernels: a staging copy each way would cost more than the few accesses.  So are
   // pinned buffers of any size that a kernel streams through once in whole rows: its
   // loads and stores cross PCIe as the copy engines' would, in both directions at once,
   // and overlap the kernel's own work.
   if (r.zeroCopy && (r.streamed || r.bytes() <= kZeroCopyMaxBytes)) {
      if (void *d = pinnedDevicePtr(r.host)) {
         r.dev = d;
         return cudaSuccess;
      }
   }
   void *buf = stagingBuffer(slot, r.bytes());
   if (!buf) return cudaErrorMemoryAllocation;
   r.dev = buf;
   r.staged = true;
   if (!copyIn) return cudaSuccess;
   if (r.pitch <= r.width || r.height == 1)
      return cudaMemcpyAsync(buf, r.host, r.bytes(), cudaMemcpyHostToDevice, s);
   return cudaMemcpy2DAsync(buf, r.pitch, r.host, r.pitch, r.width, r.height, cudaMemcpyHostToDevice, s);
}

cudaError_t regionOut(const Region &r, cudaStream_t s)
{
   if (!r.staged || r.height == 0 || r.width == 0) return cudaSuccess;
   if (r.pitch <= r.width || r.height == 1)
      return cudaMemcpyAsync(r.host, r.dev, r.bytes(), cudaMemcpyDeviceToHost, s);
   return cudaMemcpy2DAsync(r.host, r.pitch, r.dev, r.pitch, r.width, r.height, cudaMemcpyDeviceToHost, s);
}

PipeContext *pipeContext()
{
   static thread_local PipeContext ctx[kMaxDevices];
   int dev = 0;
   if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
   PipeContext &c = ctx[dev];
   if (!c.ready) {
      bool ok = cudaStreamCreateWithFlags(&c.in, cudaStreamNonBlocking) == cudaSuccess &&
                cudaStreamCreateWithFlags(&c.comp, cudaStreamNonBlocking) == cudaSuccess &&
                cudaStreamCreateWithFlags(&c.out, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&c.start, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreateWithFlags(&c.done, cudaEventDisableTiming) == cudaSuccess;
      for (int b = 0; ok && b < kPipeMaxBlocks; b++)
         ok = cudaEventCreateWithFlags(&c.copied[b], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&c.computed[b], cudaEventDisableTiming) == cudaSuccess;
      if (!ok) {
         (void) cudaGetLastError();
         return nullptr;
      }
      c.ready = true;
   }
   return &c;
}

DSPLIB_STATUS pipeFail(HandleCommon *h, PipeContext *pc, cudaError_t e, const char *what)
{
   if (pc) {
      (void) cudaStreamSynchronize(pc->in);
      (void) cudaStreamSynchronize(pc->comp);
      (void) cudaStreamSynchronize(pc->out);
   }
   return cudaFail(h, e, what);
}

cudaError_t copyRows(void *dst, const void *src, size_t width, size_t rows, size_t pitch, cudaMemcpyKind kind,
                     cudaStream_t s)
{
   if (rows == 0 || width == 0) return cudaSuccess;
   if (pitch <= width || rows == 1) return cudaMemcpyAsync(dst, src, (rows - 1) * pitch + width, kind, s);
   return cudaMemcpy2DAsync(dst, pitch, src, pitch, width, rows, kind, s);
}

static HandleCommon *common(DSPLIB_kernelHandle h)
{
   if (!h) return nullptr;
   HandleCommon *c = (HandleCommon *) h;
   switch (c->magic) {
   case kMagicFir:
   case kMagicBiquad:
   case kMagicFltoq15:
   case kMagicQ15tofl:
   case kMagicInterleave:
   case kMagicDeinterleave:
   case kMagicAddNCh: break;
   default: return nullptr;
   }
   return c;
}

} // namespace dsplib

using namespace dsplib;

extern "C" {

DSPLIB_STATUS DSPLIB_gpu_setStream(DSPLIB_kernelHandle handle, void *stream)
{
   HandleCommon *c = common(handle);
   if (!c) return DSPLIB_ERR_NULL_POINTER;
   c->stream = (cudaStream_t) stream;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_setAsync(DSPLIB_kernelHandle handle, int32_t async)
{
   HandleCommon *c = common(handle);
   if (!c) return DSPLIB_ERR_NULL_POINTER;
   c->async = async <= 0 ? 0 : (async >= 2 ? 2 : 1);
   return DSPLIB_SUCCESS;
}

const char *DSPLIB_gpu_lastError(DSPLIB_kernelHandle handle)
{
   HandleCommon *c = common(handle);
   if (!c) return "invalid or uninitialised handle";
   return c->err;
}

DSPLIB_STATUS DSPLIB_gpu_firSetPrecision(DSPLIB_kernelHandle handle, int32_t precision)
{
   HandleCommon *c = common(handle);
   if (!c || c->magic != kMagicFir) return DSPLIB_ERR_NULL_POINTER;
   if (precision != DSPLIB_GPU_FIR_SIMT && precision != DSPLIB_GPU_FIR_BF16X3) return DSPLIB_ERR_INVALID_VALUE;
   c->firPrecision = precision;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_firSetQMode(DSPLIB_kernelHandle handle, int32_t enable)
{
   HandleCommon *c = common(handle);
   if (!c || c->magic != kMagicFir) return DSPLIB_ERR_NULL_POINTER;
   c->firQMode = enable ? 1 : 0;
   return DSPLIB_SUCCESS;
}

int64_t DSPLIB_gpu_kernelLaunchCount(void) { return g_launches.load(); }

DSPLIB_STATUS DSPLIB_gpu_releaseHandle(DSPLIB_kernelHandle handle)
{
   HandleCommon *c = common(handle);
   if (!c) return DSPLIB_ERR_NULL_POINTER;
   // Work queued by an asynchronous exec may still read buffers the caller is about to free.
   const cudaError_t e = c->async ? cudaStreamSynchronize(c->stream) : cudaSuccess;
   c->magic = 0;
   return e == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

} // extern "C"
