// Runtime plumbing shared by the FIR and biquad entry points: error text on the
// handle, device/host pointer classification, staging of host buffers through
// per-thread device scratch, and the DSPLIB_gpu_* extension functions.
#include <atomic>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <vector>

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

// ---------------------------------------------------------------- error words

namespace {
constexpr int kErrWords = 4096;
std::mutex g_errMutex;
int *g_errPool = nullptr;  // mapped, portable page-locked words
std::vector<int> g_errFree; // free slots
int g_errNext = 1;          // slot 0 is shared by handles once the pool is exhausted

bool errPool()
{
   if (g_errPool) return true;
   void *p = nullptr;
   if (cudaHostAlloc(&p, kErrWords * sizeof(int), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
      (void) cudaGetLastError();
      return false;
   }
   std::memset(p, 0, kErrWords * sizeof(int));
   g_errPool = (int *) p;
   return true;
}

int takeSlot()
{
   if (!g_errFree.empty()) {
      const int k = g_errFree.back();
      g_errFree.pop_back();
      return k;
   }
   return g_errNext < kErrWords ? g_errNext++ : 0;
}
} // namespace

int *errorWord(HandleCommon *h)
{
   std::lock_guard<std::mutex> lock(g_errMutex);
   if (!errPool()) return nullptr;
   if (h->errSlot == 0) {
      h->errSlot = 1 + takeSlot();
      g_errPool[h->errSlot - 1] = 0;
   }
   return g_errPool + (h->errSlot - 1);
}

void releaseErrorWord(HandleCommon *h)
{
   std::lock_guard<std::mutex> lock(g_errMutex);
   if (h->errSlot > 1) g_errFree.push_back(h->errSlot - 1);
   h->errSlot = 0;
}

int takeErrorWord(HandleCommon *h)
{
   if (h->errSlot == 0 || !g_errPool) return 0;
   volatile int *w = g_errPool + (h->errSlot - 1);
   const int v = *w;
   if (v) *w = 0;
   return v;
}

int *allocErrorWord()
{
   std::lock_guard<std::mutex> lock(g_errMutex);
   if (!errPool()) return nullptr;
   const int k = takeSlot();
   g_errPool[k] = 0;
   return g_errPool + k;
}

void freeErrorWord(int *w)
{
   std::lock_guard<std::mutex> lock(g_errMutex);
   if (w && g_errPool && w > g_errPool && w < g_errPool + kErrWords) g_errFree.push_back((int) (w - g_errPool));
}

// ---------------------------------------------------------------- fault injection

namespace {
thread_local int t_injectLeft = 0;
}

void injectArm(HandleCommon *h)
{
   t_injectLeft = h ? h->injectAt : 0;
   if (h) h->injectAt = 0; // one call
}

void injectDisarm() { t_injectLeft = 0; }

cudaError_t injectCheck(cudaError_t e)
{
   if (e != cudaSuccess || t_injectLeft <= 0) return e;
   return --t_injectLeft == 0 ? cudaErrorUnknown : cudaSuccess;
}

// Wait for what is already queued on s (copies into or out of the caller's host
// buffers, kernels reading them) unless s is being captured into a graph.
static void drainStream(cudaStream_t s)
{
   cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
   if (cudaStreamIsCapturing(s, &cs) == cudaSuccess && cs == cudaStreamCaptureStatusNone)
      (void) cudaStreamSynchronize(s);
   (void) cudaGetLastError();
}

DSPLIB_STATUS cudaFail(HandleCommon *h, cudaError_t e, const char *what)
{
   setError(h, "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
   // A failing call returns only after the work it already queued has finished, so no
   // copy touches the caller's buffers after the error is reported.
   if (h) drainStream(h->stream);
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
// Staging buffers of one host thread.  They come from the device's stream-ordered
// memory pool (no device-wide synchronisation when one grows) and go back to it
// when the thread exits.
struct Scratch {
   void *ptr[kMaxDevices][kSlots] = {};
   size_t cap[kMaxDevices][kSlots] = {};
   ~Scratch()
   {
      int prev = -1;
      if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
      for (int d = 0; d < kMaxDevices; d++)
         for (int k = 0; k < kSlots; k++)
            if (ptr[d][k] && cudaSetDevice(d) == cudaSuccess) (void) cudaFree(ptr[d][k]);
      if (prev >= 0) (void) cudaSetDevice(prev);
      (void) cudaGetLastError();
   }
};
thread_local Scratch t_scratch;
} // namespace

void *stagingBuffer(int slot, size_t bytes, cudaStream_t s)
{
   int dev = 0;
   if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices || slot < 0 || slot >= kSlots)
      return nullptr;
   if (bytes == 0) bytes = 16;
   if (t_scratch.cap[dev][slot] < bytes) {
      // Every call that staged through this buffer completed before it returned, so the
      // old buffer can go back to the pool in the order of s.
      if (t_scratch.ptr[dev][slot]) (void) cudaFreeAsync(t_scratch.ptr[dev][slot], s);
      t_scratch.ptr[dev][slot] = nullptr;
      t_scratch.cap[dev][slot] = 0;
      size_t want = bytes + bytes / 4; // grow with headroom
      void *p = nullptr;
      if (cudaMallocAsync(&p, want, s) != cudaSuccess) {
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
   void *buf = stagingBuffer(slot, r.bytes(), s);
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

namespace {
// The pipeline streams and events of one host thread, destroyed when it exits.
struct PipeContexts {
   PipeContext ctx[kMaxDevices];
   ~PipeContexts()
   {
      for (PipeContext &c : ctx) {
         if (!c.ready) continue;
         (void) cudaStreamDestroy(c.in);
         (void) cudaStreamDestroy(c.comp);
         (void) cudaStreamDestroy(c.out);
         (void) cudaEventDestroy(c.start);
         (void) cudaEventDestroy(c.done);
         for (int b = 0; b < kPipeMaxBlocks; b++) {
            (void) cudaEventDestroy(c.copied[b]);
            (void) cudaEventDestroy(c.computed[b]);
         }
      }
      (void) cudaGetLastError();
   }
};
thread_local PipeContexts t_pipes;
} // namespace

PipeContext *pipeContext()
{
   PipeContext *ctx = t_pipes.ctx;
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
   releaseErrorWord(c);
   c->magic = 0;
   return e == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

DSPLIB_STATUS DSPLIB_gpu_status(DSPLIB_kernelHandle handle)
{
   HandleCommon *c = common(handle);
   if (!c) return DSPLIB_ERR_NULL_POINTER;
   if (takeErrorWord(c) != 0) {
      setError(c, "a bounded wait for the tensor core expired in an earlier call; its outputs are incomplete");
      return DSPLIB_ERR_FAILURE;
   }
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_injectFault(DSPLIB_kernelHandle handle, int32_t operation)
{
   HandleCommon *c = common(handle);
   if (!c) return DSPLIB_ERR_NULL_POINTER;
   if (operation < 0) return DSPLIB_ERR_INVALID_VALUE;
   c->injectAt = operation;
   return DSPLIB_SUCCESS;
}

} // extern "C"
