// C-ABI entry points of DSPLIB_fltoq15 and DSPLIB_q15tofl (reference
// src/DSPLIB_fltoq15/DSPLIB_fltoq15.cpp, src/DSPLIB_q15tofl/DSPLIB_q15tofl.cpp):
// same parameter checks and status codes, conversions on the GPU.
//
// Buffer residency per exec:
//   device memory            read / written in place by the kernel;
//   page-locked host memory  reached by the kernel through its mapped device
//                            address (each byte crosses PCIe once, reads and
//                            writes overlap, no staging buffer);
//   pageable host memory     staged through device buffers; above 8 MB the
//                            array is cut into blocks whose host-to-device copy,
//                            conversion and device-to-host copy overlap on three
//                            streams.
#include <cstring>

#include "dsplib_internal.h"

using namespace dsplib;

namespace {

constexpr size_t kConvPipeMinBytes = 8u << 20;
constexpr size_t kConvPipeBlockBytes = 8u << 20;

Q15Priv *q15Handle(DSPLIB_kernelHandle h, uint32_t magic)
{
   Q15Priv *p = (Q15Priv *) h;
   if (!p || p->common.magic != magic || !p->initialized) return nullptr;
   return p;
}

void q15Reset(Q15Priv *p, uint32_t magic)
{
   if (p->common.magic != magic) {
      std::memset(&p->common, 0, sizeof(p->common));
      p->common.magic = magic;
   }
   p->common.err[0] = 0;
   p->initialized = 0;
}

bool isFloatType(uint32_t t) { return t == DSPLIB_FLOAT32 || t == DSPLIB_FLOAT64; }

// One side of a conversion: where the kernel reads or writes it.
struct Side {
   void *host;  // caller pointer
   void *dev;   // pointer the kernel uses
   size_t elt;  // bytes per element
   bool staged; // pageable host memory, copied through a staging buffer
};

void prepare(Side &sd)
{
   sd.staged = false;
   sd.dev = sd.host;
   if (isDevicePtr(sd.host)) return;
   if (void *m = mappedHostPtr(sd.host)) sd.dev = m;
   else sd.staged = true;
}

// Run launch(in, out, count, stream) over n elements with the residency rules above.
template <typename Launch>
DSPLIB_STATUS convertExec(HandleCommon *hc, void *pIn, size_t eltIn, void *pOut, size_t eltOut, long long n,
                          const char *what, Launch launch)
{
   cudaStream_t s = hc->stream;
   Side in{pIn, nullptr, eltIn, false}, out{pOut, nullptr, eltOut, false};
   prepare(in);
   prepare(out);
   cudaError_t e;
   injectArm(hc);
   struct Disarm {
      ~Disarm() { injectDisarm(); }
   } disarm;
   if (!in.staged && !out.staged) {
      if ((e = injectCheck(launch(in.dev, out.dev, n, s))) != cudaSuccess) return cudaFail(hc, e, what);
      const bool hostSide = in.dev != in.host || out.dev != out.host;
      if (mustSync(hc, false, hostSide) && (e = cudaStreamSynchronize(s)) != cudaSuccess) return cudaFail(hc, e, what);
      return DSPLIB_SUCCESS;
   }
   const size_t inBytes = (size_t) n * eltIn, outBytes = (size_t) n * eltOut;
   if (in.staged && !(in.dev = stagingBuffer(0, inBytes, s))) return cudaFail(hc, cudaErrorMemoryAllocation, "staging");
   if (out.staged && !(out.dev = stagingBuffer(2, outBytes, s)))
      return cudaFail(hc, cudaErrorMemoryAllocation, "staging");
   const size_t staged = (in.staged ? inBytes : 0) + (out.staged ? outBytes : 0);
   PipeContext *pc = staged >= kConvPipeMinBytes ? pipeContext() : nullptr;
   if (!pc) {
      if (in.staged &&
          (e = injectCheck(cudaMemcpyAsync(in.dev, in.host, inBytes, cudaMemcpyHostToDevice, s))) != cudaSuccess)
         return cudaFail(hc, e, "copy input");
      if ((e = injectCheck(launch(in.dev, out.dev, n, s))) != cudaSuccess) return cudaFail(hc, e, what);
      if (out.staged &&
          (e = injectCheck(cudaMemcpyAsync(out.host, out.dev, outBytes, cudaMemcpyDeviceToHost, s))) != cudaSuccess)
         return cudaFail(hc, e, "copy output");
   }
   else {
      // Blocks of whole 8-element groups, so every block start keeps 16-byte alignment.
      int nblk = (int) (staged / kConvPipeBlockBytes);
      nblk = nblk < 2 ? 2 : (nblk > kPipeMaxBlocks ? kPipeMaxBlocks : nblk);
      long long per = (n + nblk - 1) / nblk;
      per = (per + 7) / 8 * 8;
      if ((e = cudaEventRecord(pc->start, s)) != cudaSuccess || (e = cudaStreamWaitEvent(pc->in, pc->start, 0)) ||
          (e = cudaStreamWaitEvent(pc->comp, pc->start, 0)) || (e = cudaStreamWaitEvent(pc->out, pc->start, 0)))
         return cudaFail(hc, e, "pipeline set-up");
      for (int b = 0; (long long) b * per < n; b++) {
         const long long e0 = (long long) b * per, cnt = (n - e0) < per ? (n - e0) : per;
         char *di = (char *) in.dev + e0 * eltIn, *dout = (char *) out.dev + e0 * eltOut;
         if (in.staged && (e = injectCheck(cudaMemcpyAsync(di, (char *) in.host + e0 * eltIn, cnt * eltIn,
                                                           cudaMemcpyHostToDevice, pc->in))))
            return pipeFail(hc, pc, e, "copy input block");
         if ((e = cudaEventRecord(pc->copied[b], pc->in)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(pc->comp, pc->copied[b], 0)) != cudaSuccess)
            return pipeFail(hc, pc, e, "pipeline");
         if ((e = injectCheck(launch(di, dout, cnt, pc->comp))) != cudaSuccess) return pipeFail(hc, pc, e, what);
         if ((e = cudaEventRecord(pc->computed[b], pc->comp)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(pc->out, pc->computed[b], 0)) != cudaSuccess)
            return pipeFail(hc, pc, e, "pipeline");
         if (out.staged && (e = injectCheck(cudaMemcpyAsync((char *) out.host + e0 * eltOut, dout, cnt * eltOut,
                                                            cudaMemcpyDeviceToHost, pc->out))))
            return pipeFail(hc, pc, e, "copy output block");
      }
      if ((e = cudaEventRecord(pc->done, pc->out)) != cudaSuccess || (e = cudaStreamWaitEvent(s, pc->done, 0)))
         return pipeFail(hc, pc, e, "pipeline join");
   }
   if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cudaFail(hc, e, what);
   return DSPLIB_SUCCESS;
}

} // namespace

extern "C" {

// ------------------------------------------------------------------ fltoq15

int32_t DSPLIB_fltoq15_getHandleSize(DSPLIB_fltoq15_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(Q15Priv); // DSPLIB_fltoq15.cpp:7-14
}

DSPLIB_STATUS DSPLIB_fltoq15_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams1D_t *bufParamsIn,
                                              const DSPLIB_bufParams1D_t *bufParamsOut,
                                              const DSPLIB_fltoq15_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER; // DSPLIB_fltoq15.cpp:24-26
   if (bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (!isFloatType(bufParamsIn->data_type)) return DSPLIB_ERR_INVALID_TYPE;  // :29-31
   if (bufParamsOut->data_type != DSPLIB_INT16) return DSPLIB_ERR_INVALID_TYPE; // :32-34
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_fltoq15_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut)
{
   (void) handle;
   return (pIn == NULL || pOut == NULL) ? DSPLIB_ERR_NULL_POINTER : DSPLIB_SUCCESS; // DSPLIB_fltoq15.cpp:52-57
}

DSPLIB_STATUS DSPLIB_fltoq15_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams1D_t *bufParamsIn,
                                  DSPLIB_bufParams1D_t *bufParamsOut, const DSPLIB_fltoq15_InitArgs *pKerInitArgs)
{
   (void) bufParamsOut;
   if (handle == NULL || bufParamsIn == NULL || pKerInitArgs == NULL) return DSPLIB_ERR_NULL_POINTER;
   Q15Priv *p = (Q15Priv *) handle;
   q15Reset(p, kMagicFltoq15);
   p->dataSize = pKerInitArgs->dataSize; // DSPLIB_fltoq15.cpp:71
   // DSPLIB_fltoq15.cpp:76-104: FLOAT32 / FLOAT64 input in either style, anything else
   // INVALID_TYPE; every style other than NATC runs the optimized variant.
   if (!isFloatType(bufParamsIn->data_type)) return DSPLIB_ERR_INVALID_TYPE;
   p->funcStyle = pKerInitArgs->funcStyle == DSPLIB_FUNCTION_NATC ? DSPLIB_FUNCTION_NATC : DSPLIB_FUNCTION_OPTIMIZED;
   p->isDouble = bufParamsIn->data_type == DSPLIB_FLOAT64;
   p->initialized = 1;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_fltoq15_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut)
{
   Q15Priv *p = q15Handle(handle, kMagicFltoq15);
   if (!p) return DSPLIB_ERR_FAILURE;
   if (pIn == NULL || pOut == NULL) {
      setError(&p->common, "exec: null buffer");
      return DSPLIB_ERR_NULL_POINTER;
   }
   if (p->dataSize == 0) return DSPLIB_SUCCESS;
   const bool dbl = p->isDouble != 0, natc = p->funcStyle == DSPLIB_FUNCTION_NATC;
   return convertExec(&p->common, pIn, dbl ? 8 : 4, pOut, 2, (long long) p->dataSize, "fltoq15 kernel",
                      [dbl, natc](void *in, void *out, long long n, cudaStream_t s) {
                         return launchFltoq15(in, (int16_t *) out, n, dbl, natc, s);
                      });
}

// ------------------------------------------------------------------ q15tofl

int32_t DSPLIB_q15tofl_getHandleSize(DSPLIB_q15tofl_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(Q15Priv); // DSPLIB_q15tofl.cpp:7-14
}

DSPLIB_STATUS DSPLIB_q15tofl_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams1D_t *bufParamsIn,
                                              const DSPLIB_bufParams1D_t *bufParamsOut,
                                              const DSPLIB_q15tofl_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER; // DSPLIB_q15tofl.cpp:24-26
   if (bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (bufParamsIn->data_type != DSPLIB_INT16) return DSPLIB_ERR_INVALID_TYPE; // :29-31
   if (!isFloatType(bufParamsOut->data_type)) return DSPLIB_ERR_INVALID_TYPE; // :32-34
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_q15tofl_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut)
{
   (void) handle;
   return (pIn == NULL || pOut == NULL) ? DSPLIB_ERR_NULL_POINTER : DSPLIB_SUCCESS; // DSPLIB_q15tofl.cpp:52-57
}

DSPLIB_STATUS DSPLIB_q15tofl_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams1D_t *bufParamsIn,
                                  DSPLIB_bufParams1D_t *bufParamsOut, const DSPLIB_q15tofl_InitArgs *pKerInitArgs)
{
   (void) bufParamsIn;
   if (handle == NULL || bufParamsOut == NULL || pKerInitArgs == NULL) return DSPLIB_ERR_NULL_POINTER;
   Q15Priv *p = (Q15Priv *) handle;
   q15Reset(p, kMagicQ15tofl);
   p->dataSize = pKerInitArgs->dataSize; // DSPLIB_q15tofl.cpp:71
   // DSPLIB_q15tofl.cpp:76-104: the output type selects the variant; anything but
   // FLOAT32 / FLOAT64 is INVALID_TYPE (the input type is checked by checkParams only).
   if (!isFloatType(bufParamsOut->data_type)) return DSPLIB_ERR_INVALID_TYPE;
   p->funcStyle = pKerInitArgs->funcStyle == DSPLIB_FUNCTION_NATC ? DSPLIB_FUNCTION_NATC : DSPLIB_FUNCTION_OPTIMIZED;
   p->isDouble = bufParamsOut->data_type == DSPLIB_FLOAT64;
   p->initialized = 1;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_q15tofl_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut)
{
   Q15Priv *p = q15Handle(handle, kMagicQ15tofl);
   if (!p) return DSPLIB_ERR_FAILURE;
   if (pIn == NULL || pOut == NULL) {
      setError(&p->common, "exec: null buffer");
      return DSPLIB_ERR_NULL_POINTER;
   }
   if (p->dataSize == 0) return DSPLIB_SUCCESS;
   const bool dbl = p->isDouble != 0;
   return convertExec(&p->common, pIn, 2, pOut, dbl ? 8 : 4, (long long) p->dataSize, "q15tofl kernel",
                      [dbl](void *in, void *out, long long n, cudaStream_t s) {
                         return launchQ15tofl((const int16_t *) in, out, n, dbl, s);
                      });
}

} // extern "C"
