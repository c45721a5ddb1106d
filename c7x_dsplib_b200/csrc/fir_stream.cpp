// Streaming (overlap-save) FIR over consecutive blocks.
//
// DSPLIB_fir is a "valid" filter: a call on N input samples per channel gives
// N - T + 1 outputs, and a caller that filters a continuous signal block by
// block has to carry the last T - 1 input samples of every channel into the
// next call itself (the reference leaves that to the caller).  A stream keeps
// that history on the device: each call takes N new samples per channel and
// returns N outputs per channel, the first T - 1 of them computed over the
// previous block's tail (zeros before the first block).
//
// Per call, on the handle's stream: the history and the new block are copied
// into one device window per channel, [T - 1 history | N new], DSPLIB_fir_exec
// runs over the windows, and the window's last T - 1 samples become the history.
#include <cstdlib>
#include <cstring>

#include "dsplib_internal.h"

namespace dsplib {

struct FirStream {
   FirPriv *handle = nullptr; // internal DSPLIB_fir handle over the windows
   void *win = nullptr;       // channels x (T - 1 + N) elements
   void *hist = nullptr;      // channels x (T - 1) elements
   int channels = 0, T = 0, N = 0, elt = 0;
   size_t inPitch = 0;        // bytes between the caller's input rows
};

static void destroyStream(FirStream *s)
{
   if (!s) return;
   cudaFree(s->win);
   cudaFree(s->hist);
   std::free(s->handle);
   delete s;
}

} // namespace dsplib

using namespace dsplib;

extern "C" {

DSPLIB_STATUS DSPLIB_gpu_firStreamCreate(DSPLIB_gpu_firStream *stream, const DSPLIB_fir_InitArgs *args,
                                         const DSPLIB_bufParams2D_t *bufParamsIn,
                                         const DSPLIB_bufParams2D_t *bufParamsFilter,
                                         const DSPLIB_bufParams2D_t *bufParamsOut)
{
   if (!stream || !args || !bufParamsIn || !bufParamsFilter || !bufParamsOut) return DSPLIB_ERR_NULL_POINTER;
   *stream = nullptr;
   const int elt = DSPLIB_sizeof((uint32_t) bufParamsIn->data_type);
   const int T = args->filterSize, N = args->dataSize, C = args->batchSize;
   if (elt <= 0) return DSPLIB_ERR_INVALID_TYPE;
   if (T < 1 || N < 1 || C < 1 || (int) bufParamsOut->dim_x != N || bufParamsIn->stride_y < N * elt)
      return DSPLIB_ERR_INVALID_DIMENSION;
   FirStream *s = new FirStream();
   s->channels = C;
   s->T = T;
   s->N = N;
   s->elt = elt;
   s->inPitch = (size_t) bufParamsIn->stride_y;
   const int W = T - 1 + N;
   DSPLIB_fir_InitArgs a = *args;
   a.dataSize = W;
   DSPLIB_bufParams2D_t win = *bufParamsIn;
   win.dim_x = (uint32_t) W;
   win.dim_y = (uint32_t) C;
   win.stride_y = W * elt;
   DSPLIB_bufParams2D_t filt = *bufParamsFilter, out = *bufParamsOut;
   s->handle = (FirPriv *) std::calloc(1, (size_t) DSPLIB_fir_getHandleSize(&a));
   DSPLIB_STATUS st = s->handle ? DSPLIB_fir_init(s->handle, &win, &filt, &out, &a) : DSPLIB_ERR_FAILURE;
   if (st == DSPLIB_SUCCESS &&
       (cudaMalloc(&s->win, (size_t) C * W * elt) != cudaSuccess ||
        (T > 1 && cudaMalloc(&s->hist, (size_t) C * (T - 1) * elt) != cudaSuccess) ||
        (T > 1 && cudaMemset(s->hist, 0, (size_t) C * (T - 1) * elt) != cudaSuccess)))
      st = DSPLIB_ERR_FAILURE;
   if (st != DSPLIB_SUCCESS) {
      (void) cudaGetLastError();
      destroyStream(s);
      return st;
   }
   *stream = (DSPLIB_gpu_firStream) s;
   return DSPLIB_SUCCESS;
}

DSPLIB_kernelHandle DSPLIB_gpu_firStreamHandle(DSPLIB_gpu_firStream stream)
{
   return stream ? (DSPLIB_kernelHandle) ((FirStream *) stream)->handle : nullptr;
}

DSPLIB_STATUS DSPLIB_gpu_firStreamExec(DSPLIB_gpu_firStream stream, const void *pIn, void *pFilter, void *pOut)
{
   FirStream *s = (FirStream *) stream;
   if (!s || !pIn || !pFilter || !pOut) return DSPLIB_ERR_NULL_POINTER;
   HandleCommon *hc = &s->handle->common;
   const cudaStream_t cs = hc->stream;
   const size_t hb = (size_t) (s->T - 1) * s->elt, nb = (size_t) s->N * s->elt, wb = hb + nb;
   char *win = (char *) s->win;
   cudaError_t e = cudaSuccess;
   if (hb && (e = cudaMemcpy2DAsync(win, wb, s->hist, hb, hb, s->channels, cudaMemcpyDeviceToDevice, cs)))
      return cudaFail(hc, e, "stream: restore history");
   if ((e = cudaMemcpy2DAsync(win + hb, wb, pIn, s->inPitch, nb, s->channels, cudaMemcpyDefault, cs)))
      return cudaFail(hc, e, "stream: copy block");
   const DSPLIB_STATUS st = DSPLIB_fir_exec(s->handle, win, pFilter, pOut);
   if (st != DSPLIB_SUCCESS) return st;
   if (hb && (e = cudaMemcpy2DAsync(s->hist, hb, win + nb, wb, hb, s->channels, cudaMemcpyDeviceToDevice, cs)))
      return cudaFail(hc, e, "stream: save history");
   // a host block is copied in asynchronously: complete before returning unless async level 2
   if (mustSync(hc, false, !isDevicePtr(pIn)) && (e = cudaStreamSynchronize(cs)))
      return cudaFail(hc, e, "stream: execution");
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_firStreamReset(DSPLIB_gpu_firStream stream)
{
   FirStream *s = (FirStream *) stream;
   if (!s) return DSPLIB_ERR_NULL_POINTER;
   if (s->T > 1 && cudaMemsetAsync(s->hist, 0, (size_t) s->channels * (s->T - 1) * s->elt,
                                   s->handle->common.stream) != cudaSuccess)
      return cudaFail(&s->handle->common, cudaGetLastError(), "stream: reset");
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_firStreamDestroy(DSPLIB_gpu_firStream stream)
{
   FirStream *s = (FirStream *) stream;
   if (!s) return DSPLIB_ERR_NULL_POINTER;
   (void) cudaStreamSynchronize(s->handle->common.stream);
   destroyStream(s);
   return DSPLIB_SUCCESS;
}

} // extern "C"
