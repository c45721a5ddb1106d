// C-ABI entry points of DSPLIB_interleave, DSPLIB_deinterleave and DSPLIB_addNCh
// (reference src/DSPLIB_interleave/DSPLIB_interleave.cpp, src/DSPLIB_deinterleave/
// DSPLIB_deinterleave.cpp, src/DSPLIB_addNCh/DSPLIB_addNCh.cpp): the reference's
// parameter checks in their order, the work on the GPU.  Device buffers are used in
// place; host buffers are staged (row by row on the output side, so the bytes
// between the caller's output rows stay untouched).
#include <cstring>

#include "dsplib_internal.h"

using namespace dsplib;

namespace {

bool layoutType(uint32_t t)
{
   switch (t) {
   case DSPLIB_INT8:
   case DSPLIB_UINT8:
   case DSPLIB_INT16:
   case DSPLIB_UINT16:
   case DSPLIB_INT32:
   case DSPLIB_UINT32:
   case DSPLIB_FLOAT32:
   case DSPLIB_INT64:
   case DSPLIB_UINT64:
   case DSPLIB_FLOAT64: return true;
   default: return false;
   }
}

bool is16(uint32_t t) { return t == DSPLIB_INT16 || t == DSPLIB_UINT16; }
bool is8(uint32_t t) { return t == DSPLIB_INT8 || t == DSPLIB_UINT8; }

template <typename P> P *handleOf(DSPLIB_kernelHandle h, uint32_t magic)
{
   P *p = (P *) h;
   if (!p || p->common.magic != magic || !p->initialized) return nullptr;
   return p;
}

template <typename P> void resetHandle(P *p, uint32_t magic)
{
   if (p->common.magic != magic) {
      std::memset(&p->common, 0, sizeof(p->common));
      p->common.magic = magic;
   }
   p->common.err[0] = 0;
   p->initialized = 0;
}

// Shared by interleave and deinterleave: both run the matrix transpose
// (DSPLIB_interleave.cpp:89-253, DSPLIB_deinterleave.cpp:89-251 record the same fields).
DSPLIB_STATUS layoutInit(DSPLIB_kernelHandle handle, const DSPLIB_bufParams2D_t *in, const DSPLIB_bufParams2D_t *out,
                         uint32_t magic)
{
   if (handle == NULL || in == NULL || out == NULL) return DSPLIB_ERR_NULL_POINTER;
   LayoutPriv *p = (LayoutPriv *) handle;
   resetHandle(p, magic);
   p->widthIn = in->dim_x;
   p->heightIn = in->dim_y;
   p->strideIn = in->stride_y;
   p->strideOut = out->stride_y;
   p->dataType = (int32_t) in->data_type;
   if (!layoutType(in->data_type)) return DSPLIB_ERR_INVALID_TYPE;
   p->initialized = 1;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS layoutExec(DSPLIB_kernelHandle handle, void *pIn, void *pOut, uint32_t magic)
{
   LayoutPriv *p = handleOf<LayoutPriv>(handle, magic);
   if (!p) return DSPLIB_ERR_FAILURE;
   HandleCommon *hc = &p->common;
   if (pIn == NULL || pOut == NULL) {
      setError(hc, "exec: null buffer");
      return DSPLIB_ERR_NULL_POINTER;
   }
   const int elt = DSPLIB_sizeof((uint32_t) p->dataType);
   const long long W = p->widthIn, H = p->heightIn;
   if (W == 0 || H == 0) return DSPLIB_SUCCESS;
   if (p->strideIn < elt || p->strideOut < elt) {
      setError(hc, "exec: row strides smaller than one element");
      return DSPLIB_ERR_INVALID_DIMENSION;
   }
   const long long sInE = p->strideIn / elt; // DSPLIB_matTrans_cn.cpp:43: (strideIn / dataSize) * j
   cudaStream_t s = hc->stream;
   // input: H rows of W elements, strideIn bytes apart; output: W rows of H elements at
   // (i * strideOut) / elt
   Region rin{pIn, nullptr, (size_t) W * elt, (size_t) H, (size_t) sInE * elt, false, false};
   Region rout{pOut, nullptr, (size_t) H * elt, (size_t) W, (size_t) p->strideOut, false, false};
   if (p->strideOut % elt) { // rows not element aligned: stage the whole span
      rout.width = (size_t) (((W - 1) * p->strideOut) / elt + H) * elt;
      rout.height = 1;
      rout.pitch = rout.width;
   }
   cudaError_t e;
   if ((e = regionIn(rin, 0, true, s)) != cudaSuccess) return cudaFail(hc, e, "stage input");
   if ((e = regionIn(rout, 2, rout.height == 1 && p->strideOut % elt, s)) != cudaSuccess)
      return cudaFail(hc, e, "stage output");
   TransposeLaunch a{rin.dev, rout.dev, W, H, sInE, (long long) p->strideOut, elt};
   if ((e = launchTranspose(a, s)) != cudaSuccess) return cudaFail(hc, e, "transpose kernel");
   if ((e = regionOut(rout, s)) != cudaSuccess) return cudaFail(hc, e, "copy output");
   if (mustSync(hc, rin.staged || rout.staged, rin.onHost || rout.onHost) && (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cudaFail(hc, e, "transpose execution");
   return DSPLIB_SUCCESS;
}

void layoutPerf(LayoutPriv *p, uint64_t *archCycles, uint64_t *estCycles)
{
   const double bytes = 2.0 * p->widthIn * p->heightIn * DSPLIB_sizeof((uint32_t) p->dataType);
   const double ns = bytes / 6.5e12 * 1e9;
   if (archCycles) *archCycles = (uint64_t) ns;
   if (estCycles) *estCycles = (uint64_t) ns + 4000; // + launch and synchronisation
}

} // namespace

extern "C" {

// ------------------------------------------------------------------ interleave

int32_t DSPLIB_interleave_getHandleSize(DSPLIB_interleaveInitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(LayoutPriv);
}

DSPLIB_STATUS DSPLIB_interleave_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams2D_t *bufParamsIn,
                                                 const DSPLIB_bufParams2D_t *bufParamsOut,
                                                 const DSPLIB_interleaveInitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER; // DSPLIB_interleave.cpp:25-27
   if (bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   DSPLIB_STATUS status = DSPLIB_SUCCESS;
   const uint32_t strideElements = (uint32_t) (bufParamsOut->stride_y / DSPLIB_sizeof(bufParamsOut->data_type));
   if (!layoutType(bufParamsIn->data_type)) status = DSPLIB_ERR_INVALID_TYPE; // :32-41
   // :42-64 -- the second test's verdict replaces the first one's outside the 1/2-row packed case
   if ((bufParamsIn->dim_y == 1u || bufParamsIn->dim_y == 2u) && strideElements == bufParamsOut->dim_x) {
   }
   else if (bufParamsIn->data_type != bufParamsOut->data_type) status = DSPLIB_ERR_INVALID_TYPE;
   else if (is16(bufParamsIn->data_type) && bufParamsIn->dim_x % 2 != 0) status = DSPLIB_ERR_INVALID_VALUE;
   else if (is8(bufParamsIn->data_type) && bufParamsIn->dim_x % 4 != 0) status = DSPLIB_ERR_INVALID_VALUE;
   else status = DSPLIB_SUCCESS;
   return status;
}

DSPLIB_STATUS DSPLIB_interleave_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut)
{
   (void) handle;
   return (pIn == NULL || pOut == NULL) ? DSPLIB_ERR_NULL_POINTER : DSPLIB_SUCCESS; // DSPLIB_interleave.cpp:76-81
}

DSPLIB_STATUS DSPLIB_interleave_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams2D_t *bufParamsIn,
                                     DSPLIB_bufParams2D_t *bufParamsOut, const DSPLIB_interleaveInitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return layoutInit(handle, bufParamsIn, bufParamsOut, kMagicInterleave);
}

DSPLIB_STATUS DSPLIB_interleave_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut)
{
   return layoutExec(handle, pIn, pOut, kMagicInterleave);
}

void DSPLIB_interleave_perfEst(DSPLIB_kernelHandle handle, uint64_t *archCycles, uint64_t *estCycles)
{
   if (LayoutPriv *p = handleOf<LayoutPriv>(handle, kMagicInterleave)) layoutPerf(p, archCycles, estCycles);
}

// ------------------------------------------------------------------ deinterleave

int32_t DSPLIB_deinterleave_getHandleSize(DSPLIB_deinterleaveInitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(LayoutPriv);
}

DSPLIB_STATUS DSPLIB_deinterleave_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams2D_t *bufParamsIn,
                                                   const DSPLIB_bufParams2D_t *bufParamsOut,
                                                   const DSPLIB_deinterleaveInitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER; // DSPLIB_deinterleave.cpp:25-27
   if (bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   // :30-33: one channel, or two channels packed in the row, always pass
   if (bufParamsIn->dim_x == 1u ||
       (bufParamsIn->dim_x == 2u &&
        (uint32_t) bufParamsIn->dim_x == (uint32_t) bufParamsIn->stride_y / DSPLIB_sizeof(bufParamsIn->data_type)))
      return DSPLIB_SUCCESS;
   if (!layoutType(bufParamsIn->data_type)) return DSPLIB_ERR_INVALID_TYPE; // :35-40
   if (bufParamsIn->data_type != bufParamsOut->data_type) return DSPLIB_ERR_INVALID_TYPE; // :43-45
   if (is16(bufParamsIn->data_type) && bufParamsIn->dim_x % 2 != 0) return DSPLIB_ERR_INVALID_VALUE;
   if (is8(bufParamsIn->data_type) && bufParamsIn->dim_x % 4 != 0) return DSPLIB_ERR_INVALID_VALUE;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_deinterleave_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut)
{
   (void) handle;
   return (pIn == NULL || pOut == NULL) ? DSPLIB_ERR_NULL_POINTER : DSPLIB_SUCCESS; // DSPLIB_deinterleave.cpp:76-81
}

DSPLIB_STATUS DSPLIB_deinterleave_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams2D_t *bufParamsIn,
                                       DSPLIB_bufParams2D_t *bufParamsOut,
                                       const DSPLIB_deinterleaveInitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return layoutInit(handle, bufParamsIn, bufParamsOut, kMagicDeinterleave);
}

DSPLIB_STATUS DSPLIB_deinterleave_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut)
{
   return layoutExec(handle, pIn, pOut, kMagicDeinterleave);
}

void DSPLIB_deinterleave_perfEst(DSPLIB_kernelHandle handle, uint64_t *archCycles, uint64_t *estCycles,
                                 uint64_t dataType)
{
   (void) dataType;
   if (LayoutPriv *p = handleOf<LayoutPriv>(handle, kMagicDeinterleave)) layoutPerf(p, archCycles, estCycles);
}

// ------------------------------------------------------------------ addNCh

int32_t DSPLIB_addNCh_getHandleSize(DSPLIB_addNCh_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(AddNChPriv);
}

DSPLIB_STATUS DSPLIB_addNCh_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams3D_t *bufParamsIn,
                                             const DSPLIB_bufParams2D_t *bufParamsOut,
                                             const DSPLIB_addNCh_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER; // DSPLIB_addNCh.cpp:20-22
   if (bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (bufParamsIn->data_type != DSPLIB_FLOAT32 && bufParamsIn->data_type != DSPLIB_FLOAT64)
      return DSPLIB_ERR_INVALID_TYPE; // :25-27
   if (bufParamsIn->data_type != bufParamsOut->data_type) return DSPLIB_ERR_INVALID_TYPE; // :28-30
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_addNCh_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut)
{
   (void) handle;
   return (pIn == NULL || pOut == NULL) ? DSPLIB_ERR_NULL_POINTER : DSPLIB_SUCCESS; // DSPLIB_addNCh.cpp:48-53
}

DSPLIB_STATUS DSPLIB_addNCh_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams3D_t *bufParamsIn,
                                 DSPLIB_bufParams2D_t *bufParamsOut, const DSPLIB_addNCh_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   if (handle == NULL || bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   AddNChPriv *p = (AddNChPriv *) handle;
   resetHandle(p, kMagicAddNCh);
   // DSPLIB_addNCh.cpp:67-72
   const int32_t elt = DSPLIB_sizeof(bufParamsIn->data_type);
   p->samples = bufParamsIn->dim_x;
   p->channels = bufParamsIn->dim_y;
   p->inputs = bufParamsIn->dim_z;
   p->strideInElementsY = bufParamsIn->stride_y / elt;
   p->strideInElementsZ = bufParamsIn->stride_z / elt;
   p->strideOutElements = bufParamsOut->stride_y / elt;
   p->dataType = (int32_t) bufParamsIn->data_type;
   // :77-131: FLOAT32 / FLOAT64 in either style
   if (bufParamsIn->data_type != DSPLIB_FLOAT32 && bufParamsIn->data_type != DSPLIB_FLOAT64)
      return DSPLIB_ERR_INVALID_TYPE;
   p->initialized = 1;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_addNCh_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut)
{
   AddNChPriv *p = handleOf<AddNChPriv>(handle, kMagicAddNCh);
   if (!p) return DSPLIB_ERR_FAILURE;
   HandleCommon *hc = &p->common;
   if (pIn == NULL || pOut == NULL) {
      setError(hc, "exec: null buffer");
      return DSPLIB_ERR_NULL_POINTER;
   }
   const long long S = p->samples, C = p->channels, L = p->inputs;
   if (S == 0 || C == 0) return DSPLIB_SUCCESS;
   const long long sY = p->strideInElementsY, sZ = p->strideInElementsZ, sO = p->strideOutElements;
   if ((C > 1 && sY < S) || (L > 1 && sZ < 1) || (C > 1 && sO < S)) {
      setError(hc, "exec: inconsistent strides (sY=%lld sZ=%lld sO=%lld)", sY, sZ, sO);
      return DSPLIB_ERR_INVALID_DIMENSION;
   }
   const size_t elt = p->dataType == DSPLIB_FLOAT64 ? 8 : 4;
   cudaStream_t s = hc->stream;
   // input: the span the kernel reads; output: C rows of S elements, sO apart
   const long long span = (L > 0 ? (L - 1) * sZ : 0) + (C - 1) * sY + S;
   Region rin{pIn, nullptr, (size_t) span * elt, 1, (size_t) span * elt, false, false};
   Region rout{pOut, nullptr, (size_t) S * elt, (size_t) C, (size_t) (C > 1 ? sO : S) * elt, false, false};
   cudaError_t e;
   if (L > 0 && (e = regionIn(rin, 0, true, s)) != cudaSuccess) return cudaFail(hc, e, "stage input");
   if ((e = regionIn(rout, 2, false, s)) != cudaSuccess) return cudaFail(hc, e, "stage output");
   AddNChLaunch a{rin.dev, rout.dev, S, C, (int) L, sY, sZ, C > 1 ? sO : S, p->dataType == DSPLIB_FLOAT64};
   if ((e = launchAddNCh(a, s)) != cudaSuccess) return cudaFail(hc, e, "addNCh kernel");
   if ((e = regionOut(rout, s)) != cudaSuccess) return cudaFail(hc, e, "copy output");
   if (mustSync(hc, rin.staged || rout.staged, rin.onHost || rout.onHost) && (e = cudaStreamSynchronize(s)) != cudaSuccess)
      return cudaFail(hc, e, "addNCh execution");
   return DSPLIB_SUCCESS;
}

void DSPLIB_addNCh_perfEst(DSPLIB_kernelHandle handle, uint64_t *archCycles, uint64_t *estCycles, uint32_t dataType)
{
   (void) dataType;
   AddNChPriv *p = handleOf<AddNChPriv>(handle, kMagicAddNCh);
   if (!p) return;
   const double elt = p->dataType == DSPLIB_FLOAT64 ? 8.0 : 4.0;
   const double bytes = elt * p->samples * p->channels * (p->inputs + 1.0);
   const double ns = bytes / 6.5e12 * 1e9;
   if (archCycles) *archCycles = (uint64_t) ns;
   if (estCycles) *estCycles = (uint64_t) ns + 4000;
}

} // extern "C"
