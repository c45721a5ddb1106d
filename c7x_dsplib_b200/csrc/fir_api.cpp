// DSPLIB_fir C-ABI entry points (drop-in for src/DSPLIB_fir/DSPLIB_fir.cpp and
// the getSizes part of DSPLIB_fir_ci.cpp).  Parameter handling mirrors the
// reference line by line where callers can observe it (status codes, computed
// sizes and pitches); exec launches CUDA kernels instead of C7x code.
#include <cstring>
#include <string>
#include <vector>

#include "dsplib_internal.h"

using namespace dsplib;

namespace {

bool firTypeKnown(uint32_t t)
{
   return t == DSPLIB_INT16 || t == DSPLIB_INT32 || t == DSPLIB_INT8 || t == DSPLIB_FLOAT32;
}

// DSPLIB_fir_ci.cpp:63-103.  Computed in uint32 like the reference, so an
// oversize filter wraps the output length the same way.
void firSizes(const DSPLIB_fir_InitArgs *a, int32_t elt, DSPLIB_bufParams2D_t *filt, DSPLIB_bufParams2D_t *out)
{
   uint32_t dataSize = (uint32_t) a->dataSize;
   uint32_t filterSize = (uint32_t) a->filterSize;
   uint32_t mma = (uint32_t) a->MMA_SIZE;
   out->dim_x = dataSize - filterSize + 1;
   filt->dim_y = (a->enableNchCoefs == 0) ? 1 : (uint32_t) a->batchSize;
   if (a->enableMMA) {
      filt->dim_x = 2 * mma + filterSize + mma - 1;
      filt->stride_y = (int32_t) (filt->dim_x * (uint32_t) elt);
   }
}

FirPriv *firHandle(DSPLIB_kernelHandle h)
{
   FirPriv *p = (FirPriv *) h;
   if (!p || p->common.magic != kMagicFir || !p->initialized) return nullptr;
   return p;
}

// The kernel an exec of this handle runs for launch a (a's taps and sizes filled).
FirKernelKind firKindOf(const FirPriv *p, const FirLaunch &a)
{
   const DSPLIB_fir_InitArgs &ia = p->initArgs;
   const HandleCommon *hc = &p->common;
   const bool natc = ia.funcStyle == DSPLIB_FUNCTION_NATC;
   const bool floatQ = !natc && p->dtype == DSPLIB_FLOAT32 && ia.enableQ != 0;
   FirKernelKind kind;
   if (natc) kind = FIR_NATC;
   else if (floatQ) kind = FIR_F32_Q;
   else if (p->dtype == DSPLIB_FLOAT32)
      kind = hc->firPrecision == DSPLIB_GPU_FIR_BF16X3 ? FIR_F32_BF16X3 : FIR_F32_SIMT;
   else kind = hc->firQMode ? FIR_QMODE : FIR_NATC;
   // Optimized 8/16-bit integers run on the tensor cores when the taps fit the band buffer.
   if (!natc && (p->dtype == DSPLIB_INT8 || p->dtype == DSPLIB_INT16) && firIntTcSupported(a))
      kind = hc->firQMode ? FIR_INT_Q_TC : FIR_INT_WRAP_TC;
   // Split-BF16x3 covers up to 512 taps; longer filters run the FP32 CUDA-core kernel.
   if (kind == FIR_F32_BF16X3 && !firBf16x3Supported(a)) kind = FIR_F32_SIMT;
   return kind;
}

// A launch of this handle's problem on compact buffers (no pointers): what the autotuner
// keys and measures.
FirLaunch firShape(const FirPriv *p)
{
   const DSPLIB_fir_InitArgs &ia = p->initArgs;
   FirLaunch a{};
   a.dtype = p->dtype;
   a.batch = ia.batchSize;
   a.T = ia.filterSize;
   a.outSize = p->outputSize;
   a.inPitch = (long long) p->outputSize + (ia.filterSize > 0 ? ia.filterSize : 1) - 1;
   a.outPitch = p->outputSize;
   a.filtPitch = ia.enableNchCoefs ? ia.filterSize : 0;
   const bool floatQ = ia.funcStyle != DSPLIB_FUNCTION_NATC && p->dtype == DSPLIB_FLOAT32 && ia.enableQ != 0;
   a.shift = floatQ ? (int) ia.Q : (int) ia.shift;
   return a;
}

// Whether the handle's stream is being captured into a graph (no measurement then).
bool capturing(cudaStream_t s)
{
   cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
   if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
      (void) cudaGetLastError();
      return true;
   }
   return cs != cudaStreamCaptureStatusNone;
}

// The handle's cached autotuner choice for kind, resolved again when the table changed.
// In MEASURE mode a class still without an entry (settings changed after init: precision,
// Q mode) is measured here, on scratch buffers, before the call's own launch.
int firChoice(FirPriv *p, const FirLaunch &a, FirKernelKind kind);
DSPLIB_STATUS firMeasureFor(FirPriv *p);

int firChoice(FirPriv *p, const FirLaunch &a, FirKernelKind kind)
{
   const unsigned gen = tuneGeneration();
   if (p->tuneGen != gen || p->tuneKind != (int32_t) kind) {
      int c = -1;
      const std::string key = firTuneKey(a, kind);
      if (!key.empty() && !tuneLookup(key, &c) && tuneMode() == DSPLIB_GPU_TUNE_MEASURE &&
          !capturing(p->common.stream))
         (void) firMeasureFor(p);
      if (key.empty() || !tuneLookup(key, &c)) c = -1;
      p->tuneGen = gen;
      p->tuneKind = (int32_t) kind;
      p->tuneChoice = c;
   }
   return p->tuneChoice;
}

DSPLIB_STATUS firMeasureFor(FirPriv *p) { return firHandleTune((DSPLIB_kernelHandle) p); }

} // namespace

namespace dsplib {

std::string firHandleTuneKey(DSPLIB_kernelHandle h, std::vector<int> *cands)
{
   FirPriv *p = firHandle(h);
   if (!p || p->initArgs.batchSize <= 0 || p->outputSize <= 0) return std::string();
   const FirLaunch a = firShape(p);
   const FirKernelKind kind = firKindOf(p, a);
   if (cands) *cands = firTuneCandidates(a, kind);
   return firTuneKey(a, kind);
}

// Every candidate on scratch buffers of the handle's shape filled with a hashed
// pattern, on a private stream; the fastest is stored.
DSPLIB_STATUS firHandleTune(DSPLIB_kernelHandle h)
{
   FirPriv *p = firHandle(h);
   if (!p) return DSPLIB_ERR_NULL_POINTER;
   std::vector<int> cands;
   const std::string key = firHandleTuneKey(h, &cands);
   if (key.empty() || cands.empty()) return DSPLIB_ERR_NOT_IMPLEMENTED;
   FirLaunch a = firShape(p);
   const FirKernelKind kind = firKindOf(p, a);
   const size_t xb = (size_t) a.batch * a.inPitch * p->elt;
   const size_t hb = (size_t) (a.filtPitch ? a.batch : 1) * (a.T > 0 ? a.T : 1) * p->elt;
   const size_t yb = (size_t) a.batch * a.outPitch * p->elt;
   void *x = nullptr, *hh = nullptr, *y = nullptr;
   DSPLIB_STATUS st = DSPLIB_ERR_FAILURE;
   if (cudaMalloc(&x, xb) == cudaSuccess && cudaMalloc(&hh, hb) == cudaSuccess && cudaMalloc(&y, yb) == cudaSuccess &&
       tuneFill(x, xb, p->dtype == DSPLIB_FLOAT32) && tuneFill(hh, hb, p->dtype == DSPLIB_FLOAT32)) {
      a.x = x;
      a.h = hh;
      a.y = y;
      a.err = errorWord(&p->common);
      const int best = tunePick(key, cands, [&](int c, cudaStream_t s) {
         FirLaunch b = a;
         firApplyChoice(b, kind, c);
         return launchFir(b, kind, s);
      });
      (void) takeErrorWord(&p->common);
      if (best >= 0) st = DSPLIB_SUCCESS;
   }
   (void) cudaGetLastError();
   cudaFree(x);
   cudaFree(hh);
   cudaFree(y);
   p->tuneGen = 0;
   return st;
}

} // namespace dsplib

extern "C" {

int32_t DSPLIB_fir_getHandleSize(DSPLIB_fir_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(FirPriv);
}

DSPLIB_STATUS DSPLIB_fir_getSizes(const DSPLIB_fir_InitArgs *pKerInitArgs,
                                  DSPLIB_bufParams2D_t *bufParamsIn,
                                  DSPLIB_bufParams2D_t *bufParamsFilter,
                                  DSPLIB_bufParams2D_t *bufParamsOut)
{
   if (!firTypeKnown(bufParamsIn->data_type)) return DSPLIB_ERR_NOT_IMPLEMENTED; // DSPLIB_fir.cpp:93-95
   firSizes(pKerInitArgs, DSPLIB_sizeof(bufParamsIn->data_type), bufParamsFilter, bufParamsOut);
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_fir_init_checkParams(DSPLIB_kernelHandle handle,
                                          const DSPLIB_bufParams2D_t *bufParamsIn,
                                          const DSPLIB_bufParams2D_t *bufParamsFilter,
                                          const DSPLIB_bufParams2D_t *bufParamsOut,
                                          const DSPLIB_fir_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   // DSPLIB_fir.cpp:27-66
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (!firTypeKnown(bufParamsIn->data_type)) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->data_type != bufParamsOut->data_type) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->data_type != bufParamsFilter->data_type) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->data_type != DSPLIB_FLOAT32) return DSPLIB_ERR_INVALID_TYPE;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_fir_exec_checkParams(DSPLIB_kernelHandle handle,
                                          const void *pIn,
                                          const void *pFilter,
                                          const void *pOut)
{
   (void) handle;
   if (pIn == NULL || pFilter == NULL || pOut == NULL) return DSPLIB_ERR_NULL_POINTER; // DSPLIB_fir.cpp:110-115
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_fir_init(DSPLIB_kernelHandle handle,
                              DSPLIB_bufParams2D_t *bufParamsIn,
                              DSPLIB_bufParams2D_t *bufParamsFilter,
                              DSPLIB_bufParams2D_t *bufParamsOut,
                              DSPLIB_fir_InitArgs *pKerInitArgs)
{
   if (handle == NULL || pKerInitArgs == NULL || bufParamsIn == NULL) return DSPLIB_ERR_NULL_POINTER;
   FirPriv *p = (FirPriv *) handle;
   if (p->common.magic != kMagicFir) {
      std::memset(&p->common, 0, sizeof(p->common));
      p->common.magic = kMagicFir;
   }
   p->common.err[0] = 0;
   p->initArgs = *pKerInitArgs;
   p->initialized = 0;
   p->dtype = (int32_t) bufParamsIn->data_type;

   // DSPLIB_fir.cpp:134-157
   int32_t elt = 0;
   DSPLIB_STATUS status = DSPLIB_SUCCESS;
   switch (bufParamsIn->data_type) {
   case DSPLIB_FLOAT32:
   case DSPLIB_INT32:
   case DSPLIB_UINT32: elt = 4; break;
   case DSPLIB_INT16:
   case DSPLIB_UINT16: elt = 2; break;
   case DSPLIB_INT8:
   case DSPLIB_UINT8: elt = 1; break;
   default: status = DSPLIB_ERR_INVALID_TYPE; break;
   }
   p->elt = elt;
   if (elt != 0) {
      p->inPitch = bufParamsIn->stride_y / elt;
      p->outPitch = bufParamsOut->stride_y / elt;
      p->outputSize = (int32_t) bufParamsOut->dim_x;
      p->filterPitch = bufParamsFilter->stride_y / elt;
   }
   // DSPLIB_fir.cpp:159-196: both styles accept exactly INT8/INT16/INT32/FLOAT32.
   if (elt == 0 || !firTypeKnown(bufParamsIn->data_type)) return DSPLIB_ERR_INVALID_TYPE;
   if (pKerInitArgs->funcStyle != DSPLIB_FUNCTION_NATC && pKerInitArgs->funcStyle != DSPLIB_FUNCTION_OPTIMIZED) {
      // The reference treats every non-NATC style as OPTIMIZED (DSPLIB_fir.cpp:177).
      p->initArgs.funcStyle = DSPLIB_FUNCTION_OPTIMIZED;
   }
   p->initialized = 1;
   p->tuneGen = 0;
   if (status == DSPLIB_SUCCESS && tuneMode() == DSPLIB_GPU_TUNE_MEASURE) {
      int c = 0;
      const std::string key = firHandleTuneKey(handle, nullptr);
      if (!key.empty() && !tuneLookup(key, &c)) (void) firHandleTune(handle); // a failed measurement keeps the rule
   }
   return status;
}

DSPLIB_STATUS DSPLIB_fir_exec(DSPLIB_kernelHandle handle, void *pIn, void *pFilter, void *pOut)
{
   FirPriv *p = firHandle(handle);
   if (!p) return DSPLIB_ERR_FAILURE;
   HandleCommon *hc = &p->common;
   if (pIn == NULL || pFilter == NULL || pOut == NULL) {
      setError(hc, "exec: null buffer");
      return DSPLIB_ERR_NULL_POINTER;
   }
   const DSPLIB_fir_InitArgs &ia = p->initArgs;
   const int elt = p->elt;
   const int T = ia.filterSize;
   const int batch = ia.batchSize;
   const int outSize = p->outputSize;
   if (batch <= 0 || outSize <= 0) return DSPLIB_SUCCESS; // nothing to compute (reference loops run zero times)
   const bool natc = ia.funcStyle == DSPLIB_FUNCTION_NATC;
   const bool nch = ia.enableNchCoefs != 0;
   const long long M = ia.MMA_SIZE;

   // Tap rows.  NATC follows DSPLIB_fir_cn.cpp:50-52 (the caller passes the
   // first tap; MMA rows are 3*M + T - 1 apart).  OPTIMIZED follows the _ci
   // path: the caller passes the padded buffer, taps start 2*M elements in,
   // rows are stride_y apart (DSPLIB_fir_d.c:195-208, DSPLIB_fir_ci.cpp:283).
   long long tapOffset = 0, filtPitch = 0;
   if (natc) {
      filtPitch = nch ? (ia.enableMMA ? (3 * M + T - 1) : T) : 0;
   }
   else {
      tapOffset = ia.enableMMA ? 2 * M : 0;
      filtPitch = nch ? p->filterPitch : 0;
   }
   if (T < 0 || p->inPitch <= 0 || p->outPitch <= 0 || (nch && filtPitch < T) || tapOffset < 0) {
      setError(hc, "exec: inconsistent sizes (T=%d inPitch=%d outPitch=%d filterPitch=%lld)", T, p->inPitch,
               p->outPitch, filtPitch);
      return DSPLIB_ERR_INVALID_DIMENSION;
   }

   // Q mode rounds with 2^(shift-1) and shifts a 64-bit (int32 data: 128-bit) accumulator:
   // shifts beyond 62 have no defined result there.  The natural-C wrap mode ignores shift.
   const bool qmode = !natc && p->dtype != DSPLIB_FLOAT32 && hc->firQMode;
   if (qmode && ia.shift > kFirMaxQShift) {
      setError(hc, "exec: Q-mode shift %u out of range (at most %d)", ia.shift, kFirMaxQShift);
      return DSPLIB_ERR_INVALID_VALUE;
   }

   // Float Q mode: FLOAT32 filters quantised to int32 at scale 2^Q (InitArgs.enableQ / Q).
   const bool floatQ = !natc && p->dtype == DSPLIB_FLOAT32 && ia.enableQ != 0;
   if (floatQ && ia.Q > (uint32_t) kFirMaxFloatQ) {
      setError(hc, "exec: float Q mode needs Q <= %d (got %u)", kFirMaxFloatQ, ia.Q);
      return DSPLIB_ERR_INVALID_VALUE;
   }

   cudaStream_t s = hc->stream;
   Region rin{pIn, nullptr, (size_t) (outSize + (T > 0 ? T : 1) - 1) * elt, (size_t) batch,
              (size_t) p->inPitch * elt, false};
   Region rf{(char *) pFilter + tapOffset * elt, nullptr, (size_t) (T > 0 ? T : 1) * elt, (size_t) (nch ? batch : 1),
             (size_t) (nch ? filtPitch : (T > 0 ? T : 1)) * elt, false};
   Region rout{pOut, nullptr, (size_t) outSize * elt, (size_t) batch, (size_t) p->outPitch * elt, false};
   // Large host buffers: copy in, compute and copy out channel blocks in a pipeline.
   PipeContext *pc = nullptr;
   if (batch >= 2 && rin.bytes() + rout.bytes() >= kFirPipeMinBytes && !isDevicePtr(pIn) && !isDevicePtr(pOut))
      pc = pipeContext();
   cudaStream_t sIn = pc ? pc->in : s;
   cudaError_t e;
   injectArm(hc);
   struct Disarm {
      ~Disarm() { injectDisarm(); }
   } disarm;
   if (pc) {
      // after whatever the caller queued on the handle's stream
      if ((e = cudaEventRecord(pc->start, s)) != cudaSuccess || (e = cudaStreamWaitEvent(pc->in, pc->start, 0)) ||
          (e = cudaStreamWaitEvent(pc->comp, pc->start, 0)) || (e = cudaStreamWaitEvent(pc->out, pc->start, 0)))
         return cudaFail(hc, e, "pipeline set-up");
   }
   if ((e = injectCheck(regionIn(rin, 0, pc == nullptr, sIn))) != cudaSuccess) return pipeFail(hc, pc, e, "stage input");
   if ((e = injectCheck(regionIn(rf, 1, true, sIn))) != cudaSuccess) return pipeFail(hc, pc, e, "stage filter");
   if ((e = injectCheck(regionIn(rout, 2, false, sIn))) != cudaSuccess) return pipeFail(hc, pc, e, "stage output");

   FirLaunch a;
   a.x = rin.dev;
   a.h = rf.dev;
   a.y = rout.dev;
   a.dtype = p->dtype;
   a.batch = batch;
   a.T = T;
   a.outSize = outSize;
   a.inPitch = p->inPitch;
   a.outPitch = p->outPitch;
   a.filtPitch = nch ? filtPitch : 0; // staging keeps the caller's row pitch
   a.shift = floatQ ? (int) ia.Q : (int) ia.shift;
   a.err = errorWord(hc);
   const FirKernelKind kind = firKindOf(p, a);
   firApplyChoice(a, kind, firChoice(p, a, kind));
   if (!pc) {
      if ((e = injectCheck(launchFir(a, kind, s))) != cudaSuccess) return cudaFail(hc, e, "FIR kernel launch");
      if ((e = injectCheck(regionOut(rout, s))) != cudaSuccess) return cudaFail(hc, e, "copy output");
   }
   else {
      const size_t total = rin.bytes() + rout.bytes();
      int nblk = (int) (total / kFirPipeBlockBytes);
      nblk = nblk < 2 ? 2 : (nblk > kPipeMaxBlocks ? kPipeMaxBlocks : nblk);
      const int rowsPer = (batch + nblk - 1) / nblk;
      for (int b = 0; b * rowsPer < batch; b++) {
         const int r0 = b * rowsPer, rows = (batch - r0) < rowsPer ? (batch - r0) : rowsPer;
         const size_t inOff = (size_t) r0 * rin.pitch, outOff = (size_t) r0 * rout.pitch;
         if ((e = injectCheck(copyRows((char *) rin.dev + inOff, (const char *) rin.host + inOff, rin.width, rows,
                                       rin.pitch, cudaMemcpyHostToDevice, pc->in))) != cudaSuccess ||
             (e = cudaEventRecord(pc->copied[b], pc->in)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(pc->comp, pc->copied[b], 0)) != cudaSuccess)
            return pipeFail(hc, pc, e, "copy input block");
         FirLaunch blk = a;
         blk.x = (const char *) a.x + inOff;
         blk.y = (char *) a.y + outOff;
         blk.h = (const char *) a.h + (nch ? (size_t) r0 * filtPitch * elt : 0);
         blk.batch = rows;
         if ((e = injectCheck(launchFir(blk, kind, pc->comp))) != cudaSuccess)
            return pipeFail(hc, pc, e, "FIR kernel launch");
         if ((e = cudaEventRecord(pc->computed[b], pc->comp)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(pc->out, pc->computed[b], 0)) != cudaSuccess ||
             (e = injectCheck(copyRows((char *) rout.host + outOff, (const char *) rout.dev + outOff, rout.width,
                                       rows, rout.pitch, cudaMemcpyDeviceToHost, pc->out))) != cudaSuccess)
            return pipeFail(hc, pc, e, "copy output block");
      }
      if ((e = cudaEventRecord(pc->done, pc->out)) != cudaSuccess || (e = cudaStreamWaitEvent(s, pc->done, 0)))
         return pipeFail(hc, pc, e, "pipeline join");
   }
   if (mustSync(hc, rin.staged || rf.staged || rout.staged, rin.onHost || rf.onHost || rout.onHost)) {
      if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cudaFail(hc, e, "FIR execution");
      if ((kind == FIR_INT_WRAP_TC || kind == FIR_INT_Q_TC || kind == FIR_F32_BF16X3) && takeErrorWord(hc) != 0) {
         setError(hc, "tensor-core FIR: a bounded wait for MMA completion expired; outputs are incomplete");
         return DSPLIB_ERR_FAILURE;
      }
   }
   return DSPLIB_SUCCESS;
}

void DSPLIB_fir_perfEst(DSPLIB_kernelHandle handle,
                        const DSPLIB_bufParams2D_t *bufParamsIn,
                        const DSPLIB_bufParams2D_t *bufParamsFilter,
                        const DSPLIB_bufParams2D_t *bufParamsOut,
                        uint64_t *archCycles,
                        uint64_t *estCycles)
{
   (void) bufParamsIn;
   (void) bufParamsFilter;
   (void) bufParamsOut;
   FirPriv *p = firHandle(handle);
   if (!p) return;
   // Roofline estimate in nanoseconds on a B200: HBM 6.5 TB/s; FP32 FMA
   // 70 TFLOP/s (SIMT), split-BF16x3 1.6 PFLOP/s / 3 products.
   double outs = (double) p->outputSize * p->initArgs.batchSize;
   double bytes = (double) p->elt * (outs + (double) p->initArgs.batchSize * p->initArgs.dataSize);
   double flops = 2.0 * p->initArgs.filterSize * outs;
   double peak = 70e12;
   if (p->dtype == DSPLIB_FLOAT32 && p->common.firPrecision == DSPLIB_GPU_FIR_BF16X3) peak = 1.6e15 / 3.0;
   if (p->initArgs.funcStyle == DSPLIB_FUNCTION_NATC) peak = 35e12;
   double t = bytes / 6.5e12;
   if (flops / peak > t) t = flops / peak;
   if (archCycles) *archCycles = (uint64_t) (t * 1e9);
   if (estCycles) *estCycles = (uint64_t) (t * 1e9) + 4000; // + launch and sync
}

} // extern "C"
