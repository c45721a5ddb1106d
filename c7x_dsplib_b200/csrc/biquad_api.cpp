// DSPLIB_cascadeBiquad C-ABI entry points (drop-in for
// src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad.cpp and
// DSPLIB_cascadeBiquad_utils.cpp).  Parameter checks, descriptor sizes and the
// optimized coefficient layouts follow the reference; exec launches the CUDA
// kernels of biquad_kernels.cu.
#include <cstring>
#include <vector>

#include <string>
#include <vector>

#include "dsplib_internal.h"

using namespace dsplib;

namespace {

// Channel padding of the per-channel (channel-interleaved) coefficient rows:
// rows are padded to a multiple of 8 floats (32 bytes), the vector length the
// reference uses on 256-bit devices (utils.cpp:109-119).
constexpr uint32_t kCoefVec = 8;
constexpr uint32_t kTifCoefs = 4;      // DSPLIB_NUM_TIF_BIQUAD_COEFS
constexpr uint32_t kTifGroupStages = 7; // DSPLIB_CASCADEBIQUAD_TIF_STAGES_PER_STAGE_GROUP

bool formValid(uint32_t f)
{
   return f == DSPLIB_BIQUAD_TIF || f == DSPLIB_BIQUAD_DF1 || f == DSPLIB_BIQUAD_DF2 || f == DSPLIB_BIQUAD_TDF2;
}

// utils.cpp:81-93: one group up to 7 stages, otherwise groups of 7.
uint32_t tifGroups(uint32_t S) { return S <= kTifGroupStages ? 1u : (S + kTifGroupStages - 1) / kTifGroupStages; }
uint32_t tifPerGroup(uint32_t S) { return S <= kTifGroupStages ? S : kTifGroupStages; }

BiquadPriv *bqHandle(DSPLIB_kernelHandle h)
{
   BiquadPriv *p = (BiquadPriv *) h;
   if (!p || p->common.magic != kMagicBiquad || !p->initialized) return nullptr;
   return p;
}

// Copy a caller buffer (host or device) of `bytes` into host memory.
bool fetch(const void *src, void *dst, size_t bytes)
{
   if (bytes == 0) return true;
   if (isDevicePtr(src)) return cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost) == cudaSuccess;
   std::memcpy(dst, src, bytes);
   return true;
}

bool store(void *dst, const void *src, size_t bytes)
{
   if (bytes == 0) return true;
   if (isDevicePtr(dst)) return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice) == cudaSuccess;
   std::memcpy(dst, src, bytes);
   return true;
}

float recipOrZero(float b0) { return b0 == 0.0f ? 0.0f : 1.0f / b0; }

// An OPTIMIZED launch of this handle's problem on compact buffers (no pointers): what the
// autotuner keys and measures.  Per-channel coefficient rows are padded as exec pads them.
BiquadLaunch bqShape(const BiquadPriv *p)
{
   const DSPLIB_cascadeBiquad_InitArgs &ia = p->initArgs;
   BiquadLaunch a{};
   a.form = (int) ia.biquadForm;
   a.nch = ia.enableNChCoeffs ? 1 : 0;
   a.optLayout = 1;
   a.N = (int) ia.dataSize;
   a.C = (int) ia.numChannels;
   a.S = (int) ia.numStages;
   a.inPitch = a.outPitch = a.varPitch = a.C;
   a.coefPitch = a.nch ? (a.C + kCoefVec - 1) / kCoefVec * kCoefVec : 0;
   a.prefetch = 1;
   return a;
}

// The handle's cached scan choice, resolved again when the table changed.
int bqChoice(BiquadPriv *p, const BiquadLaunch &a)
{
   const unsigned gen = tuneGeneration();
   if (p->tuneGen != gen) {
      int c = -1;
      const std::string key = biquadTuneKey(a);
      if (key.empty() || !tuneLookup(key, &c)) c = -1;
      p->tuneGen = gen;
      p->tuneChoice = c;
   }
   return p->tuneChoice;
}

} // namespace

namespace dsplib {

std::string biquadHandleTuneKey(DSPLIB_kernelHandle h, std::vector<int> *cands)
{
   BiquadPriv *p = bqHandle(h);
   if (!p || p->initArgs.funcStyle == DSPLIB_FUNCTION_NATC || !formValid(p->initArgs.biquadForm)) return std::string();
   const BiquadLaunch a = bqShape(p);
   if (cands) *cands = biquadTuneCandidates(a);
   return biquadTuneKey(a);
}

// Every candidate shape on a scratch signal of the handle's sizes filled with a hashed
// pattern, zero states and coefficients (the scan's work does not depend on them), on a
// private stream.
DSPLIB_STATUS biquadHandleTune(DSPLIB_kernelHandle h)
{
   BiquadPriv *p = bqHandle(h);
   if (!p) return DSPLIB_ERR_NULL_POINTER;
   std::vector<int> cands;
   const std::string key = biquadHandleTuneKey(h, &cands);
   if (key.empty() || cands.empty()) return DSPLIB_ERR_NOT_IMPLEMENTED;
   BiquadLaunch a = bqShape(p);
   const int nv = a.form == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   const size_t rows = a.form == DSPLIB_BIQUAD_TIF ? (size_t) a.S * 4 + tifGroups(a.S) : (size_t) a.S * 5;
   const size_t xb = (size_t) a.N * a.C * 4, sb = (size_t) a.S * nv * a.C * 4;
   const size_t cb = (a.nch ? rows * (size_t) a.coefPitch : rows) * 4;
   void *x = nullptr, *y = nullptr, *st = nullptr, *cf = nullptr;
   DSPLIB_STATUS status = DSPLIB_ERR_FAILURE;
   if (cudaMalloc(&x, xb) == cudaSuccess && cudaMalloc(&y, xb) == cudaSuccess && cudaMalloc(&st, sb) == cudaSuccess &&
       cudaMalloc(&cf, cb) == cudaSuccess && tuneFill(x, xb, true) && cudaMemset(st, 0, sb) == cudaSuccess &&
       cudaMemset(cf, 0, cb) == cudaSuccess) {
      a.x = (const float *) x;
      a.y = (float *) y;
      a.state = (float *) st;
      a.coef = (const float *) cf;
      const int best = tunePick(key, cands, [&](int c, cudaStream_t s) {
         BiquadLaunch b = a;
         b.tuneChoice = c;
         return launchBiquadScan(b, s);
      });
      if (best >= 0) status = DSPLIB_SUCCESS;
   }
   (void) cudaGetLastError();
   cudaFree(x);
   cudaFree(y);
   cudaFree(st);
   cudaFree(cf);
   p->tuneGen = 0;
   return status;
}

} // namespace dsplib

extern "C" {

int32_t DSPLIB_cascadeBiquad_getHandleSize(DSPLIB_cascadeBiquad_InitArgs *pKerInitArgs)
{
   (void) pKerInitArgs;
   return (int32_t) sizeof(BiquadPriv);
}

DSPLIB_STATUS DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(uint32_t dataType,
                                                              uint32_t numStages,
                                                              uint32_t numChannels,
                                                              uint32_t biquadForm,
                                                              uint32_t enableNChCoeffs,
                                                              DSPLIB_bufParams2D_t *d)
{
   // utils.cpp:57-72
   if (d == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (dataType != DSPLIB_FLOAT32) return DSPLIB_ERR_INVALID_TYPE;
   if (!formValid(biquadForm)) return DSPLIB_ERR_INVALID_VALUE;
   if (enableNChCoeffs != 0 && enableNChCoeffs != 1) return DSPLIB_ERR_INVALID_VALUE;
   d->data_type = dataType;
   const uint32_t padded = (numChannels + kCoefVec - 1) / kCoefVec * kCoefVec;
   if (biquadForm == DSPLIB_BIQUAD_TIF) { // utils.cpp:78-121
      const uint32_t G = tifGroups(numStages);
      if (enableNChCoeffs == 0) {
         d->dim_x = numStages * kTifCoefs + G;
         d->dim_y = 1;
         d->stride_y = (int32_t) (d->dim_x * 4);
      }
      else {
         d->dim_x = numChannels;
         d->dim_y = numStages * kTifCoefs + G;
         d->stride_y = (int32_t) (padded * 4);
      }
   }
   else { // utils.cpp:122-152
      if (enableNChCoeffs == 0) {
         d->dim_x = numStages * DSPLIB_NUM_BIQUAD_COEFS;
         d->dim_y = 1;
         d->stride_y = (int32_t) (d->dim_x * 4);
      }
      else {
         d->dim_x = numChannels;
         d->dim_y = numStages * DSPLIB_NUM_BIQUAD_COEFS;
         d->stride_y = (int32_t) (padded * 4);
      }
   }
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_cascadeBiquad_get_coefficients(uint32_t biquadForm,
                                                    uint32_t enableNChCoeffs,
                                                    DSPLIB_bufParams2D_t *pIn,
                                                    DSPLIB_bufParams2D_t *pOpt,
                                                    const void *pFilterCoeff,
                                                    const void *pFilterCoeffOpt)
{
   // utils.cpp:661-677
   if (pIn == NULL || pOpt == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (pIn->data_type != DSPLIB_FLOAT32 || pOpt->data_type != DSPLIB_FLOAT32) return DSPLIB_ERR_INVALID_TYPE;
   if (!formValid(biquadForm)) return DSPLIB_ERR_INVALID_VALUE;
   if (enableNChCoeffs != 0 && enableNChCoeffs != 1) return DSPLIB_ERR_INVALID_VALUE;
   if (biquadForm != DSPLIB_BIQUAD_TIF && enableNChCoeffs == 0) return DSPLIB_ERR_INVALID_VALUE; // :691-694
   if (pFilterCoeff == NULL || pFilterCoeffOpt == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (pIn->dim_x % DSPLIB_NUM_BIQUAD_COEFS != 0) return DSPLIB_ERR_NOT_ALIGNED_WIDTHS; // :179-181, :503-505

   const uint32_t S = pIn->dim_x / DSPLIB_NUM_BIQUAD_COEFS;
   const uint32_t C = enableNChCoeffs ? pIn->dim_y : 1;
   // Both buffers in device memory: the transform runs on the GPU, in place (the call
   // returns once it is done, as the host form does).
   if (isDevicePtr(pFilterCoeff) && isDevicePtr(pFilterCoeffOpt)) {
      const long long pitch = enableNChCoeffs ? (long long) pOpt->stride_y / 4 : 0;
      if (enableNChCoeffs && pitch < (long long) C) return DSPLIB_ERR_INVALID_DIMENSION;
      if (launchBiquadCoefTransform(biquadForm == DSPLIB_BIQUAD_TIF, (int) enableNChCoeffs,
                                    (const float *) pFilterCoeff, (float *) pFilterCoeffOpt, (int) S, (int) C, pitch,
                                    0) != cudaSuccess ||
          cudaStreamSynchronize(0) != cudaSuccess)
         return DSPLIB_ERR_FAILURE;
      return DSPLIB_SUCCESS;
   }
   // Natural coefficients are read densely, [ch][stage][5] (utils.cpp:340-360).
   std::vector<float> nat((size_t) C * S * DSPLIB_NUM_BIQUAD_COEFS);
   if (!fetch(pFilterCoeff, nat.data(), nat.size() * 4)) return DSPLIB_ERR_FAILURE;

   if (biquadForm == DSPLIB_BIQUAD_TIF) {
      const uint32_t G = tifGroups(S), per = tifPerGroup(S);
      if (enableNChCoeffs == 0) {
         // utils.cpp:198-266: per stage {b1/b0 - a1, b2/b0 - a2, -a2, -a1}, then one gain per group.
         std::vector<float> out((size_t) S * kTifCoefs + G);
         for (uint32_t g = 0; g < G; g++) {
            float gain = 1.0f;
            for (uint32_t s = g * per; s < S && s < (g + 1) * per; s++) {
               const float *c = &nat[(size_t) s * 5];
               float r = recipOrZero(c[0]);
               float b1 = c[1] * r, b2 = c[2] * r, a1 = -c[3], a2 = -c[4];
               gain = gain * c[0];
               out[s * 4 + 0] = b1 + a1;
               out[s * 4 + 1] = b2 + a2;
               out[s * 4 + 2] = a2;
               out[s * 4 + 3] = a1;
            }
            out[(size_t) S * 4 + g] = gain;
         }
         if (!store((void *) pFilterCoeffOpt, out.data(), out.size() * 4)) return DSPLIB_ERR_FAILURE;
      }
      else {
         // utils.cpp:268-471: coefficient k of stage s for channel ch at row
         // k*S + s, column ch; gain of group g at row 4*S + g.
         const size_t pitch = (size_t) pOpt->stride_y / 4;
         if (pitch < C) return DSPLIB_ERR_INVALID_DIMENSION;
         const size_t rows = (size_t) S * kTifCoefs + G;
         std::vector<float> out(rows * pitch, 0.0f);
         if (!fetch(pFilterCoeffOpt, out.data(), out.size() * 4)) return DSPLIB_ERR_FAILURE;
         for (uint32_t ch = 0; ch < C; ch++) {
            for (uint32_t g = 0; g < G; g++) {
               float gain = 1.0f;
               for (uint32_t s = g * per; s < S && s < (g + 1) * per; s++) {
                  const float *c = &nat[((size_t) ch * S + s) * 5];
                  gain = c[0] * gain;
                  float r = recipOrZero(c[0]);
                  float b1 = c[1] * r, b2 = c[2] * r, a1 = -c[3], a2 = -c[4];
                  out[((size_t) 0 * S + s) * pitch + ch] = b1 + a1;
                  out[((size_t) 1 * S + s) * pitch + ch] = b2 + a2;
                  out[((size_t) 2 * S + s) * pitch + ch] = a2;
                  out[((size_t) 3 * S + s) * pitch + ch] = a1;
               }
               out[((size_t) S * 4 + g) * pitch + ch] = gain;
            }
         }
         if (!store((void *) pFilterCoeffOpt, out.data(), out.size() * 4)) return DSPLIB_ERR_FAILURE;
      }
      return DSPLIB_SUCCESS;
   }
   // DF1/DF2/TDF2 with per-channel coefficients (utils.cpp:477-650): stage s,
   // coefficient k of channel ch at row s*5 + k, column ch.
   const size_t pitch = (size_t) pOpt->stride_y / 4;
   if (pitch < C) return DSPLIB_ERR_INVALID_DIMENSION;
   const size_t rows = (size_t) S * DSPLIB_NUM_BIQUAD_COEFS;
   std::vector<float> out(rows * pitch, 0.0f);
   if (!fetch(pFilterCoeffOpt, out.data(), out.size() * 4)) return DSPLIB_ERR_FAILURE;
   for (uint32_t ch = 0; ch < C; ch++)
      for (size_t r = 0; r < rows; r++) out[r * pitch + ch] = nat[(size_t) ch * rows + r];
   if (!store((void *) pFilterCoeffOpt, out.data(), out.size() * 4)) return DSPLIB_ERR_FAILURE;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_cascadeBiquad_init_checkParams(DSPLIB_kernelHandle handle,
                                                    const DSPLIB_bufParams2D_t *bufParamsIn,
                                                    const DSPLIB_bufParams2D_t *bufParamsFilterCoeff,
                                                    const DSPLIB_bufParams2D_t *bufParamsFilterVar,
                                                    const DSPLIB_bufParams2D_t *bufParamsOut,
                                                    const DSPLIB_cascadeBiquad_InitArgs *a)
{
   // DSPLIB_cascadeBiquad.cpp:343-396, same order of checks.
   if (handle == NULL) return DSPLIB_ERR_NULL_POINTER;
   if (bufParamsIn->data_type != DSPLIB_FLOAT32) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->data_type != bufParamsFilterCoeff->data_type) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->data_type != bufParamsFilterVar->data_type) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->data_type != bufParamsOut->data_type) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->stride_y != bufParamsOut->stride_y) return DSPLIB_ERR_NOT_IMPLEMENTED;
   if (a->funcStyle != DSPLIB_FUNCTION_NATC && a->funcStyle != DSPLIB_FUNCTION_OPTIMIZED)
      return DSPLIB_ERR_INVALID_VALUE;
   if (a->dataSize == 0 || a->numChannels == 0 || a->numStages == 0) return DSPLIB_ERR_INVALID_VALUE;
   if (!formValid(a->biquadForm)) return DSPLIB_ERR_INVALID_VALUE;
   if (a->enableNChCoeffs != 0 && a->enableNChCoeffs != 1) return DSPLIB_ERR_INVALID_VALUE;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_cascadeBiquad_exec_checkParams(DSPLIB_kernelHandle handle,
                                                    const void *pIn,
                                                    const void *pFilterCoeff,
                                                    const void *pFilterVar,
                                                    const void *pOut)
{
   (void) handle;
   if (pIn == NULL || pFilterCoeff == NULL || pFilterVar == NULL || pOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_cascadeBiquad_init(DSPLIB_kernelHandle handle,
                                        DSPLIB_bufParams2D_t *bufParamsIn,
                                        DSPLIB_bufParams2D_t *bufParamsFilterCoeff,
                                        DSPLIB_bufParams2D_t *bufParamsFilterVar,
                                        DSPLIB_bufParams2D_t *bufParamsOut,
                                        DSPLIB_cascadeBiquad_InitArgs *a)
{
   if (handle == NULL || a == NULL || bufParamsIn == NULL || bufParamsOut == NULL) return DSPLIB_ERR_NULL_POINTER;
   BiquadPriv *p = (BiquadPriv *) handle;
   if (p->common.magic != kMagicBiquad) {
      std::memset(&p->common, 0, sizeof(p->common));
      p->common.magic = kMagicBiquad;
   }
   p->common.err[0] = 0;
   p->initArgs = *a;
   p->initialized = 0;
   // DSPLIB_cascadeBiquad.cpp:433-453
   if (bufParamsIn->data_type != DSPLIB_FLOAT32) return DSPLIB_ERR_INVALID_TYPE;
   if (bufParamsIn->stride_y != bufParamsOut->stride_y) return DSPLIB_ERR_NOT_IMPLEMENTED;
   p->inPitch = bufParamsIn->stride_y / 4;
   p->outPitch = bufParamsOut->stride_y / 4;
   p->varPitch = bufParamsFilterVar ? bufParamsFilterVar->stride_y / 4 : 0;
   p->coefPitch = bufParamsFilterCoeff ? bufParamsFilterCoeff->stride_y / 4 : 0;
   p->coefRows = bufParamsFilterCoeff ? (int32_t) bufParamsFilterCoeff->dim_y : 0;
   p->coefCols = bufParamsFilterCoeff ? (int32_t) bufParamsFilterCoeff->dim_x : 0;
   if (!formValid(a->biquadForm)) return DSPLIB_ERR_NOT_IMPLEMENTED; // :472-474, :611-614
   if (a->funcStyle != DSPLIB_FUNCTION_NATC) p->initArgs.funcStyle = DSPLIB_FUNCTION_OPTIMIZED;
   p->initialized = 1;
   p->tuneGen = 0;
   if (tuneMode() == DSPLIB_GPU_TUNE_MEASURE) {
      int c = 0;
      const std::string key = biquadHandleTuneKey(handle, nullptr);
      if (!key.empty() && !tuneLookup(key, &c)) (void) biquadHandleTune(handle); // a failed measurement keeps the rule
   }
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_cascadeBiquad_exec(DSPLIB_kernelHandle handle,
                                        void *pIn,
                                        void *pFilterCoeff,
                                        void *pFilterVar,
                                        void *pOut)
{
   BiquadPriv *p = bqHandle(handle);
   if (!p) return DSPLIB_ERR_FAILURE;
   HandleCommon *hc = &p->common;
   if (!pIn || !pFilterCoeff || !pFilterVar || !pOut) {
      setError(hc, "exec: null buffer");
      return DSPLIB_ERR_NULL_POINTER;
   }
   const DSPLIB_cascadeBiquad_InitArgs &ia = p->initArgs;
   const int N = (int) ia.dataSize, C = (int) ia.numChannels, S = (int) ia.numStages;
   if (N <= 0 || C <= 0 || S <= 0) return DSPLIB_SUCCESS;
   const bool natc = ia.funcStyle == DSPLIB_FUNCTION_NATC;
   const bool nch = ia.enableNChCoeffs != 0;
   // NATC runs DF2 for the TI form on natural coefficients (DSPLIB_cascadeBiquad.cpp:468-471).
   const int form = (natc && ia.biquadForm == DSPLIB_BIQUAD_TIF) ? DSPLIB_BIQUAD_DF2 : (int) ia.biquadForm;
   const int nv = form == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   if (p->inPitch < C || p->outPitch < C || p->varPitch < C) {
      setError(hc, "exec: pitch smaller than the channel count (in %d, out %d, state %d, C %d)", p->inPitch,
               p->outPitch, p->varPitch, C);
      return DSPLIB_ERR_INVALID_DIMENSION;
   }

   // Coefficient buffer extent.
   long long coefPitch = 0;
   size_t cw, ch, cp;
   if (natc || !nch) {
      size_t perRow = (natc || form != DSPLIB_BIQUAD_TIF) ? (size_t) S * 5 : (size_t) S * 4 + tifGroups(S);
      cw = perRow * 4;
      ch = (natc && nch) ? (size_t) C : 1;
      cp = cw;
   }
   else {
      coefPitch = p->coefPitch;
      if (coefPitch < C) coefPitch = (C + kCoefVec - 1) / kCoefVec * kCoefVec;
      size_t rows = form == DSPLIB_BIQUAD_TIF ? (size_t) S * 4 + tifGroups(S) : (size_t) S * 5;
      cw = (size_t) C * 4;
      ch = rows;
      cp = (size_t) coefPitch * 4;
   }

   cudaStream_t s = hc->stream;
   Region rin{pIn, nullptr, (size_t) C * 4, (size_t) N, (size_t) p->inPitch * 4, false};
   Region rout{pOut, nullptr, (size_t) C * 4, (size_t) N, (size_t) p->outPitch * 4, false};
   // Page-locked signal buffers are read and written in place by the lane-per-channel scan
   // kernel, which reads each input sample once and writes each output sample once, one
   // coalesced row of 32 channels or more at a time: its loads and stores cross PCIe in
   // both directions at once.  The sequential kernel (NATC, deep cascades) revisits the
   // output once per stage and narrower rows are scattered, so those are staged.
   const bool scanInPlace = !natc && S <= biquadScanMaxStages() && C >= 32 && pOut != pIn;
   const bool pinned = !isDevicePtr(pIn) && !isDevicePtr(pOut) && mappedHostPtr(pIn) && mappedHostPtr(pOut);
   // Page-locked host signals of 4 MB or more: copy in, filter and copy out blocks of rows
   // (time) in a pipeline on three streams, so that both copy directions and the kernels
   // overlap (timed on B200 over PCIe: 128 MB each way 3.5 ms against 4.9 ms in place,
   // 16 channels x 262144 0.72 ms against 1.10 ms staged whole).  Each block's kernel
   // starts from the state the previous block's kernel left in the state buffer, the
   // streaming contract of the entry point, so the blocks chain into the same recursion
   // as one call over all rows.  Pageable buffers are staged whole: the driver's copies
   // out of pageable memory are slower when split.
   PipeContext *pc = nullptr;
   if (pinned && N >= 64 && rin.bytes() >= kBqPipeMinBytes) pc = pipeContext();
   if (scanInPlace && !pc) {
      rin.zeroCopy = rin.streamed = true;
      rout.zeroCopy = rout.streamed = true;
   }
   // states and coefficients are read (states also written) about once per channel and stage
   Region rst{pFilterVar, nullptr, (size_t) C * 4, (size_t) S * nv, (size_t) p->varPitch * 4, false, true};
   Region rc{pFilterCoeff, nullptr, cw, ch, cp, false, true};
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
   if ((e = injectCheck(regionIn(rc, 1, true, sIn))) != cudaSuccess) return pipeFail(hc, pc, e, "stage coefficients");
   if ((e = injectCheck(regionIn(rst, 3, true, sIn))) != cudaSuccess) return pipeFail(hc, pc, e, "stage state");
   if (pOut == pIn && rin.staged) {
      rout = rin; // in-place on a host buffer: the staged copy is both input and output
   }
   else if ((e = injectCheck(regionIn(rout, 2, false, sIn))) != cudaSuccess) {
      return pipeFail(hc, pc, e, "stage output");
   }

   BiquadLaunch a;
   a.x = (const float *) rin.dev;
   a.y = (float *) rout.dev;
   a.state = (float *) rst.dev;
   a.coef = (const float *) rc.dev;
   a.form = form;
   a.nch = nch ? 1 : 0;
   a.optLayout = natc ? 0 : 1;
   a.N = N;
   a.C = C;
   a.S = S;
   a.inPitch = p->inPitch;
   a.outPitch = p->outPitch;
   a.varPitch = p->varPitch;
   a.coefPitch = coefPitch;
   a.prefetch = (!rin.onHost || rin.staged) ? 1 : 0; // not for mapped host memory
   if (!natc) a.tuneChoice = bqChoice(p, bqShape(p));
   auto launch = [&](const BiquadLaunch &l, cudaStream_t st) {
      return natc ? launchBiquadSequential(l, st) : launchBiquadScan(l, st);
   };
   if (!pc) {
      if ((e = injectCheck(launch(a, s))) != cudaSuccess) return cudaFail(hc, e, "biquad kernel launch");
      if ((e = injectCheck(regionOut(rout, s))) != cudaSuccess) return cudaFail(hc, e, "copy output");
   }
   else {
      int nblk = (int) (rin.bytes() / kBqPipeBlockBytes);
      nblk = nblk < 2 ? 2 : (nblk > kPipeMaxBlocks ? kPipeMaxBlocks : nblk);
      // rows per block: a multiple of 32 (whole chunks of the scan kernel)
      const int rowsPer = ((N + nblk - 1) / nblk + 31) / 32 * 32;
      for (int b = 0; b * rowsPer < N; b++) {
         const int r0 = b * rowsPer, rows = (N - r0) < rowsPer ? (N - r0) : rowsPer;
         const size_t inOff = (size_t) r0 * rin.pitch, outOff = (size_t) r0 * rout.pitch;
         if ((e = injectCheck(copyRows((char *) rin.dev + inOff, (const char *) rin.host + inOff, rin.width, rows,
                                       rin.pitch, cudaMemcpyHostToDevice, pc->in))) != cudaSuccess ||
             (e = cudaEventRecord(pc->copied[b], pc->in)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(pc->comp, pc->copied[b], 0)) != cudaSuccess)
            return pipeFail(hc, pc, e, "copy input block");
         BiquadLaunch blk = a;
         blk.x = a.x + (size_t) r0 * a.inPitch;
         blk.y = a.y + (size_t) r0 * a.outPitch;
         blk.N = rows;
         if ((e = injectCheck(launch(blk, pc->comp))) != cudaSuccess) return pipeFail(hc, pc, e, "biquad kernel launch");
         if ((e = cudaEventRecord(pc->computed[b], pc->comp)) != cudaSuccess ||
             (e = cudaStreamWaitEvent(pc->out, pc->computed[b], 0)) != cudaSuccess ||
             (e = injectCheck(copyRows((char *) rout.host + outOff, (const char *) rout.dev + outOff, rout.width,
                                       rows, rout.pitch, cudaMemcpyDeviceToHost, pc->out))) != cudaSuccess)
            return pipeFail(hc, pc, e, "copy output block");
      }
      // the state is final once the last block's kernel has run (the out stream waited for it)
      if ((e = cudaEventRecord(pc->done, pc->out)) != cudaSuccess || (e = cudaStreamWaitEvent(s, pc->done, 0)))
         return pipeFail(hc, pc, e, "pipeline join");
   }
   if ((e = injectCheck(regionOut(rst, s))) != cudaSuccess) return pipeFail(hc, pc, e, "copy state");
   if (mustSync(hc, rin.staged || rout.staged || rst.staged || rc.staged,
                rin.onHost || rout.onHost || rst.onHost || rc.onHost)) {
      if ((e = cudaStreamSynchronize(s)) != cudaSuccess) return cudaFail(hc, e, "biquad execution");
   }
   return DSPLIB_SUCCESS;
}

void DSPLIB_cascadeBiquad_perfEst(DSPLIB_kernelHandle handle,
                                  const DSPLIB_bufParams2D_t *bufParamsIn,
                                  const DSPLIB_bufParams2D_t *bufParamsFilterCoeff,
                                  const DSPLIB_bufParams2D_t *bufParamsFilterVar,
                                  const DSPLIB_bufParams2D_t *bufParamsOut,
                                  uint64_t *archCycles,
                                  uint64_t *estCycles)
{
   (void) bufParamsIn;
   (void) bufParamsFilterCoeff;
   (void) bufParamsFilterVar;
   (void) bufParamsOut;
   BiquadPriv *p = bqHandle(handle);
   if (!p) return;
   // Roofline in nanoseconds: bytes = 4*(in + out) + coefficients + 2*state, HBM 6.5 TB/s.
   double samples = (double) p->initArgs.dataSize * p->initArgs.numChannels;
   double bytes = 8.0 * samples + 20.0 * p->initArgs.numStages * p->initArgs.numChannels;
   double t = bytes / 6.5e12;
   if (p->initArgs.funcStyle == DSPLIB_FUNCTION_NATC) {
      // one sequential recursion per channel: ~25 ns per stage-sample on one thread
      double seq = 25e-9 * p->initArgs.dataSize * p->initArgs.numStages;
      if (seq > t) t = seq;
   }
   if (archCycles) *archCycles = (uint64_t) (t * 1e9);
   if (estCycles) *estCycles = (uint64_t) (t * 1e9) + 5000;
}

} // extern "C"
