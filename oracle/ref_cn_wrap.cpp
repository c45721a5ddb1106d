/*
 * Thin C entry points around the reference's natural-C kernels.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled by oracle/Makefile together with the
 * reference's own DSPLIB_fir_cn.cpp, DSPLIB_cascadeBiquad_cn.cpp,
 * DSPLIB_fltoq15_cn.cpp, DSPLIB_q15tofl_cn.cpp, DSPLIB_matTrans_cn.cpp and
 * DSPLIB_addNCh_cn.cpp (taken unmodified from the read-only reference checkout) into oracle/_ref/.
 * Nothing in the product library links or loads this file; only tests/,
 * the smoke check and bench.py's CPU-baseline leg use it, as the checker.
 *
 * The reference _cn kernels read their configuration from a PrivArgs handle
 * that the reference's init() fills (src/DSPLIB_fir/DSPLIB_fir.cpp:120-176,
 * src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad.cpp:419-476).  Linking that
 * dispatcher would drag in the C7x-only _ci variants, so the handful of
 * fields the _cn code reads are filled here by hand, exactly as init() would.
 *
 * The *_mt variants split independent channels over std::threads (channels
 * never interact in either kernel: DSPLIB_fir_cn.cpp:54,
 * DSPLIB_cascadeBiquad_cn.cpp:46); they are the timed CPU baseline.
 */
#include <cstring>
#include <thread>
#include <vector>

#include "DSPLIB_fir_priv.h"
#include "DSPLIB_cascadeBiquad_priv.h"
#include "DSPLIB_fltoq15_priv.h"
#include "DSPLIB_q15tofl_priv.h"
#include "DSPLIB_matTrans_priv.h"
#include "DSPLIB_addNCh_priv.h"

namespace {

template <typename T, typename A>
int fir_one(const void *in, const void *filt, void *out, int batch, int filterSize,
            int outputSize, int inPitch, int outPitch, int enableNch, int enableMMA, int mmaSize)
{
   DSPLIB_fir_PrivArgs priv;
   std::memset(&priv, 0, sizeof(priv));
   priv.initArgs.batchSize = batch;
   priv.initArgs.filterSize = filterSize;
   priv.initArgs.enableNchCoefs = (uint32_t) enableNch;
   priv.initArgs.enableMMA = (uint32_t) enableMMA;
   priv.initArgs.MMA_SIZE = mmaSize;
   priv.dataBufferInPitch = (uint32_t) inPitch;
   priv.dataBufferOutPitch = (uint32_t) outPitch;
   priv.outputSize = outputSize;
   return (int) DSPLIB_fir_exec_cn<T, A>((DSPLIB_kernelHandle) &priv, (void *) in, (void *) filt, out);
}

int fir_dispatch(int dtype, const void *in, const void *filt, void *out, int batch, int filterSize,
                 int outputSize, int inPitch, int outPitch, int enableNch, int enableMMA, int mmaSize)
{
   switch (dtype) {
   case DSPLIB_INT8:
      return fir_one<int8_t, int32_t>(in, filt, out, batch, filterSize, outputSize, inPitch, outPitch,
                                      enableNch, enableMMA, mmaSize);
   case DSPLIB_INT16:
      return fir_one<int16_t, int64_t>(in, filt, out, batch, filterSize, outputSize, inPitch, outPitch,
                                       enableNch, enableMMA, mmaSize);
   case DSPLIB_INT32:
      return fir_one<int32_t, DSPLIB_int128_t>(in, filt, out, batch, filterSize, outputSize, inPitch,
                                               outPitch, enableNch, enableMMA, mmaSize);
   case DSPLIB_FLOAT32:
      return fir_one<float, int32_t>(in, filt, out, batch, filterSize, outputSize, inPitch, outPitch,
                                     enableNch, enableMMA, mmaSize);
   default:
      return DSPLIB_ERR_INVALID_TYPE;
   }
}

int biquad_one(int form, const void *in, const void *coef, void *state, void *out, int dataSize,
               int numStages, int numChannels, int enableNch, int inPitch, int outPitch, int varPitch)
{
   DSPLIB_cascadeBiquad_PrivArgs priv;
   std::memset(&priv, 0, sizeof(priv));
   priv.initArgs.dataSize = (uint32_t) dataSize;
   priv.initArgs.numStages = (uint32_t) numStages;
   priv.initArgs.numChannels = (uint32_t) numChannels;
   priv.initArgs.enableNChCoeffs = (uint32_t) enableNch;
   priv.initArgs.biquadForm = (uint32_t) form;
   priv.dataBufferInPitch = (uint32_t) inPitch;
   priv.dataBufferOutPitch = (uint32_t) outPitch;
   priv.filterVarPitch = (uint32_t) varPitch;
   DSPLIB_kernelHandle h = (DSPLIB_kernelHandle) &priv;
   switch (form) {
   case DSPLIB_BIQUAD_DF1:
      return (int) DSPLIB_cascadeBiquad_df1_exec_cn<float>(h, (void *) in, (void *) coef, state, out);
   case DSPLIB_BIQUAD_DF2:
   case DSPLIB_BIQUAD_TIF: /* NATC runs DF2 for the TI form: DSPLIB_cascadeBiquad.cpp:468-471 */
      return (int) DSPLIB_cascadeBiquad_df2_exec_cn<float>(h, (void *) in, (void *) coef, state, out);
   case DSPLIB_BIQUAD_TDF2:
      return (int) DSPLIB_cascadeBiquad_tdf2_exec_cn<float>(h, (void *) in, (void *) coef, state, out);
   default:
      return DSPLIB_ERR_NOT_IMPLEMENTED;
   }
}

} // namespace

extern "C" {

int ref_fir_cn(int dtype, const void *in, const void *filt, void *out, int batch, int filterSize,
               int outputSize, int inPitch, int outPitch, int enableNch, int enableMMA, int mmaSize)
{
   return fir_dispatch(dtype, in, filt, out, batch, filterSize, outputSize, inPitch, outPitch, enableNch,
                       enableMMA, mmaSize);
}

/* Channels split into contiguous blocks, one std::thread per block. */
int ref_fir_cn_mt(int dtype, const void *in, const void *filt, void *out, int batch, int filterSize,
                  int outputSize, int inPitch, int outPitch, int enableNch, int enableMMA, int mmaSize,
                  int nthreads)
{
   if (nthreads < 1) nthreads = 1;
   if (nthreads > batch) nthreads = batch;
   int esz = DSPLIB_sizeof((uint32_t) dtype);
   int filtPitch = enableNch ? (enableMMA ? (3 * mmaSize + filterSize - 1) : filterSize) : 0;
   std::vector<std::thread> th;
   std::vector<int> rc(nthreads, 0);
   for (int t = 0; t < nthreads; t++) {
      int c0 = (int) ((long long) batch * t / nthreads);
      int c1 = (int) ((long long) batch * (t + 1) / nthreads);
      th.emplace_back([=, &rc]() {
         rc[t] = fir_dispatch(dtype, (const char *) in + (size_t) c0 * inPitch * esz,
                              (const char *) filt + (size_t) c0 * filtPitch * esz,
                              (char *) out + (size_t) c0 * outPitch * esz, c1 - c0, filterSize, outputSize,
                              inPitch, outPitch, enableNch, enableMMA, mmaSize);
      });
   }
   int r = 0;
   for (int t = 0; t < nthreads; t++) {
      th[t].join();
      if (rc[t] != 0) r = rc[t];
   }
   return r;
}

int ref_biquad_cn(int form, const void *in, const void *coef, void *state, void *out, int dataSize,
                  int numStages, int numChannels, int enableNch, int inPitch, int outPitch, int varPitch)
{
   return biquad_one(form, in, coef, state, out, dataSize, numStages, numChannels, enableNch, inPitch,
                     outPitch, varPitch);
}

int ref_biquad_cn_mt(int form, const void *in, const void *coef, void *state, void *out, int dataSize,
                     int numStages, int numChannels, int enableNch, int inPitch, int outPitch, int varPitch,
                     int nthreads)
{
   if (nthreads < 1) nthreads = 1;
   if (nthreads > numChannels) nthreads = numChannels;
   std::vector<std::thread> th;
   std::vector<int> rc(nthreads, 0);
   for (int t = 0; t < nthreads; t++) {
      int c0 = (int) ((long long) numChannels * t / nthreads);
      int c1 = (int) ((long long) numChannels * (t + 1) / nthreads);
      th.emplace_back([=, &rc]() {
         rc[t] = biquad_one(form, (const float *) in + c0,
                            (const float *) coef + (enableNch ? (size_t) c0 * numStages * 5 : 0),
                            (float *) state + c0, (float *) out + c0, dataSize, numStages, c1 - c0, enableNch,
                            inPitch, outPitch, varPitch);
      });
   }
   int r = 0;
   for (int t = 0; t < nthreads; t++) {
      th[t].join();
      if (rc[t] != 0) r = rc[t];
   }
   return r;
}


/* Q.15 conversions: the reference init() stores dataSize as blockSize and
 * picks the _cn template by the float type (DSPLIB_fltoq15.cpp:64-90,
 * DSPLIB_q15tofl.cpp:64-90); the _cn code reads nothing else. */
int ref_fltoq15_cn(int dtype, const void *in, void *out, int n)
{
   DSPLIB_fltoq15_PrivArgs priv;
   std::memset(&priv, 0, sizeof(priv));
   priv.blockSize = n;
   if (dtype == DSPLIB_FLOAT32)
      return (int) DSPLIB_fltoq15_exec_cn<float>((DSPLIB_kernelHandle) &priv, (void *) in, out);
   if (dtype == DSPLIB_FLOAT64)
      return (int) DSPLIB_fltoq15_exec_cn<double>((DSPLIB_kernelHandle) &priv, (void *) in, out);
   return DSPLIB_ERR_INVALID_TYPE;
}

int ref_q15tofl_cn(int dtype, const void *in, void *out, int n)
{
   DSPLIB_q15tofl_PrivArgs priv;
   std::memset(&priv, 0, sizeof(priv));
   priv.blockSize = n;
   if (dtype == DSPLIB_FLOAT32)
      return (int) DSPLIB_q15tofl_exec_cn<float>((DSPLIB_kernelHandle) &priv, (void *) in, out);
   if (dtype == DSPLIB_FLOAT64)
      return (int) DSPLIB_q15tofl_exec_cn<double>((DSPLIB_kernelHandle) &priv, (void *) in, out);
   return DSPLIB_ERR_INVALID_TYPE;
}

/* Interleave / deinterleave: the reference init() records widthIn, heightIn and the
 * two byte strides in DSPLIB_matTrans_PrivArgs and selects DSPLIB_matTrans_exec_cn
 * by type (DSPLIB_interleave.cpp:89-253, DSPLIB_deinterleave.cpp:89-251). */
int ref_transpose_cn(int dtype, const void *in, void *out, int W, int H, int strideIn, int strideOut)
{
   DSPLIB_matTrans_PrivArgs priv;
   std::memset(&priv, 0, sizeof(priv));
   priv.widthIn = (uint32_t) W;
   priv.heightIn = (uint32_t) H;
   priv.strideIn = strideIn;
   priv.strideOut = strideOut;
   DSPLIB_kernelHandle h = (DSPLIB_kernelHandle) &priv;
   void *i = (void *) in;
   switch (dtype) {
   case DSPLIB_INT8: return (int) DSPLIB_matTrans_exec_cn<int8_t>(h, i, out);
   case DSPLIB_UINT8: return (int) DSPLIB_matTrans_exec_cn<uint8_t>(h, i, out);
   case DSPLIB_INT16: return (int) DSPLIB_matTrans_exec_cn<int16_t>(h, i, out);
   case DSPLIB_UINT16: return (int) DSPLIB_matTrans_exec_cn<uint16_t>(h, i, out);
   case DSPLIB_INT32: return (int) DSPLIB_matTrans_exec_cn<int32_t>(h, i, out);
   case DSPLIB_UINT32: return (int) DSPLIB_matTrans_exec_cn<uint32_t>(h, i, out);
   case DSPLIB_FLOAT32: return (int) DSPLIB_matTrans_exec_cn<float>(h, i, out);
   case DSPLIB_INT64: return (int) DSPLIB_matTrans_exec_cn<int64_t>(h, i, out);
   case DSPLIB_UINT64: return (int) DSPLIB_matTrans_exec_cn<uint64_t>(h, i, out);
   case DSPLIB_FLOAT64: return (int) DSPLIB_matTrans_exec_cn<double>(h, i, out);
   default: return DSPLIB_ERR_INVALID_TYPE;
   }
}

/* addNCh: the fields DSPLIB_addNCh.cpp:67-72 fills (strides in elements). */
int ref_addnch_cn(int dtype, const void *in, void *out, int samples, int channels, int inputs, int sY, int sZ,
                  int sO)
{
   DSPLIB_addNCh_PrivArgs priv;
   std::memset(&priv, 0, sizeof(priv));
   priv.samples = (uint32_t) samples;
   priv.channels = (uint32_t) channels;
   priv.inputs = (uint32_t) inputs;
   priv.strideInElementsY = sY;
   priv.strideInElementsZ = sZ;
   priv.strideOutElements = sO;
   DSPLIB_kernelHandle h = (DSPLIB_kernelHandle) &priv;
   if (dtype == DSPLIB_FLOAT32) return (int) DSPLIB_addNCh_exec_cn<float>(h, (void *) in, out);
   if (dtype == DSPLIB_FLOAT64) return (int) DSPLIB_addNCh_exec_cn<double>(h, (void *) in, out);
   return DSPLIB_ERR_INVALID_TYPE;
}

} /* extern "C" */
