// FIR CUDA kernels for sm_100a.
//
//   fir_direct_kernel  one output per thread per tile, taps in shared memory.
//                      MODE_NATC reproduces the reference natural-C kernel
//                      (src/DSPLIB_fir/DSPLIB_fir_cn.cpp:54-83) bit for bit:
//                      integers wrap modulo 2^32 before the truncating store
//                      (the reference sums modulo 2^bits; 2^bits divides 2^32),
//                      floats are summed in tap order with separately rounded
//                      multiply and add.  MODE_Q keeps the exact accumulator
//                      and applies round-half-up / shift / saturate.
//   fir_f32_simt_kernel the plain FP32 CUDA-core kernel: 8 consecutive outputs
//                      per thread held in registers, taps unrolled by 8, fused
//                      multiply-add.
//
// Layout (channel-major, DSPLIB_fir_cn.cpp:57-58): x[l*inPitch + t],
// y[l*outPitch + j]; stored taps h[T-1-c] multiply x[j+c].
#include <cuda_runtime.h>

#include <cstdint>

#include "dsplib_internal.h"

namespace dsplib {

namespace {

constexpr int MODE_NATC = 0;
constexpr int MODE_Q = 1;

template <typename T> struct QLimits;
template <> struct QLimits<int8_t> { static constexpr long long lo = -128, hi = 127; };
template <> struct QLimits<int16_t> { static constexpr long long lo = -32768, hi = 32767; };
template <> struct QLimits<int32_t> { static constexpr long long lo = -2147483648LL, hi = 2147483647LL; };

template <typename T, int MODE> struct Acc;
template <> struct Acc<float, MODE_NATC> {
   float v = 0.0f;
   __device__ void add(float x, float h) { v = __fadd_rn(v, __fmul_rn(x, h)); }
   __device__ float out(int) const { return v; }
};
template <typename T> struct Acc<T, MODE_NATC> {
   uint32_t v = 0;
   __device__ void add(T x, T h) { v += (uint32_t) (int32_t) x * (uint32_t) (int32_t) h; }
   __device__ T out(int) const { return (T) v; }
};
template <typename T> struct Acc<T, MODE_Q> {
   // int8/int16 products fit 31 bits; 2^32 taps would still fit int64.  int32
   // products need 63 bits, so that case accumulates in 128 bits.
   using W = typename std::conditional<sizeof(T) == 4, __int128, long long>::type;
   W v = 0;
   __device__ void add(T x, T h) { v += (W) x * (W) h; }
   __device__ T out(int shift) const
   {
      W r = v;
      if (shift > 0) r = (r + ((W) 1 << (shift - 1))) >> shift;
      if (r < (W) QLimits<T>::lo) r = (W) QLimits<T>::lo;
      if (r > (W) QLimits<T>::hi) r = (W) QLimits<T>::hi;
      return (T) r;
   }
};

constexpr int kDirTile = 1024; // outputs per CTA
constexpr int kDirTaps = 1024; // taps per shared-memory block
constexpr int kDirThreads = 256;

template <typename T, int MODE>
__global__ void __launch_bounds__(kDirThreads) fir_direct_kernel(FirLaunch a)
{
   __shared__ T xs[kDirTile + kDirTaps];
   __shared__ T hs[kDirTaps];
   const int j0 = blockIdx.x * kDirTile;
   const long long inExtent = (long long) a.outSize + a.T - 1; // samples of a row that are read
   for (int l = blockIdx.y; l < a.batch; l += gridDim.y) {
      const T *x = (const T *) a.x + (long long) l * a.inPitch;
      const T *h = (const T *) a.h + (long long) l * a.filtPitch;
      T *y = (T *) a.y + (long long) l * a.outPitch;
      Acc<T, MODE> acc[kDirTile / kDirThreads];
      for (int cb = 0; cb < a.T; cb += kDirTaps) {
         const int tb = min(kDirTaps, a.T - cb);
         for (int k = threadIdx.x; k < kDirTile + tb - 1; k += kDirThreads) {
            long long idx = (long long) j0 + cb + k;
            xs[k] = idx < inExtent ? x[idx] : (T) 0;
         }
         for (int k = threadIdx.x; k < tb; k += kDirThreads) hs[k] = h[a.T - 1 - (cb + k)];
         __syncthreads();
#pragma unroll
         for (int r = 0; r < kDirTile / kDirThreads; r++) {
            const int j = threadIdx.x + r * kDirThreads;
            if (j0 + j < a.outSize) {
               for (int c = 0; c < tb; c++) acc[r].add(xs[j + c], hs[c]);
            }
         }
         __syncthreads();
      }
#pragma unroll
      for (int r = 0; r < kDirTile / kDirThreads; r++) {
         const int j = threadIdx.x + r * kDirThreads;
         if (j0 + j < a.outSize) y[j0 + j] = acc[r].out(a.shift);
      }
   }
}

// FLOAT32 filters in Q mode (InitArgs.enableQ): the C7x fixed-point MMA path of
// src/DSPLIB_fir/DSPLIB_fir_ci.cpp:1559-1625.  Signal and taps are scaled by 2^Q and
// converted to int32 (round to nearest even, saturating; NaN -> 0), the products are
// summed exactly (128 bits), the sum is shifted right by Q with half-LSB rounding and
// saturated to int32 (the MMA output stage, X_SHIFT = Q with rounding and saturation),
// then converted to float and scaled by 2^-Q.
__device__ __forceinline__ int quantQ(float v, float scale) { return __float2int_rn(v * scale); }

__global__ void __launch_bounds__(kDirThreads) fir_floatq_kernel(FirLaunch a)
{
   __shared__ int xs[kDirTile + kDirTaps];
   __shared__ int hs[kDirTaps];
   const int j0 = blockIdx.x * kDirTile;
   const long long inExtent = (long long) a.outSize + a.T - 1;
   const int Q = a.shift;
   const float scale = ldexpf(1.0f, Q), unscale = ldexpf(1.0f, -Q);
   for (int l = blockIdx.y; l < a.batch; l += gridDim.y) {
      const float *x = (const float *) a.x + (long long) l * a.inPitch;
      const float *h = (const float *) a.h + (long long) l * a.filtPitch;
      float *y = (float *) a.y + (long long) l * a.outPitch;
      __int128 acc[kDirTile / kDirThreads];
#pragma unroll
      for (int r = 0; r < kDirTile / kDirThreads; r++) acc[r] = 0;
      for (int cb = 0; cb < a.T; cb += kDirTaps) {
         const int tb = min(kDirTaps, a.T - cb);
         for (int k = threadIdx.x; k < kDirTile + tb - 1; k += kDirThreads) {
            long long idx = (long long) j0 + cb + k;
            xs[k] = idx < inExtent ? quantQ(x[idx], scale) : 0;
         }
         for (int k = threadIdx.x; k < tb; k += kDirThreads) hs[k] = quantQ(h[a.T - 1 - (cb + k)], scale);
         __syncthreads();
#pragma unroll
         for (int r = 0; r < kDirTile / kDirThreads; r++) {
            const int j = threadIdx.x + r * kDirThreads;
            if (j0 + j < a.outSize)
               for (int c = 0; c < tb; c++) acc[r] += (__int128) ((long long) xs[j + c] * (long long) hs[c]);
         }
         __syncthreads();
      }
#pragma unroll
      for (int r = 0; r < kDirTile / kDirThreads; r++) {
         const int j = threadIdx.x + r * kDirThreads;
         if (j0 + j < a.outSize) {
            __int128 v = acc[r];
            if (Q > 0) v = (v + ((__int128) 1 << (Q - 1))) >> Q;
            if (v < (__int128) INT32_MIN) v = INT32_MIN;
            if (v > (__int128) INT32_MAX) v = INT32_MAX;
            y[j0 + j] = (float) (int) v * unscale;
         }
      }
   }
}

constexpr int kSimtTile = 2048; // outputs per CTA, 8 per thread
constexpr int kSimtTaps = 256;  // taps per shared-memory block
constexpr int kSimtThreads = 256;

__global__ void __launch_bounds__(kSimtThreads) fir_f32_simt_kernel(FirLaunch a)
{
   __shared__ __align__(16) float xs[kSimtTile + kSimtTaps + 8];
   __shared__ __align__(16) float gs[kSimtTaps];
   const int j0 = blockIdx.x * kSimtTile;
   const long long inExtent = (long long) a.outSize + a.T - 1;
   for (int l = blockIdx.y; l < a.batch; l += gridDim.y) {
      const float *x = (const float *) a.x + (long long) l * a.inPitch;
      const float *h = (const float *) a.h + (long long) l * a.filtPitch;
      float *y = (float *) a.y + (long long) l * a.outPitch;
      float acc[8];
#pragma unroll
      for (int r = 0; r < 8; r++) acc[r] = 0.0f;
      for (int cb = 0; cb < a.T; cb += kSimtTaps) {
         const int tb = min(kSimtTaps, a.T - cb);
         const int tbr = (tb + 7) & ~7;
         for (int k = threadIdx.x; k < kSimtTile + tbr + 8; k += kSimtThreads) {
            long long idx = (long long) j0 + cb + k;
            xs[k] = idx < inExtent ? x[idx] : 0.0f;
         }
         for (int k = threadIdx.x; k < tbr; k += kSimtThreads) gs[k] = k < tb ? h[a.T - 1 - (cb + k)] : 0.0f;
         __syncthreads();
         const float *xw = xs + 8 * threadIdx.x;
         for (int c = 0; c < tbr; c += 8) {
            float w[16], g[8];
            *(float4 *) &w[0] = *(const float4 *) &xw[c];
            *(float4 *) &w[4] = *(const float4 *) &xw[c + 4];
            *(float4 *) &w[8] = *(const float4 *) &xw[c + 8];
            *(float4 *) &w[12] = *(const float4 *) &xw[c + 12];
            *(float4 *) &g[0] = *(const float4 *) &gs[c];
            *(float4 *) &g[4] = *(const float4 *) &gs[c + 4];
#pragma unroll
            for (int i = 0; i < 8; i++) {
#pragma unroll
               for (int r = 0; r < 8; r++) acc[r] = fmaf(w[r + i], g[i], acc[r]);
            }
         }
         __syncthreads();
      }
      // Stage the 8 consecutive outputs per thread through shared memory so
      // the global stores are coalesced.
#pragma unroll
      for (int r = 0; r < 8; r++) xs[8 * threadIdx.x + r] = acc[r];
      __syncthreads();
      for (int k = threadIdx.x; k < kSimtTile; k += kSimtThreads)
         if (j0 + k < a.outSize) y[j0 + k] = xs[k];
      __syncthreads();
   }
}

template <typename T, int MODE> cudaError_t launchDirect(const FirLaunch &a, cudaStream_t s)
{
   dim3 grid((a.outSize + kDirTile - 1) / kDirTile, a.batch < 65535 ? a.batch : 65535);
   fir_direct_kernel<T, MODE><<<grid, kDirThreads, 0, s>>>(a);
   countLaunch();
   return cudaGetLastError();
}

} // namespace

cudaError_t launchFirBf16x3(const FirLaunch &a, cudaStream_t s);

cudaError_t launchFir(const FirLaunch &a, FirKernelKind kind, cudaStream_t s)
{
   if (a.batch <= 0 || a.outSize <= 0) return cudaSuccess;
   switch (kind) {
   case FIR_NATC:
      switch (a.dtype) {
      case DSPLIB_INT8: return launchDirect<int8_t, MODE_NATC>(a, s);
      case DSPLIB_INT16: return launchDirect<int16_t, MODE_NATC>(a, s);
      case DSPLIB_INT32: return launchDirect<int32_t, MODE_NATC>(a, s);
      case DSPLIB_FLOAT32: return launchDirect<float, MODE_NATC>(a, s);
      default: return cudaErrorInvalidValue;
      }
   case FIR_QMODE:
      switch (a.dtype) {
      case DSPLIB_INT8: return launchDirect<int8_t, MODE_Q>(a, s);
      case DSPLIB_INT16: return launchDirect<int16_t, MODE_Q>(a, s);
      case DSPLIB_INT32: return launchDirect<int32_t, MODE_Q>(a, s);
      default: return cudaErrorInvalidValue;
      }
   case FIR_F32_SIMT: {
      if (a.dtype != DSPLIB_FLOAT32) return cudaErrorInvalidValue;
      dim3 grid((a.outSize + kSimtTile - 1) / kSimtTile, a.batch < 65535 ? a.batch : 65535);
      fir_f32_simt_kernel<<<grid, kSimtThreads, 0, s>>>(a);
      countLaunch();
      return cudaGetLastError();
   }
   case FIR_F32_Q: {
      if (a.dtype != DSPLIB_FLOAT32 || a.shift < 0 || a.shift > kFirMaxFloatQ) return cudaErrorInvalidValue;
      dim3 grid((a.outSize + kDirTile - 1) / kDirTile, a.batch < 65535 ? a.batch : 65535);
      fir_floatq_kernel<<<grid, kDirThreads, 0, s>>>(a);
      countLaunch();
      return cudaGetLastError();
   }
   case FIR_F32_BF16X3:
      if (a.dtype != DSPLIB_FLOAT32) return cudaErrorInvalidValue;
      return launchFirBf16x3(a, s);
   case FIR_INT_WRAP_TC:
   case FIR_INT_Q_TC:
      if (!firIntTcSupported(a)) return cudaErrorInvalidValue;
      return launchFirIntTc(a, kind == FIR_INT_Q_TC, s);
   }
   return cudaErrorInvalidValue;
}

} // namespace dsplib
