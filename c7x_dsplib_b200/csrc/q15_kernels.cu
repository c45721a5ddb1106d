// Q.15 format conversion kernels for sm_100a (DSPLIB_fltoq15, DSPLIB_q15tofl).
//
// Both are pure streams: 6 bytes per element for FLOAT32 <-> Q.15 and 10 for
// FLOAT64 <-> Q.15, so they are bound by memory bandwidth.  Each thread moves
// eight elements per iteration with 16-byte vector accesses (the int16 side is
// one 16-byte word), loads marked streaming (read once, not kept in L1) and
// stores marked evict-first; the grid is a whole number of waves over the 148
// SMs and strides over the array.  When a pointer is not 16-byte aligned the
// scalar kernel runs instead (same arithmetic, coalesced 4/8-byte loads).
//
// The same kernels also run on mapped pinned host memory (the API's zero-copy
// path for page-locked host buffers): every byte is touched exactly once, so
// reading it across PCIe inside the kernel costs no more than a copy engine
// would, and reads and writes overlap.
#include <cuda_runtime.h>

#include <cstdint>

#include "dsplib_internal.h"

namespace dsplib {

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 8;

__device__ __forceinline__ int16_t sat16(int v) { return (int16_t) min(max(v, -32768), 32767); }

// DSPLIB_fltoq15_cn.cpp:36-60 step by step, every float operation rounded
// separately (no contraction).  The conversions truncate toward zero and, where
// the C cast would be undefined (|m| >= 2^31, NaN), saturate by sign / give 0.
__device__ __forceinline__ int16_t q15Natc(float a)
{
   const float m = __fmul_rn(a, 32768.0f);
   const int ip = __float2int_rz(m);
   const float fp = __fsub_rn(m, __int2float_rn(ip));
   int r;
   if ((ip % 2 == 0) && fabsf(fp) == 0.5f) r = ip;
   else if (a < 0.0f) r = __float2int_rz(__fsub_rn(m, 0.5f));
   else r = __float2int_rz(__fadd_rn(m, 0.5f));
   return sat16(r);
}

__device__ __forceinline__ int16_t q15Natc(double a)
{
   const double m = __dmul_rn(a, 32768.0);
   const int ip = __double2int_rz(m);
   const double fp = __dsub_rn(m, (double) ip);
   int r;
   if ((ip % 2 == 0) && fabs(fp) == 0.5) r = ip;
   else if (a < 0.0) r = __double2int_rz(__dsub_rn(m, 0.5));
   else r = __double2int_rz(__dadd_rn(m, 0.5));
   return sat16(r);
}

// One round-to-nearest-even conversion, saturated: the C7x kernel's
// __float_to_int / __double_to_int followed by __int_to_short_sat.
__device__ __forceinline__ int16_t q15Rne(float a) { return sat16(__float2int_rn(__fmul_rn(a, 32768.0f))); }
__device__ __forceinline__ int16_t q15Rne(double a) { return sat16(__double2int_rn(__dmul_rn(a, 32768.0))); }

// NaN converts to 0 (cvt gives 0 for f32 sources but 0x80000000 for f64 ones,
// so it is tested explicitly).
template <bool NATC, typename F> __device__ __forceinline__ int16_t toQ15(F a)
{
   if (a != a) return 0;
   return NATC ? q15Natc(a) : q15Rne(a);
}

// x / 32768 is exact in both float types (a power-of-two scaling of an integer
// of at most 16 bits), so the multiply by 2^-15 equals the reference quotient.
__device__ __forceinline__ float fromQ15f(int16_t v) { return __fmul_rn((float) v, 3.0517578125e-05f); }
__device__ __forceinline__ double fromQ15d(int16_t v) { return __dmul_rn((double) v, 3.0517578125e-05); }

__device__ __forceinline__ void load8(const float *p, float (&v)[8])
{
   const float4 a = __ldcs((const float4 *) p), b = __ldcs((const float4 *) p + 1);
   v[0] = a.x, v[1] = a.y, v[2] = a.z, v[3] = a.w, v[4] = b.x, v[5] = b.y, v[6] = b.z, v[7] = b.w;
}

__device__ __forceinline__ void load8(const double *p, double (&v)[8])
{
#pragma unroll
   for (int k = 0; k < 4; k++) {
      const double2 a = __ldcs((const double2 *) p + k);
      v[2 * k] = a.x;
      v[2 * k + 1] = a.y;
   }
}

template <bool NATC, typename F>
__global__ void __launch_bounds__(kThreads) fltoq15_vec_kernel(const F *__restrict__ in, int16_t *__restrict__ out,
                                                               long long groups)
{
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g = (long long) blockIdx.x * kThreads + threadIdx.x; g < groups; g += stride) {
      F v[8];
      load8(in + g * kPerThread, v);
      uint32_t w[4];
#pragma unroll
      for (int k = 0; k < 4; k++)
         w[k] = (uint32_t) (uint16_t) toQ15<NATC>(v[2 * k]) | ((uint32_t) (uint16_t) toQ15<NATC>(v[2 * k + 1]) << 16);
      __stcs((int4 *) (out + g * kPerThread), make_int4((int) w[0], (int) w[1], (int) w[2], (int) w[3]));
   }
}

template <bool NATC, typename F>
__global__ void __launch_bounds__(kThreads) fltoq15_scalar_kernel(const F *__restrict__ in, int16_t *__restrict__ out,
                                                                  long long first, long long n)
{
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long i = first + (long long) blockIdx.x * kThreads + threadIdx.x; i < n; i += stride)
      out[i] = toQ15<NATC>(__ldcs(in + i));
}

__global__ void __launch_bounds__(kThreads) q15tofl_vec_kernel(const int16_t *__restrict__ in, float *__restrict__ out,
                                                               long long groups)
{
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g = (long long) blockIdx.x * kThreads + threadIdx.x; g < groups; g += stride) {
      const int4 w = __ldcs((const int4 *) (in + g * kPerThread));
      const uint32_t u[4] = {(uint32_t) w.x, (uint32_t) w.y, (uint32_t) w.z, (uint32_t) w.w};
      float v[8];
#pragma unroll
      for (int k = 0; k < 4; k++) {
         v[2 * k] = fromQ15f((int16_t) (u[k] & 0xffffu));
         v[2 * k + 1] = fromQ15f((int16_t) (u[k] >> 16));
      }
      float4 *o = (float4 *) (out + g * kPerThread);
      __stcs(o, make_float4(v[0], v[1], v[2], v[3]));
      __stcs(o + 1, make_float4(v[4], v[5], v[6], v[7]));
   }
}

__global__ void __launch_bounds__(kThreads) q15tofl_vec_kernel(const int16_t *__restrict__ in,
                                                               double *__restrict__ out, long long groups)
{
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g = (long long) blockIdx.x * kThreads + threadIdx.x; g < groups; g += stride) {
      const int4 w = __ldcs((const int4 *) (in + g * kPerThread));
      const uint32_t u[4] = {(uint32_t) w.x, (uint32_t) w.y, (uint32_t) w.z, (uint32_t) w.w};
      double2 *o = (double2 *) (out + g * kPerThread);
#pragma unroll
      for (int k = 0; k < 4; k++)
         __stcs(o + k, make_double2(fromQ15d((int16_t) (u[k] & 0xffffu)), fromQ15d((int16_t) (u[k] >> 16))));
   }
}

template <typename F>
__global__ void __launch_bounds__(kThreads) q15tofl_scalar_kernel(const int16_t *__restrict__ in, F *__restrict__ out,
                                                                  long long first, long long n)
{
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long i = first + (long long) blockIdx.x * kThreads + threadIdx.x; i < n; i += stride) {
      const int16_t v = __ldcs(in + i);
      if (sizeof(F) == 4) out[i] = (F) fromQ15f(v);
      else out[i] = (F) fromQ15d(v);
   }
}

// Blocks for `work` threads' worth of items: at most 8 resident 256-thread CTAs
// on each of the device's SMs (one full wave), fewer for small arrays.
int gridFor(long long work)
{
   static int sms = 0;
   if (sms == 0) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                      cudaSuccess || sms <= 0)
         sms = 148;
   }
   const long long want = (work + kThreads - 1) / kThreads;
   const long long cap = (long long) sms * 8;
   return (int) (want < 1 ? 1 : (want > cap ? cap : want));
}

bool aligned16(const void *p) { return ((uintptr_t) p & 15u) == 0; }

template <bool NATC, typename F> cudaError_t fltoq15Typed(const F *in, int16_t *out, long long n, cudaStream_t s)
{
   long long done = 0;
   if (aligned16(in) && aligned16(out)) {
      const long long groups = n / kPerThread;
      if (groups > 0) {
         fltoq15_vec_kernel<NATC, F><<<gridFor(groups), kThreads, 0, s>>>(in, out, groups);
         countLaunch();
      }
      done = groups * kPerThread;
   }
   if (done < n) {
      fltoq15_scalar_kernel<NATC, F><<<gridFor(n - done), kThreads, 0, s>>>(in, out, done, n);
      countLaunch();
   }
   return cudaGetLastError();
}

template <typename F> cudaError_t q15toflTyped(const int16_t *in, F *out, long long n, cudaStream_t s)
{
   long long done = 0;
   if (aligned16(in) && aligned16(out)) {
      const long long groups = n / kPerThread;
      if (groups > 0) {
         q15tofl_vec_kernel<<<gridFor(groups), kThreads, 0, s>>>(in, out, groups);
         countLaunch();
      }
      done = groups * kPerThread;
   }
   if (done < n) {
      q15tofl_scalar_kernel<F><<<gridFor(n - done), kThreads, 0, s>>>(in, out, done, n);
      countLaunch();
   }
   return cudaGetLastError();
}

} // namespace

cudaError_t launchFltoq15(const void *in, int16_t *out, long long n, bool isDouble, bool natc, cudaStream_t s)
{
   if (n <= 0) return cudaSuccess;
   if (isDouble)
      return natc ? fltoq15Typed<true>((const double *) in, out, n, s) : fltoq15Typed<false>((const double *) in, out, n, s);
   return natc ? fltoq15Typed<true>((const float *) in, out, n, s) : fltoq15Typed<false>((const float *) in, out, n, s);
}

cudaError_t launchQ15tofl(const int16_t *in, void *out, long long n, bool isDouble, cudaStream_t s)
{
   if (n <= 0) return cudaSuccess;
   return isDouble ? q15toflTyped(in, (double *) out, n, s) : q15toflTyped(in, (float *) out, n, s);
}

} // namespace dsplib
