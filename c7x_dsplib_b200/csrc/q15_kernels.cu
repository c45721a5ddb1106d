// Q.15 format conversion kernels for sm_100a (DSPLIB_fltoq15, DSPLIB_q15tofl).
//
// Both are pure streams: 6 bytes per element for FLOAT32 <-> Q.15 and 10 for
// FLOAT64 <-> Q.15, so they are bound by memory bandwidth.  Each thread moves
// 16-byte groups of the float side (and the matching 8 / 4 bytes of int16), warp
// instructions cover contiguous spans, loads are marked streaming (read once, not
// kept in L1) and stores evict-first; the grid is one wave over the 148 SMs and
// strides over the array.  When a pointer is not 16-byte aligned the
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

// Vector kernels: one "group" is 16 bytes of the wide (float) side, G = 16 / sizeof(F)
// elements, and 2G bytes of the narrow (int16) side.  Consecutive threads take
// consecutive groups, so every load and store instruction of a warp covers one
// contiguous span (512 bytes wide side, 128 or 256 bytes narrow side): full lines in
// HBM and full-line PCIe transactions on mapped host memory.  kUnroll independent
// groups per thread are loaded before any is converted.
constexpr int kUnroll = 4;

template <typename F> struct Wide;
template <> struct Wide<float> { using T = float4; };
template <> struct Wide<double> { using T = double2; };
template <int G> struct Narrow;
template <> struct Narrow<4> { using T = uint2; };
template <> struct Narrow<2> { using T = unsigned int; };

__device__ __forceinline__ void packQ15(uint2 &w, const int16_t (&q)[4])
{
   w.x = (uint32_t) (uint16_t) q[0] | ((uint32_t) (uint16_t) q[1] << 16);
   w.y = (uint32_t) (uint16_t) q[2] | ((uint32_t) (uint16_t) q[3] << 16);
}
__device__ __forceinline__ void packQ15(unsigned int &w, const int16_t (&q)[2])
{
   w = (uint32_t) (uint16_t) q[0] | ((uint32_t) (uint16_t) q[1] << 16);
}
__device__ __forceinline__ void unpackQ15(const uint2 &w, int16_t (&q)[4])
{
   q[0] = (int16_t) (w.x & 0xffffu), q[1] = (int16_t) (w.x >> 16);
   q[2] = (int16_t) (w.y & 0xffffu), q[3] = (int16_t) (w.y >> 16);
}
__device__ __forceinline__ void unpackQ15(const unsigned int &w, int16_t (&q)[2])
{
   q[0] = (int16_t) (w & 0xffffu), q[1] = (int16_t) (w >> 16);
}

template <bool NATC, typename F>
__global__ void __launch_bounds__(kThreads) fltoq15_vec_kernel(const F *__restrict__ in, int16_t *__restrict__ out,
                                                               long long groups)
{
   constexpr int G = 16 / (int) sizeof(F);
   using W = typename Wide<F>::T;
   using N = typename Narrow<G>::T;
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g0 = (long long) blockIdx.x * kThreads + threadIdx.x; g0 < groups; g0 += stride * kUnroll) {
      W v[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; u++) {
         const long long g = g0 + u * stride;
         if (g < groups) v[u] = __ldcs((const W *) in + g);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; u++) {
         const long long g = g0 + u * stride;
         if (g < groups) {
            const F *e = reinterpret_cast<const F *>(&v[u]);
            int16_t q[G];
#pragma unroll
            for (int k = 0; k < G; k++) q[k] = toQ15<NATC>(e[k]);
            N w;
            packQ15(w, q);
            __stcs((N *) out + g, w);
         }
      }
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

template <typename F>
__global__ void __launch_bounds__(kThreads) q15tofl_vec_kernel(const int16_t *__restrict__ in, F *__restrict__ out,
                                                               long long groups)
{
   constexpr int G = 16 / (int) sizeof(F);
   using W = typename Wide<F>::T;
   using N = typename Narrow<G>::T;
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g0 = (long long) blockIdx.x * kThreads + threadIdx.x; g0 < groups; g0 += stride * kUnroll) {
      N w[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; u++) {
         const long long g = g0 + u * stride;
         if (g < groups) w[u] = __ldcs((const N *) in + g);
      }
#pragma unroll
      for (int u = 0; u < kUnroll; u++) {
         const long long g = g0 + u * stride;
         if (g < groups) {
            int16_t q[G];
            unpackQ15(w[u], q);
            W v;
            F *e = reinterpret_cast<F *>(&v);
#pragma unroll
            for (int k = 0; k < G; k++) e[k] = sizeof(F) == 4 ? (F) fromQ15f(q[k]) : (F) fromQ15d(q[k]);
            __stcs((W *) out + g, v);
         }
      }
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
   constexpr int G = 16 / (int) sizeof(F);
   long long done = 0;
   if (aligned16(in) && aligned16(out)) {
      const long long groups = n / G;
      if (groups > 0) {
         fltoq15_vec_kernel<NATC, F><<<gridFor((groups + kUnroll - 1) / kUnroll), kThreads, 0, s>>>(in, out, groups);
         countLaunch();
      }
      done = groups * G;
   }
   if (done < n) {
      fltoq15_scalar_kernel<NATC, F><<<gridFor(n - done), kThreads, 0, s>>>(in, out, done, n);
      countLaunch();
   }
   return cudaGetLastError();
}

template <typename F> cudaError_t q15toflTyped(const int16_t *in, F *out, long long n, cudaStream_t s)
{
   constexpr int G = 16 / (int) sizeof(F);
   long long done = 0;
   if (aligned16(in) && aligned16(out)) {
      const long long groups = n / G;
      if (groups > 0) {
         q15tofl_vec_kernel<F><<<gridFor((groups + kUnroll - 1) / kUnroll), kThreads, 0, s>>>(in, out, groups);
         countLaunch();
      }
      done = groups * G;
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
