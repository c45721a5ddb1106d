// 2x2 affine-map helpers shared by the chunked parallel-in-time biquad scans.
#pragma once

#include <cuda_runtime.h>

namespace dsplib {
namespace scan {

// [[a, b], [c, d]]
struct M2 {
   double a, b, c, d;
};

__device__ __forceinline__ M2 mmul(const M2 &x, const M2 &y)
{
   return {fma(x.a, y.a, x.b * y.c), fma(x.a, y.b, x.b * y.d), fma(x.c, y.a, x.d * y.c), fma(x.c, y.b, x.d * y.d)};
}

// m * v + e
__device__ __forceinline__ double2 affine(const M2 &m, double2 v, double2 e)
{
   return make_double2(fma(m.a, v.x, fma(m.b, v.y, e.x)), fma(m.c, v.x, fma(m.d, v.y, e.y)));
}

__device__ __forceinline__ double2 shflUp(double2 v, int d, int width)
{
   v.x = __shfl_up_sync(0xffffffffu, v.x, d, width);
   v.y = __shfl_up_sync(0xffffffffu, v.y, d, width);
   return v;
}

__device__ __forceinline__ double2 shflIdx(double2 v, int src)
{
   v.x = __shfl_sync(0xffffffffu, v.x, src);
   v.y = __shfl_sync(0xffffffffu, v.y, src);
   return v;
}

// FP32 forms: matrices formed in FP64 (mmul) and rounded once, scans in FP32 (the
// chunk transitions of stable sections contract, so the scan's rounding stays at the
// level of the FP32 recursion while its dependent chains are several times shorter).
struct M2f {
   float a, b, c, d;
};

__device__ __forceinline__ M2f toF(const M2 &m) { return {(float) m.a, (float) m.b, (float) m.c, (float) m.d}; }

__device__ __forceinline__ float2 affine(const M2f &m, float2 v, float2 e)
{
   return make_float2(fmaf(m.a, v.x, fmaf(m.b, v.y, e.x)), fmaf(m.c, v.x, fmaf(m.d, v.y, e.y)));
}

__device__ __forceinline__ float2 shflUp(float2 v, int d, int width)
{
   v.x = __shfl_up_sync(0xffffffffu, v.x, d, width);
   v.y = __shfl_up_sync(0xffffffffu, v.y, d, width);
   return v;
}

__device__ __forceinline__ float2 shflIdx(float2 v, int src)
{
   v.x = __shfl_sync(0xffffffffu, v.x, src);
   v.y = __shfl_sync(0xffffffffu, v.y, src);
   return v;
}

} // namespace scan
} // namespace dsplib
