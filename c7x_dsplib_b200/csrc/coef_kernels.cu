// DSPLIB_cascadeBiquad_get_coefficients on device buffers: the transform from the
// natural [ch][stage][b0 b1 b2 a1 a2] coefficients to the optimized layouts, in
// place on the GPU (no copy through host memory).  The arithmetic is the host
// function's, operation for operation and without contraction (IEEE division,
// separately rounded products and sums), so both give the same bits.
//   TIF shared:       out[s*4 + k] = {b1/b0 - a1, b2/b0 - a2, -a2, -a1}, out[4S + g] = gain of group g
//                     (src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_utils.cpp:198-266)
//   TIF per channel:  row k*S + s, column ch; gain rows 4S + g (utils.cpp:268-471)
//   DF* per channel:  row s*5 + k, column ch (utils.cpp:477-650)
#include <cuda_runtime.h>

#include "dsplib_internal.h"

namespace dsplib {
namespace {

constexpr int kTifGroupStages = 7;

__device__ __forceinline__ float recipOrZero(float b0) { return b0 == 0.0f ? 0.0f : __fdiv_rn(1.0f, b0); }

// One thread per (channel, group): the group's stages in order, the gain as a running product.
__global__ void tif_coef_kernel(const float *nat, float *out, int S, int C, int G, int per, long long pitch, int nch)
{
   const int idx = blockIdx.x * blockDim.x + threadIdx.x;
   if (idx >= C * G) return;
   const int ch = idx / G, g = idx % G;
   float gain = 1.0f;
   for (int s = g * per; s < S && s < (g + 1) * per; s++) {
      const float *c = nat + ((long long) ch * S + s) * 5;
      gain = __fmul_rn(c[0], gain);
      const float r = recipOrZero(c[0]);
      const float b1 = __fmul_rn(c[1], r), b2 = __fmul_rn(c[2], r), a1 = -c[3], a2 = -c[4];
      const float v[4] = {__fadd_rn(b1, a1), __fadd_rn(b2, a2), a2, a1};
      for (int k = 0; k < 4; k++) {
         if (nch) out[((long long) k * S + s) * pitch + ch] = v[k];
         else out[s * 4 + k] = v[k];
      }
   }
   if (nch) out[((long long) S * 4 + g) * pitch + ch] = gain;
   else out[(long long) S * 4 + g] = gain;
}

// One thread per (row, channel): coefficient-major reorder.
__global__ void df_coef_kernel(const float *nat, float *out, int rows, int C, long long pitch)
{
   const long long idx = (long long) blockIdx.x * blockDim.x + threadIdx.x;
   if (idx >= (long long) rows * C) return;
   const int r = (int) (idx / C), ch = (int) (idx % C);
   out[r * pitch + ch] = nat[(long long) ch * rows + r];
}

} // namespace

cudaError_t launchBiquadCoefTransform(int tif, int nch, const float *nat, float *opt, int S, int C, long long pitch,
                                      cudaStream_t s)
{
   if (S <= 0 || C <= 0) return cudaSuccess;
   if (tif) {
      const int G = S <= kTifGroupStages ? 1 : (S + kTifGroupStages - 1) / kTifGroupStages;
      const int per = S <= kTifGroupStages ? S : kTifGroupStages;
      const int n = C * G;
      tif_coef_kernel<<<(n + 127) / 128, 128, 0, s>>>(nat, opt, S, C, G, per, pitch, nch);
   }
   else {
      const long long n = (long long) S * 5 * C;
      df_coef_kernel<<<(unsigned) ((n + 255) / 256), 256, 0, s>>>(nat, opt, S * 5, C, pitch);
   }
   countLaunch();
   return cudaGetLastError();
}

} // namespace dsplib
