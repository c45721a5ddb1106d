// Batched filter bank over channels of uneven length: per channel c
//     u = FIR_valid(x_c, h_c)          (T_c taps, DSPLIB_fir semantics)
//     y = cascade of S_c DF2 biquads (u) from a zero state
// and its adjoint (gradients w.r.t. x, taps and the natural biquad
// coefficients).  Channels are packed densely: x/y/work planes at xOff[c]
// (length L_c; u and y use the first Lu_c = L_c - T_c + 1 entries), taps at
// hOff[c], coefficients [S_c][b0 b1 b2 a1 a2] at cOff[c].
//
// Kernels (every launch covers the whole batch):
//   fir_bf16x3_ragged_kernel (fir_tc.cu)  FIR forward (valid correlation) and
//                          input gradient (full convolution with the same taps)
//                          as split-BF16x3 tcgen05 contractions over runs of
//                          8192-output tiles, one run per CTA.
//   biquad_ragged_kernel   one 512-thread CTA per channel (longest first),
//                          512 chunks of 16 samples per 8192-sample window,
//                          chunked scan with FP64 chunk-boundary states (A^16
//                          and its powers).  Forward: all stages, every stage
//                          output stored (the activations the adjoint needs).
//                          Adjoint: the same cascade run backwards in time with
//                          the stages in reverse order (the adjoint of a
//                          zero-state DF2 section is the section itself on the
//                          time-reversed gradient), accumulating the five
//                          coefficient gradients of every stage in FP64 in a
//                          fixed order (deterministic).
//   fir_dh_partial_kernel / fir_dh_reduce_kernel  taps gradient
//                          dh[T-1-c] = sum_j gu[j] x[j+c], split over tiles
//                          and summed in tile order (deterministic).
//   mse_partial_kernel / mse_reduce_kernel  loss and its gradient.
//
// Adjoint of one DF2 stage y = (B/A) u with zero initial state: with
// v = the anti-causal filtering of gy by 1/A (v[t] = gy[t] - a1 v[t+1] - a2 v[t+2]),
//     gu[t] = b0 v[t] + b1 v[t+1] + b2 v[t+2],
//     dL/db_i = sum_t v[t] u[t-i],   dL/da_i = -sum_t v[t] y[t-i].
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "dsplib_internal.h"
#include "scan_common.cuh"
#include "tc_common.cuh"

namespace dsplib {

struct RaggedPlan {
   int C = 0;
   long long totalLen = 0, totalTaps = 0, totalCoefs = 0, totalOut = 0;
   long long planeStride = 0; // floats per work plane: sum of round16(Lu)
   int Smax = 0, Tmax = 0;
   int nFwdItems = 0, nFirFwdRuns = 0, nFirDxRuns = 0;
   RaggedChan *dChan = nullptr;
   int2 *dFwdItems = nullptr;   // (channel, 2048-sample tile over Lu): adjoint reductions, loss
   int4 *dFirFwdRuns = nullptr; // (channel, first tile, tiles): FIR forward, 8192-output tiles over Lu
   int4 *dFirDxRuns = nullptr;  // the same over L: FIR input gradient
   int *dFwdStart = nullptr;  // first forward item of each channel (C + 1 entries)
   int *dOrder = nullptr;     // channels by descending Lu
   int device = 0;
};

namespace {

using scan::M2;
using scan::M2f;


constexpr int kRTile = 2048; // samples per item of the adjoint reductions and the loss

// ------------------------------------------------------------------ biquad scan per channel

constexpr int kBLogWarps = 4;
constexpr int kBWarps = 1 << kBLogWarps;
constexpr int kBThreads = kBWarps * 32;  // chunks per window
constexpr int kBL = 16;                  // samples per chunk
constexpr int kBWindow = kBThreads * kBL;
constexpr int kBPad = kBL + 1;           // padded shared row per chunk (bank-conflict free)
constexpr int kBPowers = 6 + kBLogWarps; // M^(2^k), M = A^16: lanes (k < 5), warps, and the window (last)
constexpr int kRaggedMaxStages = 64;
// Dynamic shared memory of biquad_ragged_kernel: per-stage carry, powers, coefficients and
// (adjoint) FP64 coefficient-gradient sums; the adjoint adds each thread's u / y chunk.
constexpr size_t kBDynCommon = kRaggedMaxStages * sizeof(float2) + kRaggedMaxStages * kBPowers * sizeof(M2f) +
                               (kRaggedMaxStages * 5 + 4) * sizeof(float) + kRaggedMaxStages * 5 * sizeof(double);
constexpr size_t kBDynPlanes = (size_t) kBThreads * 40 * sizeof(float);

// DF2 over one chunk; WRITE: outputs replace v and, when w0 is given, the
// recursion's internal sequence w0[i] is kept too.
template <bool WRITE>
__device__ __forceinline__ void df2Chunk(float (&v)[kBL], const float *cf, float &w1, float &w2, float *w0s)
{
   const float b0 = cf[0], b1 = cf[1], b2 = cf[2], a1 = cf[3], a2 = cf[4];
#pragma unroll
   for (int i = 0; i < kBL; i++) {
      const float w0 = fmaf(-a1, w1, fmaf(-a2, w2, v[i]));
      if (WRITE) {
         v[i] = fmaf(b0, w0, fmaf(b1, w1, b2 * w2));
         if (w0s) w0s[i] = w0;
      }
      w2 = w1;
      w1 = w0;
   }
}

// Padded shared-memory index of window sample k (one 17-float row per 16-sample chunk).
__device__ __forceinline__ int padIdx(int k) { return (k >> 4) * kBPad + (k & 15); }

// One stage of the chunked scan over a window: v (this thread's 16 samples)
// is filtered from the stage's carried state, the carry is advanced.  P: the
// stage's M^(2^k); tot: a kBWarps-entry shared buffer not in use by the previous stage.
template <bool KEEP_W0>
__device__ __forceinline__ void scanStage(float (&v)[kBL], const float *cf, const M2f *P, float2 *carry,
                                          float2 *tot, float *w0s, int lane, int warp)
{
   const float2 zero = make_float2(0.0f, 0.0f);
   // 1. zero-state end state of this chunk
   float w1 = 0.f, w2 = 0.f;
   df2Chunk<false>(v, cf, w1, w2, nullptr);
   // 2. warp-level inclusive scan over 32 chunks
   float2 val = make_float2(w1, w2);
#pragma unroll
   for (int k = 0; k < 5; k++) {
      const float2 o = scan::shflUp(val, 1 << k, 32);
      if (lane >= (1 << k)) val = scan::affine(P[k], o, val);
   }
   if (lane == 31) tot[warp] = val;
   __syncthreads();
   // 3. warp 0: scan over the warp totals (powers M^(32 * 2^k)), entry states, window carry
   if (warp == 0) {
      float2 tv = lane < kBWarps ? tot[lane] : zero;
#pragma unroll
      for (int k = 0; k < kBLogWarps; k++) {
         const float2 o = scan::shflUp(tv, 1 << k, 32);
         if (lane >= (1 << k) && lane < kBWarps) tv = scan::affine(P[5 + k], o, tv);
      }
      const float2 win = *carry;
      const float2 before = scan::shflUp(tv, 1, 32);
      const float2 last = scan::shflIdx(tv, kBWarps - 1);
      if (lane < kBWarps) {
         // entry of warp `lane`: M^(32*lane) win + inclusive total of warps < lane
         float2 e = win;
#pragma unroll
         for (int k = 0; k < kBLogWarps; k++)
            if ((lane >> k) & 1) e = scan::affine(P[5 + k], e, zero);
         if (lane > 0) e = make_float2(e.x + before.x, e.y + before.y);
         tot[lane] = e;
      }
      if (lane == 0) *carry = scan::affine(P[5 + kBLogWarps], win, last);
   }
   __syncthreads();
   // 4. this chunk's initial state: M^lane * entry(warp) + exclusive warp prefix
   float2 ex = scan::shflUp(val, 1, 32);
   if (lane == 0) ex = zero;
   float2 st = tot[warp];
#pragma unroll
   for (int k = 0; k < 5; k++)
      if ((lane >> k) & 1) st = scan::affine(P[k], st, zero);
   w1 = st.x + ex.x;
   w2 = st.y + ex.y;
   df2Chunk<true>(v, cf, w1, w2, KEEP_W0 ? w0s : nullptr);
}

// One CTA per channel, longest first; windows of 8192 samples in sequence.
// Work planes hold each channel's slice at pOff (a multiple of 16 floats), so a
// thread's 16-sample chunk is one aligned 64-byte run: stage outputs go to and
// come from the planes as 16-byte vectors, without a pass through shared memory.
//
// Forward (BWD = false): the cascade s = 0 .. S-1 over plane 0 (the FIR
// output); stage s's output is stored to plane s+1 (the activations the
// adjoint needs) and the last one to yout.
//
// Adjoint (BWD = true): the adjoint of a zero-state DF2 section is the same
// section run backwards in time (w0 = g - a1 w0[t+1] - a2 w0[t+2], gu = b0 w0 +
// b1 w0[t+1] + b2 w0[t+2]), so the whole cascade adjoint is the cascade over
// the time-reversed output gradient with the stages in reverse order; gu of
// stage 0 goes to gout.  Reversed time runs over the padded length
// LuP = round16(Lu) (tau = LuP-1-t, zero input for t >= Lu), so its chunks are
// the forward chunks.  On the way, with v = that stage's w0 sequence, u its
// forward input (plane s) and y its output (plane s+1):
//     dL/db_i = sum_t v[t] u[t-i],  dL/da_i = -sum_t v[t] y[t-i]
// summed per chunk in FP32, per window and channel in FP64 in a fixed order;
// each thread fetches its chunk of u and y (plus the two samples before it)
// with asynchronous copies issued before the stage's scan.
template <bool BWD>
__global__ void __launch_bounds__(kBThreads, 1)
    biquad_ragged_kernel(const RaggedChan *chans, const int *order, const float *coefs, const float *gin,
                         float *planes, long long planeStride, float *yout, float *gout, float *gcoefs)
{
   __shared__ float sbuf[kBThreads * kBPad];
   __shared__ float2 sTot[2][kBWarps];
   __shared__ float sRed[kBWarps][5];
   extern __shared__ __align__(16) unsigned char dyn[];
   float2 *sWin = (float2 *) dyn;                       // carry per stage
   M2f *sPow = (M2f *) (sWin + kRaggedMaxStages);       // M^(2^k) per stage (formed in FP64)
   float *sCf = (float *) (sPow + kRaggedMaxStages * kBPowers); // coefficients per stage
   double *sAcc = (double *) (sCf + kRaggedMaxStages * 5 + 4);  // BWD: coefficient gradients per stage
   float *sUY = (float *) (sAcc + kRaggedMaxStages * 5);  // BWD: per thread, u and y of its chunk (20 + 20 floats)

   const RaggedChan c = chans[order[blockIdx.x]];
   const int S = c.S;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const int Lu = c.Lu;
   const int LuP = (Lu + 15) & ~15;
   const float *cbase = coefs + c.cOff;
   for (int s = tid; s < S; s += kBThreads) {
      sWin[s] = make_float2(0.0f, 0.0f);
      float cf[5];
#pragma unroll
      for (int k = 0; k < 5; k++) {
         cf[k] = cbase[s * 5 + k];
         sCf[s * 5 + k] = cf[k];
         if (BWD) sAcc[s * 5 + k] = 0.0;
      }
      M2 A = {-(double) cf[3], -(double) cf[4], 1.0, 0.0};
#pragma unroll
      for (int r = 1; r < kBL; r <<= 1) A = scan::mmul(A, A);
      sPow[s * kBPowers] = scan::toF(A);
      for (int k = 1; k < kBPowers; k++) {
         A = scan::mmul(A, A);
         sPow[s * kBPowers + k] = scan::toF(A);
      }
   }
   float *plane0 = planes + c.pOff;
   // The FIR leaves plane 0 past Lu unwritten: zero it (the adjoint reads u there, times zero).
   if (!BWD && tid < LuP - Lu) plane0[Lu + tid] = 0.0f;
   float *uy = sUY + tid * 40; // u[tb-4 .. tb+15] then y[tb-4 .. tb+15]
   __syncthreads();
   int phase = 0;
   for (int win0 = 0; win0 < LuP; win0 += kBWindow) {
      const int c0 = win0 + tid * kBL; // chunk start: forward t, adjoint tau
      const bool inChunk = c0 < LuP;
      const int tb = LuP - kBL - c0;   // adjoint: the chunk's first t (a multiple of 16)
      float v[kBL];
      if (BWD) {
         // output gradient, time-reversed, zero past Lu
         for (int k = tid; k < kBWindow; k += kBThreads) {
            const int t = LuP - 1 - (win0 + k);
            sbuf[padIdx(k)] = (t >= 0 && t < Lu) ? gin[c.xOff + t] : 0.0f;
         }
         __syncthreads();
#pragma unroll
         for (int i = 0; i < kBL; i++) v[i] = sbuf[tid * kBPad + i];
      }
      else if (inChunk) {
#pragma unroll
         for (int i4 = 0; i4 < kBL / 4; i4++) {
            const float4 f = *(const float4 *) (plane0 + c0 + 4 * i4);
            v[4 * i4 + 0] = c0 + 4 * i4 + 0 < Lu ? f.x : 0.0f;
            v[4 * i4 + 1] = c0 + 4 * i4 + 1 < Lu ? f.y : 0.0f;
            v[4 * i4 + 2] = c0 + 4 * i4 + 2 < Lu ? f.z : 0.0f;
            v[4 * i4 + 3] = c0 + 4 * i4 + 3 < Lu ? f.w : 0.0f;
         }
      }
      else {
#pragma unroll
         for (int i = 0; i < kBL; i++) v[i] = 0.0f;
      }
      for (int q = 0; q < S; q++, phase++) {
         const int s = BWD ? S - 1 - q : q;
         if (BWD && inChunk) {
            // u = plane s, y = plane s+1 over [tb-4, tb+16): fetched while the scan runs
            const float *pu = planes + (long long) s * planeStride + c.pOff + tb;
            const float *py = pu + planeStride;
#pragma unroll
            for (int i4 = 0; i4 < 5; i4++) {
               if (i4 > 0 || tb >= 4) {
                  tc::cpAsync16(uy + 4 * i4, pu + 4 * i4 - 4);
                  tc::cpAsync16(uy + 20 + 4 * i4, py + 4 * i4 - 4);
               }
               else {
                  *(float4 *) uy = make_float4(0.f, 0.f, 0.f, 0.f); // before the channel's start
                  *(float4 *) (uy + 20) = make_float4(0.f, 0.f, 0.f, 0.f);
               }
            }
            tc::cpAsyncCommit();
         }
         float w0s[kBL];
         scanStage<BWD>(v, sCf + s * 5, sPow + s * kBPowers, sWin + s, sTot[phase & 1], w0s, lane, warp);
         if (BWD) {
            // chunk element i is t = tb + 15 - i: u[t-j] = uy[19 - i - j], y[t-j] = uy[39 - i - j]
            float p[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
            if (inChunk) {
               tc::cpAsyncWaitAll();
#pragma unroll
               for (int i = 0; i < kBL; i++) {
                  p[0] = fmaf(w0s[i], uy[19 - i], p[0]);
                  p[1] = fmaf(w0s[i], uy[18 - i], p[1]);
                  p[2] = fmaf(w0s[i], uy[17 - i], p[2]);
                  p[3] = fmaf(-w0s[i], uy[38 - i], p[3]);
                  p[4] = fmaf(-w0s[i], uy[37 - i], p[4]);
               }
            }
#pragma unroll
            for (int q5 = 0; q5 < 5; q5++) {
#pragma unroll
               for (int o = 16; o > 0; o >>= 1) p[q5] += __shfl_xor_sync(0xffffffffu, p[q5], o);
            }
            if (lane == 0)
#pragma unroll
               for (int q5 = 0; q5 < 5; q5++) sRed[warp][q5] = p[q5];
            __syncthreads(); // sRed complete
            if (tid < 5) {
               double acc = 0.0;
               for (int w = 0; w < kBWarps; w++) acc += (double) sRed[w][tid];
               sAcc[s * 5 + tid] += acc;
            }
         }
         else if (inChunk) {
            float *pl = planes + (long long) (s + 1) * planeStride + c.pOff + c0;
#pragma unroll
            for (int i4 = 0; i4 < kBL / 4; i4++)
               *(float4 *) (pl + 4 * i4) = make_float4(v[4 * i4], v[4 * i4 + 1], v[4 * i4 + 2], v[4 * i4 + 3]);
         }
      }
      // window result (coalesced through shared memory): forward -> yout; adjoint -> gout, time order restored
      __syncthreads(); // everyone has read sbuf
#pragma unroll
      for (int i = 0; i < kBL; i++) sbuf[tid * kBPad + i] = v[i];
      __syncthreads();
      float *dst = BWD ? gout + c.xOff : yout + c.xOff;
      for (int k = tid; k < kBWindow; k += kBThreads) {
         const int t = BWD ? LuP - 1 - (win0 + k) : win0 + k;
         if (t >= 0 && t < Lu) dst[t] = sbuf[padIdx(k)];
      }
      __syncthreads();
   }
   if (!BWD)
      for (int t = Lu + tid; t < c.L; t += kBThreads) yout[c.xOff + t] = 0.0f;
   if (BWD) {
      __syncthreads();
      for (int k = tid; k < 5 * S; k += kBThreads) gcoefs[c.cOff + k] = (float) sAcc[k];
   }
}

// Taps gradient, partial over one (channel, tile) item:
//     part[item][c] = sum_{j in tile} gu[j] x[j + c],  c < T.
// Thread (cg, sl) accumulates 16 consecutive taps c0 = 16 cg .. c0 + 15 over
// slice sl of the tile with a 24-sample register window: 128 multiply-adds per
// 6 vector loads of x and 2 broadcast loads of gu.  x sits in shared memory
// with 4 padding floats after every 32 (sxIdx), so the 16-byte loads of the
// lanes of a warp, 16 floats apart, fall on distinct banks.  Slices are summed
// in a fixed order.
constexpr int kDhMaxT = 512;
constexpr int kDhTaps = 16; // taps per thread
constexpr int kDhX = kRTile + kDhMaxT + 32; // x samples staged per item
__device__ __forceinline__ int sxIdx(int i) { return i + ((i >> 5) << 2); }

__global__ void __launch_bounds__(256) fir_dh_partial_kernel(const RaggedChan *chans, const int2 *items,
                                                              const float *x, const float *gu, float *part)
{
   __shared__ __align__(16) float sg[kRTile];
   __shared__ __align__(16) float sx[kDhX + kDhX / 8];
   __shared__ float red[256 * kDhTaps];
   const int2 it = items[blockIdx.x];
   const RaggedChan c = chans[it.x];
   const int tid = threadIdx.x;
   const int j0 = it.y * kRTile;
   const int n = min(kRTile, c.Lu - j0);
   for (int k = tid; k < kRTile; k += 256) sg[k] = k < n ? gu[c.xOff + j0 + k] : 0.0f;
   for (int k = tid; k < kDhX; k += 256) {
      const int idx = j0 + k;
      sx[sxIdx(k)] = idx < c.L ? x[c.xOff + idx] : 0.0f;
   }
   __syncthreads();
   const int ncg = (c.T + kDhTaps - 1) / kDhTaps; // <= 32 tap groups
   const int slices = 256 / ncg;                    // threads beyond slices * ncg stay idle
   const int slen = ((kRTile + slices - 1) / slices + 7) & ~7;
   const int cg = tid % ncg, sl = tid / ncg;
   float acc[kDhTaps];
#pragma unroll
   for (int r = 0; r < kDhTaps; r++) acc[r] = 0.0f;
   if (sl < slices) {
      const int c0 = cg * kDhTaps;
      const int jb = sl * slen, je = min(jb + slen, (n + 7) & ~7);
      for (int j = jb; j < je; j += 8) {
         float w[kDhTaps + 8], gv[8];
#pragma unroll
         for (int v = 0; v < (kDhTaps + 8) / 4; v++) *(float4 *) &w[4 * v] = *(const float4 *) &sx[sxIdx(j + c0 + 4 * v)];
         *(float4 *) &gv[0] = *(const float4 *) &sg[j];
         *(float4 *) &gv[4] = *(const float4 *) &sg[j + 4];
#pragma unroll
         for (int i = 0; i < 8; i++)
#pragma unroll
            for (int r = 0; r < kDhTaps; r++) acc[r] = fmaf(gv[i], w[r + i], acc[r]);
      }
   }
   if (sl < slices)
#pragma unroll
      for (int r = 0; r < kDhTaps; r++) red[(sl * ncg + cg) * kDhTaps + r] = acc[r];
   __syncthreads();
   for (int cc = tid; cc < c.T; cc += 256) {
      float sum = 0.0f;
      for (int q = 0; q < slices; q++) sum += red[q * ncg * kDhTaps + cc];
      part[(long long) blockIdx.x * kDhMaxT + cc] = sum;
   }
}

__global__ void __launch_bounds__(256) fir_dh_reduce_kernel(const RaggedChan *chans, const int *start,
                                                             const float *part, float *gtaps)
{
   const RaggedChan c = chans[blockIdx.x];
   for (int cc = threadIdx.x; cc < c.T; cc += 256) {
      double s = 0.0;
      for (int i = start[blockIdx.x]; i < start[blockIdx.x + 1]; i++) s += part[(long long) i * kDhMaxT + cc];
      gtaps[c.hOff + c.T - 1 - cc] = (float) s;
   }
}

// Mean squared error over the valid output samples: gy = scale * (y - target)
// (scale = 2 / n), zero on each channel's T - 1 tail samples; per-item FP64
// partial sums of (y - target)^2, then one block sums them in item order.
__global__ void __launch_bounds__(256) mse_partial_kernel(const RaggedChan *chans, const int2 *items,
                                                           const float *y, const float *target, float *gy,
                                                           double *part, float scale)
{
   const int2 it = items[blockIdx.x];
   const RaggedChan c = chans[it.x];
   const int j0 = it.y * kRTile;
   const int j1 = min(j0 + kRTile, c.Lu);
   double acc = 0.0;
   for (int j = j0 + threadIdx.x; j < j1; j += 256) {
      const float d = y[c.xOff + j] - target[c.xOff + j];
      gy[c.xOff + j] = scale * d;
      acc += (double) d * d;
   }
   if (j1 == c.Lu)
      for (int j = c.Lu + threadIdx.x; j < c.L; j += 256) gy[c.xOff + j] = 0.0f;
   __shared__ double red[256];
   red[threadIdx.x] = acc;
   __syncthreads();
   for (int w = 128; w > 0; w >>= 1) {
      if ((int) threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
   }
   if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(1024) mse_reduce_kernel(const double *part, int n, double invCount, float *loss)
{
   __shared__ double red[1024];
   double s = 0.0;
   for (int i = threadIdx.x; i < n; i += 1024) s += part[i];
   red[threadIdx.x] = s;
   __syncthreads();
   for (int w = 512; w > 0; w >>= 1) {
      if ((int) threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
      __syncthreads();
   }
   if (threadIdx.x == 0) loss[0] = (float) (red[0] * invCount);
}

template <typename T> cudaError_t upload(T **dst, const std::vector<T> &v)
{
   cudaError_t e = cudaMalloc((void **) dst, std::max<size_t>(1, v.size()) * sizeof(T));
   if (e != cudaSuccess) return e;
   if (v.empty()) return cudaSuccess;
   return cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
}

} // namespace

static void freePlan(RaggedPlan *p)
{
   if (!p) return;
   cudaFree(p->dChan);
   cudaFree(p->dFwdItems);
   cudaFree(p->dFirFwdRuns);
   cudaFree(p->dFirDxRuns);
   cudaFree(p->dFwdStart);
   cudaFree(p->dOrder);
   delete p;
}

// Makes the plan's device current for the duration of a call (and restores the
// caller's device afterwards): the plan's tables and the kernels' scratch live there.
class PlanDevice {
 public:
   explicit PlanDevice(const RaggedPlan *p)
   {
      ok_ = cudaGetDevice(&prev_) == cudaSuccess;
      if (ok_ && prev_ != p->device) {
         ok_ = cudaSetDevice(p->device) == cudaSuccess;
         switched_ = ok_;
      }
   }
   ~PlanDevice()
   {
      if (switched_) (void) cudaSetDevice(prev_);
   }
   bool ok() const { return ok_; }

 private:
   int prev_ = 0;
   bool ok_ = false, switched_ = false;
};

int raggedPlanDevice(DSPLIB_gpu_raggedPlan plan)
{
   const RaggedPlan *p = (const RaggedPlan *) plan;
   return p ? p->device : -1;
}

} // namespace dsplib

using namespace dsplib;

extern "C" {

DSPLIB_STATUS DSPLIB_gpu_raggedPlanCreate(DSPLIB_gpu_raggedPlan *plan, int32_t numChannels, const int32_t *length,
                                          const int32_t *taps, const int32_t *stages)
{
   if (!plan || !length || !taps || !stages || numChannels <= 0) return DSPLIB_ERR_NULL_POINTER;
   *plan = nullptr;
   RaggedPlan *p = new RaggedPlan();
   p->C = numChannels;
   std::vector<RaggedChan> ch(numChannels);
   std::vector<int2> fwd;
   std::vector<int4> firFwd, firDx;
   std::vector<int> start(numChannels + 1), order(numChannels);
   // runs of up to kFirBfRunTiles consecutive 8192-output tiles of one channel
   auto addRuns = [](std::vector<int4> &runs, int c, int outLen) {
      const int tiles = (outLen + kFirBfTile - 1) / kFirBfTile;
      for (int t = 0; t < tiles; t += kFirBfRunTiles) runs.push_back(make_int4(c, t, std::min(kFirBfRunTiles, tiles - t), 0));
   };
   long long xo = 0, ho = 0, co = 0, po = 0;
   for (int c = 0; c < numChannels; c++) {
      const int L = length[c], T = taps[c], S = stages[c];
      if (T < 1 || T > kFirBfMaxTaps || L < T || S < 0 || S > kRaggedMaxStages) {
         delete p;
         return DSPLIB_ERR_INVALID_DIMENSION;
      }
      ch[c] = RaggedChan{xo, ho, co, po, L, T, S, L - T + 1};
      po += (L - T + 1 + 15) & ~15;
      xo += L;
      p->totalOut += L - T + 1;
      ho += T;
      co += 5LL * S;
      p->Smax = std::max(p->Smax, S);
      p->Tmax = std::max(p->Tmax, T);
      start[c] = (int) fwd.size();
      for (int t = 0; t * kRTile < L - T + 1; t++) fwd.push_back(make_int2(c, t));
      addRuns(firFwd, c, L - T + 1);
      addRuns(firDx, c, L);
      order[c] = c;
   }
   start[numChannels] = (int) fwd.size();
   // longest runs first, so the short ones fill in behind them
   auto longer = [](const int4 &a, const int4 &b) { return a.z > b.z; };
   std::stable_sort(firFwd.begin(), firFwd.end(), longer);
   std::stable_sort(firDx.begin(), firDx.end(), longer);
   std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ch[a].Lu > ch[b].Lu; });
   p->totalLen = xo;
   p->planeStride = po;
   p->totalTaps = ho;
   p->totalCoefs = co;
   p->nFwdItems = (int) fwd.size();
   p->nFirFwdRuns = (int) firFwd.size();
   p->nFirDxRuns = (int) firDx.size();
   cudaGetDevice(&p->device);
   const bool ok = upload(&p->dChan, ch) == cudaSuccess && upload(&p->dFwdItems, fwd) == cudaSuccess &&
                   upload(&p->dFirFwdRuns, firFwd) == cudaSuccess && upload(&p->dFirDxRuns, firDx) == cudaSuccess &&
                   upload(&p->dFwdStart, start) == cudaSuccess && upload(&p->dOrder, order) == cudaSuccess;
   if (!ok) {
      freePlan(p);
      return DSPLIB_ERR_FAILURE;
   }
   *plan = (DSPLIB_gpu_raggedPlan) p;
   return DSPLIB_SUCCESS;
}

int64_t DSPLIB_gpu_raggedPlanSize(DSPLIB_gpu_raggedPlan plan, int32_t what)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p) return -1;
   switch (what) {
   case DSPLIB_GPU_RAGGED_SAMPLES: return p->totalLen;
   case DSPLIB_GPU_RAGGED_TAPS: return p->totalTaps;
   case DSPLIB_GPU_RAGGED_COEFS: return p->totalCoefs;
   case DSPLIB_GPU_RAGGED_WORK: return (long long) (p->Smax + 1) * p->planeStride;
   case DSPLIB_GPU_RAGGED_SCRATCH: return 2LL * p->totalLen + (long long) p->nFwdItems * kDhMaxT;
   case DSPLIB_GPU_RAGGED_OUTPUTS: return p->totalOut;
   default: return -1;
   }
}

DSPLIB_STATUS DSPLIB_gpu_raggedPlanDestroy(DSPLIB_gpu_raggedPlan plan)
{
   freePlan((RaggedPlan *) plan);
   return DSPLIB_SUCCESS;
}

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_fwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, float *y, float *work, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || (!coefs && p->totalCoefs) || !y || !work) return DSPLIB_ERR_NULL_POINTER;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   if (launchFirBf16x3Ragged(p->dChan, p->dFirFwdRuns, p->nFirFwdRuns, x, taps, work, false, p->Tmax, s) !=
       cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   if (cudaFuncSetAttribute(biquad_ragged_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                            (int) kBDynCommon) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   biquad_ragged_kernel<false><<<p->C, kBThreads, kBDynCommon, s>>>(p->dChan, p->dOrder, coefs, nullptr, work,
                                                                      p->planeStride, y, nullptr, nullptr);
   countLaunch(1);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_bwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, const float *work, const float *gy, float *gx,
                                              float *gtaps, float *gcoefs, float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || ((!coefs || !gcoefs) && p->totalCoefs) || !work || !gy || !gx || !gtaps || !scratch)
      return DSPLIB_ERR_NULL_POINTER;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   float *g = scratch;                      // gradient at the FIR output
   float *part = scratch + 2 * p->totalLen; // per-tile taps-gradient partials
   const size_t dyn = kBDynCommon + kBDynPlanes;
   if (cudaFuncSetAttribute(biquad_ragged_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn) !=
       cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   biquad_ragged_kernel<true><<<p->C, kBThreads, dyn, s>>>(p->dChan, p->dOrder, coefs, gy, (float *) work,
                                                            p->planeStride, nullptr, g, gcoefs);
   if (launchFirBf16x3Ragged(p->dChan, p->dFirDxRuns, p->nFirDxRuns, g, taps, gx, true, p->Tmax, s) != cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   fir_dh_partial_kernel<<<p->nFwdItems, 256, 0, s>>>(p->dChan, p->dFwdItems, x, g, part);
   fir_dh_reduce_kernel<<<p->C, 256, 0, s>>>(p->dChan, p->dFwdStart, part, gtaps);
   countLaunch(3);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

DSPLIB_STATUS DSPLIB_gpu_raggedMseGrad(DSPLIB_gpu_raggedPlan plan, const float *y, const float *target, float *gy,
                                       float *loss, float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !y || !target || !gy || !loss || !scratch) return DSPLIB_ERR_NULL_POINTER;
   if (p->totalOut <= 0) return DSPLIB_ERR_INVALID_DIMENSION;
   PlanDevice dev(p);
   if (!dev.ok()) return DSPLIB_ERR_FAILURE;
   cudaStream_t s = (cudaStream_t) stream;
   double *part = (double *) scratch;
   mse_partial_kernel<<<p->nFwdItems, 256, 0, s>>>(p->dChan, p->dFwdItems, y, target, gy, part,
                                                   (float) (2.0 / (double) p->totalOut));
   mse_reduce_kernel<<<1, 1024, 0, s>>>(part, p->nFwdItems, 1.0 / (double) p->totalOut, loss);
   countLaunch(2);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

} // extern "C"
