// Batched filter bank over channels of uneven length: per channel c
//     u = FIR_valid(x_c, h_c)          (T_c taps, DSPLIB_fir semantics)
//     y = cascade of S_c DF2 biquads (u) from a zero state
// and its adjoint (gradients w.r.t. x, taps and the natural biquad
// coefficients).  Channels are packed densely: x/y/work planes at xOff[c]
// (length L_c; u and y use the first Lu_c = L_c - T_c + 1 entries), taps at
// hOff[c], coefficients [S_c][b0 b1 b2 a1 a2] at cOff[c].
//
// Kernels (every launch covers the whole batch):
//   fir_ragged_kernel      work list of (channel, 2048-output tile) items,
//                          FP32 CUDA-core FIR; forward (valid correlation) or
//                          dx (full convolution with the same taps).
//   biquad_ragged_kernel   one CTA per channel (longest first), 512 chunks of
//                          16 samples per 8192-sample window, chunked scan with
//                          FP64 chunk-boundary states (A^16 and its powers);
//                          forward runs all stages and stores every stage
//                          output (the activations the adjoint needs); the
//                          adjoint mode runs one stage's autoregressive part
//                          backwards in time.
//   biquad_ragged_bwd_kernel  per channel and stage: input gradient
//                          gu[t] = b0 v[t] + b1 v[t+1] + b2 v[t+2] and the five
//                          coefficient gradients (FP64 block reductions, fixed
//                          order, deterministic).
//   fir_dh_partial_kernel / fir_dh_reduce_kernel  taps gradient
//                          dh[T-1-c] = sum_j gu[j] x[j+c], split over tiles
//                          and summed in tile order (deterministic).
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

namespace dsplib {

struct RaggedChan {
   long long xOff, hOff, cOff;
   int L, T, S, Lu;
};

struct RaggedPlan {
   int C = 0;
   long long totalLen = 0, totalTaps = 0, totalCoefs = 0, totalOut = 0;
   int Smax = 0, Tmax = 0;
   int nFwdItems = 0, nDxItems = 0;
   RaggedChan *dChan = nullptr;
   int2 *dFwdItems = nullptr; // (channel, tile over Lu)
   int2 *dDxItems = nullptr;  // (channel, tile over L)
   int *dFwdStart = nullptr;  // first forward item of each channel (C + 1 entries)
   int *dOrder = nullptr;     // channels by descending Lu
   int device = 0;
};

namespace {

using scan::M2;


constexpr int kRTile = 2048;
constexpr int kRThreads = 256;
constexpr int kRTaps = 256;

// out[j] = sum_{c<T} in[j + c + shift] * w(c), in[] zero outside [0, inLen);
// forward: shift 0, w(c) = h[T-1-c]; dx: shift -(T-1), w(c) = h[c].
template <bool DX>
__global__ void __launch_bounds__(kRThreads) fir_ragged_kernel(const RaggedChan *chans, const int2 *items,
                                                                const float *in, const float *taps, float *out)
{
   __shared__ __align__(16) float xs[kRTile + kRTaps + 8];
   __shared__ __align__(16) float gs[kRTaps];
   const int2 it = items[blockIdx.x];
   const RaggedChan c = chans[it.x];
   const int T = c.T;
   const int inLen = DX ? c.Lu : c.L;
   const int outLen = DX ? c.L : c.Lu;
   const int shift = DX ? -(T - 1) : 0;
   const float *x = in + c.xOff;
   const float *h = taps + c.hOff;
   float *y = out + c.xOff;
   const int j0 = it.y * kRTile;
   float acc[8];
#pragma unroll
   for (int r = 0; r < 8; r++) acc[r] = 0.0f;
   for (int cb = 0; cb < T; cb += kRTaps) {
      const int tb = min(kRTaps, T - cb);
      const int tbr = (tb + 7) & ~7;
      for (int k = threadIdx.x; k < kRTile + tbr + 8; k += kRThreads) {
         const long long idx = (long long) j0 + cb + k + shift;
         xs[k] = (idx >= 0 && idx < inLen) ? x[idx] : 0.0f;
      }
      for (int k = threadIdx.x; k < tbr; k += kRThreads)
         gs[k] = k < tb ? (DX ? h[cb + k] : h[T - 1 - (cb + k)]) : 0.0f;
      __syncthreads();
      const float *xw = xs + 8 * threadIdx.x;
      for (int cc = 0; cc < tbr; cc += 8) {
         float w[16], g[8];
         *(float4 *) &w[0] = *(const float4 *) &xw[cc];
         *(float4 *) &w[4] = *(const float4 *) &xw[cc + 4];
         *(float4 *) &w[8] = *(const float4 *) &xw[cc + 8];
         *(float4 *) &w[12] = *(const float4 *) &xw[cc + 12];
         *(float4 *) &g[0] = *(const float4 *) &gs[cc];
         *(float4 *) &g[4] = *(const float4 *) &gs[cc + 4];
#pragma unroll
         for (int i = 0; i < 8; i++)
#pragma unroll
            for (int r = 0; r < 8; r++) acc[r] = fmaf(w[r + i], g[i], acc[r]);
      }
      __syncthreads();
   }
#pragma unroll
   for (int r = 0; r < 8; r++) xs[8 * threadIdx.x + r] = acc[r];
   __syncthreads();
   for (int k = threadIdx.x; k < kRTile; k += kRThreads)
      if (j0 + k < outLen) y[j0 + k] = xs[k];
}

// ------------------------------------------------------------------ biquad scan per channel

constexpr int kBWarps = 16;
constexpr int kBThreads = kBWarps * 32; // chunks per window
constexpr int kBL = 16;                 // samples per chunk
constexpr int kBWindow = kBThreads * kBL;
constexpr int kBPad = kBL + 1;          // padded shared row per chunk (bank-conflict free)
constexpr int kBPowers = 10;            // M^(2^k), M = A^16, k = 0..9 (M^512 spans a window)
constexpr int kRaggedMaxStages = 64;

__device__ __forceinline__ void df2Chunk(float (&v)[kBL], const float *cf, float &w1, float &w2, bool write)
{
   const float b0 = cf[0], b1 = cf[1], b2 = cf[2], a1 = cf[3], a2 = cf[4];
#pragma unroll
   for (int i = 0; i < kBL; i++) {
      const float w0 = fmaf(-a1, w1, fmaf(-a2, w2, v[i]));
      if (write) v[i] = fmaf(b0, w0, fmaf(b1, w1, b2 * w2));
      w2 = w1;
      w1 = w0;
   }
}

// One CTA per channel.  Forward (BWD = false): the cascade over plane 0 (u),
// stage s output to plane s+1 and the last stage also to yout.  Adjoint
// (BWD = true): the autoregressive part of stage `stage` over gin, backwards
// in time, into vout.  Samples past the channel's length read as zero.
template <bool BWD>
__global__ void __launch_bounds__(kBThreads, 1)
    biquad_ragged_kernel(const RaggedChan *chans, const int *order, const float *coefs, const float *gin,
                         float *planes, long long planeStride, float *yout, int stage, float *vout)
{
   __shared__ float sbuf[kBThreads * kBPad];
   __shared__ double2 sTot[kBWarps];
   extern __shared__ __align__(16) unsigned char dyn[];
   double2 *sWin = (double2 *) dyn;                      // carry per stage
   M2 *sPow = (M2 *) (dyn + kRaggedMaxStages * sizeof(double2)); // M^(2^k) per stage

   const RaggedChan c = chans[order[blockIdx.x]];
   const int nst = BWD ? 1 : c.S;
   if (BWD && c.S <= stage) return; // uniform per CTA
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const int Lu = c.Lu;
   const float *cbase = coefs + c.cOff;
   // Per stage: zero carry and the powers M^(2^k), M = A^16, of its transition matrix.
   for (int s = tid; s < nst; s += kBThreads) {
      const int si = BWD ? stage : s;
      sWin[s] = make_double2(0.0, 0.0);
      M2 A = {-(double) cbase[si * 5 + 3], -(double) cbase[si * 5 + 4], 1.0, 0.0};
#pragma unroll
      for (int r = 1; r < kBL; r <<= 1) A = scan::mmul(A, A);
      sPow[s * kBPowers] = A;
      for (int k = 1; k < kBPowers; k++) {
         A = scan::mmul(A, A);
         sPow[s * kBPowers + k] = A;
      }
   }
   const float *src = BWD ? gin + c.xOff : planes + c.xOff;
   __syncthreads();
   for (int win0 = 0; win0 < Lu; win0 += kBWindow) {
      // Stage the window through shared memory (coalesced), reversed in time for the adjoint.
      for (int k = tid; k < kBWindow; k += kBThreads) {
         const int tau = win0 + k;
         float val = 0.0f;
         if (tau < Lu) val = src[BWD ? (Lu - 1 - tau) : tau];
         sbuf[(k / kBL) * kBPad + (k % kBL)] = val;
      }
      __syncthreads();
      float v[kBL];
#pragma unroll
      for (int i = 0; i < kBL; i++) v[i] = sbuf[tid * kBPad + i];
      for (int s = 0; s < nst; s++) {
         const int si = BWD ? stage : s;
         float cf[5];
         if (BWD) {
            cf[0] = 1.0f;
            cf[1] = 0.0f;
            cf[2] = 0.0f;
            cf[3] = cbase[si * 5 + 3];
            cf[4] = cbase[si * 5 + 4];
         }
         else {
#pragma unroll
            for (int k = 0; k < 5; k++) cf[k] = cbase[si * 5 + k];
         }
         const M2 *P = sPow + s * kBPowers;
         // 1. zero-state end state of this chunk
         float w1 = 0.f, w2 = 0.f;
         df2Chunk(v, cf, w1, w2, false);
         // 2. warp-level inclusive scan over 32 chunks
         double2 val = make_double2(w1, w2);
#pragma unroll
         for (int k = 0; k < 5; k++) {
            const double2 o = scan::shflUp(val, 1 << k, 32);
            if (lane >= (1 << k)) val = scan::affine(P[k], o, val);
         }
         if (lane == 31) sTot[warp] = val;
         __syncthreads();
         // 3. warp 0: scan over the 16 warp totals (powers M^(32 * 2^k)), entry states, window carry
         if (warp == 0) {
            double2 tv = lane < kBWarps ? sTot[lane] : make_double2(0.0, 0.0);
#pragma unroll
            for (int k = 0; k < 4; k++) {
               const double2 o = scan::shflUp(tv, 1 << k, 32);
               if (lane >= (1 << k) && lane < kBWarps) tv = scan::affine(P[5 + k], o, tv);
            }
            const double2 win = sWin[s];
            const double2 before = scan::shflUp(tv, 1, 32);
            const double2 last = scan::shflIdx(tv, kBWarps - 1);
            if (lane < kBWarps) {
               // entry of warp `lane`: M^(32*lane) win + inclusive total of warps < lane
               double2 e = win;
#pragma unroll
               for (int k = 0; k < 4; k++)
                  if ((lane >> k) & 1) e = scan::affine(P[5 + k], e, make_double2(0.0, 0.0));
               if (lane > 0) e = make_double2(e.x + before.x, e.y + before.y);
               sTot[lane] = e;
            }
            if (lane == 0) sWin[s] = scan::affine(P[9], win, last);
         }
         __syncthreads();
         // 4. this chunk's initial state: M^lane * entry(warp) + exclusive warp prefix
         double2 ex = scan::shflUp(val, 1, 32);
         if (lane == 0) ex = make_double2(0.0, 0.0);
         double2 st = sTot[warp];
#pragma unroll
         for (int k = 0; k < 5; k++)
            if ((lane >> k) & 1) st = scan::affine(P[k], st, make_double2(0.0, 0.0));
         w1 = (float) (st.x + ex.x);
         w2 = (float) (st.y + ex.y);
         df2Chunk(v, cf, w1, w2, true);
         // 5. store this stage's output for the window (coalesced through shared memory)
         __syncthreads(); // everyone has read sTot / sbuf
#pragma unroll
         for (int i = 0; i < kBL; i++) sbuf[tid * kBPad + i] = v[i];
         __syncthreads();
         float *dst = BWD ? vout + c.xOff : planes + (long long) (s + 1) * planeStride + c.xOff;
         for (int k = tid; k < kBWindow; k += kBThreads) {
            const int tau = win0 + k;
            if (tau < Lu) {
               const float o = sbuf[(k / kBL) * kBPad + (k % kBL)];
               dst[BWD ? (Lu - 1 - tau) : tau] = o;
               if (!BWD && s == nst - 1) yout[c.xOff + tau] = o;
            }
         }
      }
      __syncthreads();
   }
   if (!BWD) {
      // No stages: the output is the FIR output itself.
      if (nst == 0)
         for (int t = tid; t < Lu; t += kBThreads) yout[c.xOff + t] = planes[c.xOff + t];
      for (int t = Lu + tid; t < c.L; t += kBThreads) yout[c.xOff + t] = 0.0f;
   }
}

// Input gradient (in place over g) of one stage and per-item partial sums of
// its five coefficient gradients (FP64, one row of 5 per item).  Item
// (channel, tile) covers t in [j0, j0 + 2048) of the channel; the stage's v, u
// and y around the tile are staged in shared memory.
__global__ void __launch_bounds__(256) biquad_ragged_bwd_kernel(const RaggedChan *chans, const int2 *items,
                                                                 const float *coefs, const float *planes,
                                                                 long long planeStride, const float *v,
                                                                 float *g, double *part, int stage)
{
   __shared__ float sv[kRTile + 2], su[kRTile + 2], sy[kRTile + 2];
   __shared__ double red[5][256];
   const int2 it = items[blockIdx.x];
   const RaggedChan c = chans[it.x];
   if (c.S <= stage) return; // uniform per CTA
   const int tid = threadIdx.x;
   const int j0 = it.y * kRTile;
   const int n = min(kRTile, c.Lu - j0);
   const float *u = planes + (long long) stage * planeStride + c.xOff;
   const float *y = planes + (long long) (stage + 1) * planeStride + c.xOff;
   const float *vv = v + c.xOff;
   // sv[k] = v[j0 + k] (zero past the channel); su[k] = u[j0 - 2 + k], sy[k] = y[j0 - 2 + k] (zero before 0)
   for (int k = tid; k < kRTile + 2; k += 256) {
      const int tv = j0 + k, tu = j0 - 2 + k;
      sv[k] = tv < c.Lu ? vv[tv] : 0.0f;
      const bool inU = tu >= 0 && tu < j0 + n;
      su[k] = inU ? u[tu] : 0.0f;
      sy[k] = inU ? y[tu] : 0.0f;
   }
   __syncthreads();
   const float *cf = coefs + c.cOff + stage * 5;
   const float b0 = cf[0], b1 = cf[1], b2 = cf[2];
   float acc[5] = {0.f, 0.f, 0.f, 0.f, 0.f};
   float *gg = g + c.xOff + j0;
#pragma unroll
   for (int i = 0; i < kRTile / 256; i++) {
      const int k = i * 256 + tid;
      if (k < n) {
         const float vt = sv[k];
         gg[k] = fmaf(b0, vt, fmaf(b1, sv[k + 1], b2 * sv[k + 2]));
         acc[0] = fmaf(vt, su[k + 2], acc[0]);
         acc[1] = fmaf(vt, su[k + 1], acc[1]);
         acc[2] = fmaf(vt, su[k], acc[2]);
         acc[3] = fmaf(-vt, sy[k + 1], acc[3]);
         acc[4] = fmaf(-vt, sy[k], acc[4]);
      }
   }
#pragma unroll
   for (int q = 0; q < 5; q++) red[q][tid] = acc[q];
   __syncthreads();
   for (int w = 128; w > 0; w >>= 1) {
      if (tid < w)
#pragma unroll
         for (int q = 0; q < 5; q++) red[q][tid] += red[q][tid + w];
      __syncthreads();
   }
   if (tid < 5) part[(long long) blockIdx.x * 5 + tid] = red[tid][0];
}

// Coefficient gradients of one stage: the item partials of each channel summed in item order.
__global__ void __launch_bounds__(32) biquad_coef_reduce_kernel(const RaggedChan *chans, const int *start,
                                                                 const double *part, float *gcoefs, int stage)
{
   const RaggedChan c = chans[blockIdx.x];
   if (c.S <= stage || threadIdx.x >= 5) return;
   double s = 0.0;
   for (int i = start[blockIdx.x]; i < start[blockIdx.x + 1]; i++) s += part[(long long) i * 5 + threadIdx.x];
   gcoefs[c.cOff + stage * 5 + threadIdx.x] = (float) s;
}

// Taps gradient, partial over one (channel, tile) item:
//     part[item][c] = sum_{j in tile} gu[j] x[j + c],  c < T.
// Thread (cg, sl) accumulates 8 consecutive taps c0 = 8 cg .. c0 + 7 over slice sl
// of the tile with a 16-sample register window (64 multiply-adds per 6 vector
// shared-memory loads); slices are then summed in a fixed order.
constexpr int kDhMaxT = 512;
__global__ void __launch_bounds__(256) fir_dh_partial_kernel(const RaggedChan *chans, const int2 *items,
                                                              const float *x, const float *gu, float *part)
{
   __shared__ __align__(16) float sg[kRTile];
   __shared__ __align__(16) float sx[kRTile + kDhMaxT + 16];
   __shared__ float red[256 * 8];
   const int2 it = items[blockIdx.x];
   const RaggedChan c = chans[it.x];
   const int tid = threadIdx.x;
   const int j0 = it.y * kRTile;
   const int n = min(kRTile, c.Lu - j0);
   for (int k = tid; k < kRTile; k += 256) sg[k] = k < n ? gu[c.xOff + j0 + k] : 0.0f;
   for (int k = tid; k < kRTile + kDhMaxT + 16; k += 256) {
      const int idx = j0 + k;
      sx[k] = idx < c.L ? x[c.xOff + idx] : 0.0f;
   }
   __syncthreads();
   const int ncg = (c.T + 7) >> 3;
   int ncp = 1;
   while (ncp < ncg) ncp <<= 1; // <= 64
   const int slices = 256 / ncp, slen = kRTile / slices;
   const int cg = tid & (ncp - 1), sl = tid / ncp;
   float acc[8];
#pragma unroll
   for (int r = 0; r < 8; r++) acc[r] = 0.0f;
   if (cg < ncg) {
      const int c0 = cg * 8;
      const int jb = sl * slen, je = min(jb + slen, (n + 7) & ~7);
      for (int j = jb; j < je; j += 8) {
         float w[16], gv[8];
         const float *xw = sx + j + c0;
         *(float4 *) &w[0] = *(const float4 *) &xw[0];
         *(float4 *) &w[4] = *(const float4 *) &xw[4];
         *(float4 *) &w[8] = *(const float4 *) &xw[8];
         *(float4 *) &w[12] = *(const float4 *) &xw[12];
         *(float4 *) &gv[0] = *(const float4 *) &sg[j];
         *(float4 *) &gv[4] = *(const float4 *) &sg[j + 4];
#pragma unroll
         for (int i = 0; i < 8; i++)
#pragma unroll
            for (int r = 0; r < 8; r++) acc[r] = fmaf(gv[i], w[r + i], acc[r]);
      }
   }
#pragma unroll
   for (int r = 0; r < 8; r++) red[sl * ncp * 8 + cg * 8 + r] = acc[r];
   __syncthreads();
   for (int cc = tid; cc < c.T; cc += 256) {
      float sum = 0.0f;
      for (int q = 0; q < slices; q++) sum += red[q * ncp * 8 + cc];
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
   cudaFree(p->dDxItems);
   cudaFree(p->dFwdStart);
   cudaFree(p->dOrder);
   delete p;
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
   std::vector<int2> fwd, dx;
   std::vector<int> start(numChannels + 1), order(numChannels);
   long long xo = 0, ho = 0, co = 0;
   for (int c = 0; c < numChannels; c++) {
      const int L = length[c], T = taps[c], S = stages[c];
      if (T < 1 || T > kDhMaxT || L < T || S < 0 || S > kRaggedMaxStages) {
         delete p;
         return DSPLIB_ERR_INVALID_DIMENSION;
      }
      ch[c] = RaggedChan{xo, ho, co, L, T, S, L - T + 1};
      xo += L;
      p->totalOut += L - T + 1;
      ho += T;
      co += 5LL * S;
      p->Smax = std::max(p->Smax, S);
      p->Tmax = std::max(p->Tmax, T);
      start[c] = (int) fwd.size();
      for (int t = 0; t * 2048 < L - T + 1; t++) fwd.push_back(make_int2(c, t));
      for (int t = 0; t * 2048 < L; t++) dx.push_back(make_int2(c, t));
      order[c] = c;
   }
   start[numChannels] = (int) fwd.size();
   std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ch[a].Lu > ch[b].Lu; });
   p->totalLen = xo;
   p->totalTaps = ho;
   p->totalCoefs = co;
   p->nFwdItems = (int) fwd.size();
   p->nDxItems = (int) dx.size();
   cudaGetDevice(&p->device);
   const bool ok = upload(&p->dChan, ch) == cudaSuccess && upload(&p->dFwdItems, fwd) == cudaSuccess &&
                   upload(&p->dDxItems, dx) == cudaSuccess && upload(&p->dFwdStart, start) == cudaSuccess &&
                   upload(&p->dOrder, order) == cudaSuccess;
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
   case DSPLIB_GPU_RAGGED_WORK: return (long long) (p->Smax + 1) * p->totalLen;
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
   cudaStream_t s = (cudaStream_t) stream;
   fir_ragged_kernel<false><<<p->nFwdItems, kRThreads, 0, s>>>(p->dChan, p->dFwdItems, x, taps, work);
   const size_t dyn = kRaggedMaxStages * sizeof(double2) + (size_t) std::max(1, p->Smax) * kBPowers * sizeof(M2);
   if (cudaFuncSetAttribute(biquad_ragged_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn) !=
       cudaSuccess)
      return DSPLIB_ERR_FAILURE;
   biquad_ragged_kernel<false><<<p->C, kBThreads, dyn, s>>>(p->dChan, p->dOrder, coefs, nullptr, work,
                                                              p->totalLen, y, 0, nullptr);
   countLaunch(2);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_bwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, const float *work, const float *gy, float *gx,
                                              float *gtaps, float *gcoefs, float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !x || !taps || ((!coefs || !gcoefs) && p->totalCoefs) || !work || !gy || !gx || !gtaps || !scratch)
      return DSPLIB_ERR_NULL_POINTER;
   cudaStream_t s = (cudaStream_t) stream;
   float *g = scratch;                // running gradient (in place per stage)
   float *v = scratch + p->totalLen;  // anti-causal AR output of the current stage
   float *part = scratch + 2 * p->totalLen;
   cudaError_t e = cudaMemcpyAsync(g, gy, (size_t) p->totalLen * sizeof(float), cudaMemcpyDeviceToDevice, s);
   if (e != cudaSuccess) return DSPLIB_ERR_FAILURE;
   int launches = 0;
   const size_t dynBwd = kRaggedMaxStages * sizeof(double2) + kBPowers * sizeof(M2);
   for (int st = p->Smax - 1; st >= 0; st--) {
      biquad_ragged_kernel<true><<<p->C, kBThreads, dynBwd, s>>>(p->dChan, p->dOrder, coefs, g,
                                                                          (float *) work, p->totalLen, nullptr,
                                                                          st, v);
      biquad_ragged_bwd_kernel<<<p->nFwdItems, 256, 0, s>>>(p->dChan, p->dFwdItems, coefs, work, p->totalLen,
                                                            v, g, (double *) part, st);
      biquad_coef_reduce_kernel<<<p->C, 32, 0, s>>>(p->dChan, p->dFwdStart, (const double *) part, gcoefs, st);
      launches += 3;
   }
   fir_ragged_kernel<true><<<p->nDxItems, kRThreads, 0, s>>>(p->dChan, p->dDxItems, g, taps, gx);
   fir_dh_partial_kernel<<<p->nFwdItems, 256, 0, s>>>(p->dChan, p->dFwdItems, x, g, part);
   fir_dh_reduce_kernel<<<p->C, 256, 0, s>>>(p->dChan, p->dFwdStart, part, gtaps);
   countLaunch(launches + 3);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

DSPLIB_STATUS DSPLIB_gpu_raggedMseGrad(DSPLIB_gpu_raggedPlan plan, const float *y, const float *target, float *gy,
                                       float *loss, float *scratch, void *stream)
{
   RaggedPlan *p = (RaggedPlan *) plan;
   if (!p || !y || !target || !gy || !loss || !scratch) return DSPLIB_ERR_NULL_POINTER;
   if (p->totalOut <= 0) return DSPLIB_ERR_INVALID_DIMENSION;
   cudaStream_t s = (cudaStream_t) stream;
   double *part = (double *) scratch;
   mse_partial_kernel<<<p->nFwdItems, 256, 0, s>>>(p->dChan, p->dFwdItems, y, target, gy, part,
                                                   (float) (2.0 / (double) p->totalOut));
   mse_reduce_kernel<<<1, 1024, 0, s>>>(part, p->nFwdItems, 1.0 / (double) p->totalOut, loss);
   countLaunch(2);
   return cudaGetLastError() == cudaSuccess ? DSPLIB_SUCCESS : DSPLIB_ERR_FAILURE;
}

} // extern "C"
