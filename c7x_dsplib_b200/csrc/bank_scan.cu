// Cascade of direct-form-II biquads of the batched filter bank, forward and
// adjoint, split along time: every channel is cut into segments that
// independent CTAs filter at the same time, so a 262144-sample channel keeps
// 64 CTAs busy instead of one.
//
// Within a segment (one CTA) each thread owns a chunk of 16 consecutive
// samples.  Per stage:
//   1. the chunk is filtered from a zero state (the only serial pass);
//   2. the chunk end states are combined by a chunked scan: lanes of a warp
//      (shuffles), warps of the CTA (shared memory), segments of the channel
//      (decoupled look-back over records in global memory); the combine is
//      the affine map s -> M s + e with M = A^16 and its powers, A the
//      stage's 2x2 companion matrix, formed in FP64 and rounded once;
//   3. the true output follows without a serial chain: the free response
//      of the chunk's true initial state (w1, w2) is added sample by sample,
//      w[i] = w_zs[i] + alpha_i w1 + beta_i w2 with (alpha_i, beta_i) the
//      first row of A^(i+1), then y[i] = b0 w[i] + b1 w[i-1] + b2 w[i-2].
//
// Decoupled look-back: a CTA takes its segment from a ticket counter, so every
// earlier segment of its channel is already running or done.  It publishes the
// segment's zero-entry end state (aggregate, flag 1) as soon as its local scan
// is done, then walks back over its predecessors, adding each one's aggregate
// times the segment transition power until it meets an inclusive state (flag 2)
// or the power has become exactly zero in FP32 (older segments then contribute
// exactly nothing), and publishes its own inclusive state.  Every wait is
// bounded; on expiry the kernel raises the plan's error word and continues with
// what it has, so it always terminates.
//
// Forward (bank_fwd_kernel, 256 threads, 4096-sample segments): all stages of
// the cascade, the last one's output to y.  It stores no stage output: the
// state at the start of every 512-sample span (one warp) of every stage is kept
// as a checkpoint, 2 floats per 512 samples per stage.
//
// Adjoint (bank_bwd_kernel, 128 threads, 2048-sample segments, persistent):
// the forward of the segment is recomputed warp by warp from the checkpoints
// (no CTA barrier: every warp knows its entry state), keeping each stage's
// internal sequence w_s in shared memory; then the stages run in reverse
// order, each as the reverse-time recursion of the DF2 adjoint,
//     v[t] = g[t] - a1 v[t+1] - a2 v[t+2],  lambda[t] = b0 v[t] + b1 v[t+1] + b2 v[t+2],
// with the same chunked scan in reverse (segments in decreasing time order,
// look-back toward later segments), g = the stage's output gradient and lambda
// its input gradient.  Coefficient gradients:
//     dL/db_i = sum_t g[t] w[t-i],   dL/da_i = -sum_t lambda[t] w[t-i],
// summed per chunk in FP32, per warp by shuffles, per segment in FP64, and
// per channel in FP64 in segment order by the last segment's CTA (bitwise
// repeatable whatever the CTA schedule).
#include <cuda_runtime.h>

#include "dsplib_internal.h"
#include "scan_common.cuh"

namespace dsplib {
namespace {

using scan::M2;
using scan::M2f;

constexpr int kL = 16;          // samples per chunk (thread)
constexpr int kSpan = 32 * kL;  // samples per warp: checkpoint granularity
constexpr int kFwdWarps = 8;
constexpr int kFwdThreads = kFwdWarps * 32;
constexpr int kFwdSeg = kFwdThreads * kL; // 4096: transition A^4096 = M^256 = P[8]
constexpr int kBwdWarps = 4;
constexpr int kBwdThreads = kBwdWarps * 32;
constexpr int kBwdSeg = kBwdThreads * kL; // 2048: transition A^2048 = M^128 = P[7]
constexpr int kOutPad = kL + 1;           // padded shared row per chunk (conflict-free staging)

static_assert(kFwdSeg == kBankFwdSeg && kBwdSeg == kBankBwdSeg && kSpan == kBankSpan, "segment sizes");

// Stage table (floats): [0, 5) b0 b1 b2 a1 a2; [8 + 4k, 12 + 4k) P[k] = M^(2^k), M = A^16,
// k = 0..8, row-major; [44 + 2i, 46 + 2i) alpha_i, beta_i = row 0 of A^(i+1), i = 0..15.
constexpr int kTabP = 8;
constexpr int kTabAB = 44;
static_assert(kTabAB + 2 * kL <= kBankTabFloats, "stage table layout");

__device__ __forceinline__ M2f tabP(const float *tb, int k)
{
   const float4 q = *(const float4 *) (tb + kTabP + 4 * k);
   return {q.x, q.y, q.z, q.w};
}

__device__ __forceinline__ float2 f2add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ float2 shflDown(float2 v, int d)
{
   v.x = __shfl_down_sync(0xffffffffu, v.x, d);
   v.y = __shfl_down_sync(0xffffffffu, v.y, d);
   return v;
}

__device__ __forceinline__ M2f mmulF(const M2f &x, const M2f &y)
{
   return {fmaf(x.a, y.a, x.b * y.c), fmaf(x.a, y.b, x.b * y.d), fmaf(x.c, y.a, x.d * y.c),
           fmaf(x.c, y.b, x.d * y.d)};
}

// ------------------------------------------------------------------ decoupled look-back

// Bounded wait for a record flag set by another CTA; 0 when the wait gave up
// (limit 0: give up at once, which tests use to exercise the expiry path).
__device__ __forceinline__ int waitFlag(const int *flag, int limit)
{
   for (int i = 0; i < limit; i++) {
      int f;
      asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(f) : "l"(flag) : "memory");
      if (f) return f;
      __nanosleep(64);
   }
   return 0;
}

__device__ __forceinline__ float2 loadRecord(const float4 *rec, int which)
{
   const float *p = (const float *) rec + 2 * which;
   float2 v;
   asm volatile("ld.relaxed.gpu.global.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p) : "memory");
   return v;
}

// Record r: (aggregate, inclusive); flag 1 = aggregate valid, 2 = inclusive valid.
__device__ __forceinline__ void publish(float4 *recs, int *flags, int r, float2 v, int state)
{
   float *p = (float *) (recs + r) + 2 * (state - 1);
   p[0] = v.x;
   p[1] = v.y;
   asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(flags + r), "r"(state) : "memory");
}

// State entering a segment from the `preds` segments before it (in the scan's
// direction): records r, r - S, r - 2S, ... of the same stage.
__device__ float2 lookBack(const float4 *recs, const int *flags, int r, int preds, int S, const M2f &PW, int limit,
                           int *err)
{
   float2 z = make_float2(0.0f, 0.0f);
   M2f Mp = {1.0f, 0.0f, 0.0f, 1.0f};
   for (int j = 0; j < preds; j++, r -= S) {
      const int f = waitFlag(flags + r, limit);
      if (!f) {
         atomicOr(err, kBankErrWait);
         break;
      }
      z = scan::affine(Mp, loadRecord(recs + r, f - 1), z);
      if (f == 2) break;
      Mp = mmulF(Mp, PW);
      if (Mp.a == 0.0f && Mp.b == 0.0f && Mp.c == 0.0f && Mp.d == 0.0f) break;
   }
   return z;
}

// ------------------------------------------------------------------ stage tables

__global__ void __launch_bounds__(128) bank_tables_kernel(const float *coefs, int totalStages, float *tables)
{
   const int g = blockIdx.x * blockDim.x + threadIdx.x;
   if (g >= totalStages) return;
   const float *cf = coefs + 5LL * g;
   float *tb = tables + (long long) g * kBankTabFloats;
   for (int k = 0; k < 5; k++) tb[k] = cf[k];
   for (int k = 5; k < kTabP; k++) tb[k] = 0.0f;
   const double a1 = cf[3], a2 = cf[4];
   // row 0 of A^(i+1): row0(A^(i+2)) = row0(A^(i+1)) A, A = [[-a1, -a2], [1, 0]]
   double r0 = -a1, r1 = -a2;
   for (int i = 0; i < kL; i++) {
      tb[kTabAB + 2 * i] = (float) r0;
      tb[kTabAB + 2 * i + 1] = (float) r1;
      const double n0 = fma(r0, -a1, r1), n1 = r0 * -a2;
      r0 = n0;
      r1 = n1;
   }
   M2 M = {-a1, -a2, 1.0, 0.0};
   for (int r = 1; r < kL; r <<= 1) M = scan::mmul(M, M);
   for (int k = 0; k <= 8; k++) {
      const M2f f = scan::toF(M);
      *(float4 *) (tb + kTabP + 4 * k) = make_float4(f.a, f.b, f.c, f.d);
      M = scan::mmul(M, M);
   }
   for (int k = kTabAB + 2 * kL; k < kBankTabFloats; k++) tb[k] = 0.0f;
}

// ------------------------------------------------------------------ forward

struct FwdArgs {
   const RaggedChan *chans;
   const int4 *units; // {channel, segment, segments of the channel, first record}
   const float *tables;
   const float *u;    // FIR output plane (channel c at pOff)
   float *y;
   float2 *ckpt;
   float4 *recs;
   int *flags;
   int *ticket;
   int *err;
   int limit;
};

// Load the 16 samples of a chunk from a 16-float-aligned plane row, zero at t >= n.
__device__ __forceinline__ void loadChunk(float (&v)[kL], const float *row, int t0, int n)
{
   const int np = (n + 15) & ~15; // the row is allocated to a multiple of 16 floats
   if (t0 < np) {
#pragma unroll
      for (int q = 0; q < kL / 4; q++) {
         const float4 f = *(const float4 *) (row + t0 + 4 * q);
         v[4 * q + 0] = t0 + 4 * q + 0 < n ? f.x : 0.0f;
         v[4 * q + 1] = t0 + 4 * q + 1 < n ? f.y : 0.0f;
         v[4 * q + 2] = t0 + 4 * q + 2 < n ? f.z : 0.0f;
         v[4 * q + 3] = t0 + 4 * q + 3 < n ? f.w : 0.0f;
      }
   }
   else {
#pragma unroll
      for (int i = 0; i < kL; i++) v[i] = 0.0f;
   }
}

// DF2 over the chunk from a zero state (w[i]), returning the end state (w[15], w[14]).
__device__ __forceinline__ float2 zeroStatePass(const float (&v)[kL], float (&w)[kL], float a1, float a2)
{
   float p1 = 0.0f, p2 = 0.0f;
#pragma unroll
   for (int i = 0; i < kL; i++) {
      w[i] = fmaf(-a1, p1, fmaf(-a2, p2, v[i]));
      p2 = p1;
      p1 = w[i];
   }
   return make_float2(w[kL - 1], w[kL - 2]);
}

// Warp-level inclusive scan in time order (lane L combines the chunks of lanes <= L).
__device__ __forceinline__ float2 warpScanUp(float2 val, const float *tb, int lane)
{
#pragma unroll
   for (int k = 0; k < 5; k++) {
      const float2 o = scan::shflUp(val, 1 << k, 32);
      if (lane >= (1 << k)) val = scan::affine(tabP(tb, k), o, val);
   }
   return val;
}

// Chunk initial state: M^lane * warp entry + the exclusive prefix of the lanes before.
__device__ __forceinline__ float2 chunkInitUp(float2 val, float2 entry, const float *tb, int lane)
{
   float2 ex = scan::shflUp(val, 1, 32);
   if (lane == 0) ex = make_float2(0.0f, 0.0f);
#pragma unroll
   for (int k = 0; k < 5; k++)
      if ((lane >> k) & 1) entry = scan::affine(tabP(tb, k), entry, make_float2(0.0f, 0.0f));
   return f2add(entry, ex);
}

// True internal sequence (in place of the zero-state one) and stage output, from the
// chunk's initial state (w1, w2) = (w[-1], w[-2]).
__device__ __forceinline__ void correctAndOutput(float (&w)[kL], float (&out)[kL], const float *tb, float w1, float w2)
{
   const float b0 = tb[0], b1 = tb[1], b2 = tb[2];
   float q1 = w1, q2 = w2;
#pragma unroll
   for (int i = 0; i < kL; i++) {
      const float2 ab = *(const float2 *) (tb + kTabAB + 2 * i);
      const float wt = fmaf(ab.x, w1, fmaf(ab.y, w2, w[i]));
      out[i] = fmaf(b0, wt, fmaf(b1, q1, b2 * q2));
      w[i] = wt;
      q2 = q1;
      q1 = wt;
   }
}

__global__ void __launch_bounds__(kFwdThreads) bank_fwd_kernel(FwdArgs a)
{
   extern __shared__ float4 dynF[];
   float *sTab = (float *) dynF; // the channel's stage tables
   __shared__ float sOut[kFwdThreads * kOutPad];
   __shared__ float2 sAgg[kFwdWarps], sEntry[kFwdWarps];
   __shared__ int sTicket;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   if (tid == 0) sTicket = atomicAdd(a.ticket, 1);
   __syncthreads();
   const int4 U = a.units[sTicket];
   const RaggedChan c = a.chans[U.x];
   const int S = c.S, Lu = c.Lu;
   {
      const float4 *src = (const float4 *) (a.tables + (c.cOff / 5) * kBankTabFloats);
      for (int i = tid; i < S * (kBankTabFloats / 4); i += kFwdThreads) dynF[i] = src[i];
   }
   const int segStart = U.y * kFwdSeg;
   float v[kL];
   loadChunk(v, a.u + c.pOff, segStart + tid * kL, Lu);
   __syncthreads();
   const float2 zero = make_float2(0.0f, 0.0f);
   for (int s = 0; s < S; s++) {
      const float *tb = sTab + s * kBankTabFloats;
      float w[kL];
      float2 val = warpScanUp(zeroStatePass(v, w, tb[3], tb[4]), tb, lane);
      if (lane == 31) sAgg[warp] = val;
      __syncthreads();
      if (warp == 0) {
         float2 tv = lane < kFwdWarps ? sAgg[lane] : zero;
#pragma unroll
         for (int k = 0; k < 3; k++) {
            const float2 o = scan::shflUp(tv, 1 << k, 32);
            if (lane >= (1 << k) && lane < kFwdWarps) tv = scan::affine(tabP(tb, 5 + k), o, tv);
         }
         const float2 agg = scan::shflIdx(tv, kFwdWarps - 1);
         float2 z = zero;
         if (lane == 0 && U.z > 1) {
            const int r = U.w + s;
            const bool succ = U.y + 1 < U.z;
            if (U.y == 0) {
               if (succ) publish(a.recs, a.flags, r, agg, 2);
            }
            else {
               if (succ) publish(a.recs, a.flags, r, agg, 1);
               z = lookBack(a.recs, a.flags, r - S, U.y, S, tabP(tb, 8), a.limit, a.err);
               if (succ) publish(a.recs, a.flags, r, scan::affine(tabP(tb, 8), z, agg), 2);
            }
         }
         z = scan::shflIdx(z, 0);
         const float2 before = scan::shflUp(tv, 1, 32);
         if (lane < kFwdWarps) {
            float2 e = z;
#pragma unroll
            for (int k = 0; k < 3; k++)
               if ((lane >> k) & 1) e = scan::affine(tabP(tb, 5 + k), e, zero);
            if (lane > 0) e = f2add(e, before);
            sEntry[lane] = e;
            const int span = U.y * kFwdWarps + lane;
            if (span * kSpan < Lu) a.ckpt[c.ckOff + (long long) span * S + s] = e;
         }
      }
      __syncthreads();
      const float2 st = chunkInitUp(val, sEntry[warp], tb, lane);
      correctAndOutput(w, v, tb, st.x, st.y);
   }
   // output through shared memory: each warp store covers 32 consecutive samples
#pragma unroll
   for (int i = 0; i < kL; i++) sOut[tid * kOutPad + i] = v[i];
   __syncthreads();
   float *yc = a.y + c.xOff;
   const int n = min(kFwdSeg, Lu - segStart);
   for (int k = tid; k < n; k += kFwdThreads) yc[segStart + k] = sOut[(k >> 4) * kOutPad + (k & 15)];
   if (U.y + 1 == U.z)
      for (int t = Lu + tid; t < c.L; t += kFwdThreads) yc[t] = 0.0f;
}

// ------------------------------------------------------------------ adjoint

struct BwdArgs {
   const RaggedChan *chans;
   const int4 *units; // segments in decreasing time order within each channel
   int nUnits;
   const float *tables;
   const float *u;
   const float *gy;
   const float2 *ckpt;
   float *g;          // gradient w.r.t. the FIR output (channel c at xOff, Lu samples)
   float4 *recs;
   int *flags;
   double *gpart;     // per record: 5 coefficient-gradient partial sums
   int *chanDone;
   int *ticket;
   float *gcoefs;
   int *err;
   int limit;
   float *wGlobal;    // stage sequences when they do not fit in shared memory (per CTA)
   int wInShared;
   int Smax;
};

// Stage sequences of one chunk: w[0..15] and the initial state w[-1], w[-2] for each
// stage, laid out [stage][18][thread] so that the threads of a warp touch distinct banks.
constexpr int kWRows = kL + 2;

__global__ void __launch_bounds__(kBwdThreads) bank_bwd_kernel(BwdArgs a)
{
   extern __shared__ float4 dynB[];
   float *sTab = (float *) dynB;
   float *W = a.wInShared ? sTab + (size_t) a.Smax * kBankTabFloats
                          : a.wGlobal + (size_t) blockIdx.x * a.Smax * kWRows * kBwdThreads;
   __shared__ float sIO[kBwdThreads * kOutPad];
   __shared__ float2 sAgg[kBwdWarps], sEntry[kBwdWarps];
   __shared__ float sRed[2][kBwdWarps][5];
   __shared__ int sTicket, sLast;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const float2 zero = make_float2(0.0f, 0.0f);
   for (;;) {
      if (tid == 0) sTicket = atomicAdd(a.ticket, 1);
      __syncthreads();
      const int ti = sTicket;
      if (ti >= a.nUnits) break;
      const int4 U = a.units[ti];
      const RaggedChan c = a.chans[U.x];
      const int S = c.S, Lu = c.Lu;
      const int segStart = U.y * kBwdSeg;
      const int n = min(kBwdSeg, Lu - segStart);
      {
         const float4 *src = (const float4 *) (a.tables + (c.cOff / 5) * kBankTabFloats);
         for (int i = tid; i < S * (kBankTabFloats / 4); i += kBwdThreads) dynB[i] = src[i];
      }
      // output gradient of the last stage, staged for coalesced reads
      for (int k = tid; k < kBwdSeg; k += kBwdThreads)
         sIO[(k >> 4) * kOutPad + (k & 15)] = k < n ? a.gy[c.xOff + segStart + k] : 0.0f;
      float v[kL];
      loadChunk(v, a.u + c.pOff, segStart + tid * kL, Lu);
      __syncthreads();
      float g[kL];
#pragma unroll
      for (int i = 0; i < kL; i++) g[i] = sIO[tid * kOutPad + i];

      // 1. recompute the forward of this segment, warp by warp from the checkpoints
      const int span = U.y * kBwdWarps + warp;
      const bool spanValid = span * kSpan < Lu;
      for (int s = 0; s < S; s++) {
         const float *tb = sTab + s * kBankTabFloats;
         float w[kL];
         const float2 val = warpScanUp(zeroStatePass(v, w, tb[3], tb[4]), tb, lane);
         const float2 entry = spanValid ? a.ckpt[c.ckOff + (long long) span * S + s] : zero;
         const float2 st = chunkInitUp(val, entry, tb, lane);
         correctAndOutput(w, v, tb, st.x, st.y);
         float *Ws = W + (size_t) s * kWRows * kBwdThreads + tid;
#pragma unroll
         for (int i = 0; i < kL; i++) Ws[i * kBwdThreads] = w[i];
         Ws[kL * kBwdThreads] = st.x;       // w[-1]
         Ws[(kL + 1) * kBwdThreads] = st.y; // w[-2]
      }

      // 2. the stages' adjoints, last stage first, in reverse time
      for (int s = S - 1; s >= 0; s--) {
         const float *tb = sTab + s * kBankTabFloats;
         const float b0 = tb[0], b1 = tb[1], b2 = tb[2], a1 = tb[3], a2 = tb[4];
         float vz[kL];
         {
            float p1 = 0.0f, p2 = 0.0f;
#pragma unroll
            for (int i = kL - 1; i >= 0; i--) {
               vz[i] = fmaf(-a1, p1, fmaf(-a2, p2, g[i]));
               p2 = p1;
               p1 = vz[i];
            }
         }
         // reverse-time scan: lane L combines the chunks of lanes >= L
         float2 val = make_float2(vz[0], vz[1]);
#pragma unroll
         for (int k = 0; k < 5; k++) {
            const float2 o = shflDown(val, 1 << k);
            if (lane + (1 << k) < 32) val = scan::affine(tabP(tb, k), o, val);
         }
         if (lane == 0) sAgg[warp] = val;
         __syncthreads();
         // partial sums of the stage before (one stage later in time) are complete in sRed
         if (tid == 0 && s + 1 < S) {
            double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
            for (int w = 0; w < kBwdWarps; w++)
               for (int k = 0; k < 5; k++) acc[k] += (double) sRed[(s + 1) & 1][w][k];
            for (int k = 0; k < 5; k++) a.gpart[(long long) (U.w + s + 1) * 5 + k] = acc[k];
         }
         if (warp == 0) {
            float2 tv = lane < kBwdWarps ? sAgg[lane] : zero;
#pragma unroll
            for (int k = 0; k < 2; k++) {
               const float2 o = shflDown(tv, 1 << k);
               if (lane + (1 << k) < kBwdWarps) tv = scan::affine(tabP(tb, 5 + k), o, tv);
            }
            const float2 agg = scan::shflIdx(tv, 0);
            float2 z = zero;
            if (lane == 0 && U.z > 1) {
               const int r = U.w + s;
               const int preds = U.z - 1 - U.y; // later segments of the channel
               const bool succ = U.y > 0;
               if (preds == 0) {
                  if (succ) publish(a.recs, a.flags, r, agg, 2);
               }
               else {
                  if (succ) publish(a.recs, a.flags, r, agg, 1);
                  z = lookBack(a.recs, a.flags, r - S, preds, S, tabP(tb, 7), a.limit, a.err);
                  if (succ) publish(a.recs, a.flags, r, scan::affine(tabP(tb, 7), z, agg), 2);
               }
            }
            z = scan::shflIdx(z, 0);
            const float2 after = shflDown(tv, 1);
            if (lane < kBwdWarps) {
               float2 e = z;
               const int m = kBwdWarps - 1 - lane;
#pragma unroll
               for (int k = 0; k < 2; k++)
                  if ((m >> k) & 1) e = scan::affine(tabP(tb, 5 + k), e, zero);
               if (lane + 1 < kBwdWarps) e = f2add(e, after);
               sEntry[lane] = e;
            }
         }
         __syncthreads();
         // this chunk's reverse-time initial state (v[16], v[17])
         float2 ex = shflDown(val, 1);
         if (lane == 31) ex = zero;
         float2 st = sEntry[warp];
         const int m = 31 - lane;
#pragma unroll
         for (int k = 0; k < 5; k++)
            if ((m >> k) & 1) st = scan::affine(tabP(tb, k), st, zero);
         st = f2add(st, ex);
         // forward sequence of this stage: wr[i + 2] = w[i], wr[1] = w[-1], wr[0] = w[-2]
         float wr[kL + 2];
         {
            const float *Ws = W + (size_t) s * kWRows * kBwdThreads + tid;
#pragma unroll
            for (int i = 0; i < kL; i++) wr[i + 2] = Ws[i * kBwdThreads];
            wr[1] = Ws[kL * kBwdThreads];
            wr[0] = Ws[(kL + 1) * kBwdThreads];
         }
         float pb0 = 0.0f, pb1 = 0.0f, pb2 = 0.0f, pa1 = 0.0f, pa2 = 0.0f;
         float n1 = st.x, n2 = st.y; // v[i+1], v[i+2]
#pragma unroll
         for (int i = kL - 1; i >= 0; i--) {
            const float2 ab = *(const float2 *) (tb + kTabAB + 2 * (kL - 1 - i));
            const float vi = fmaf(ab.x, st.x, fmaf(ab.y, st.y, vz[i]));
            const float lam = fmaf(b0, vi, fmaf(b1, n1, b2 * n2));
            n2 = n1;
            n1 = vi;
            pb0 = fmaf(g[i], wr[i + 2], pb0);
            pb1 = fmaf(g[i], wr[i + 1], pb1);
            pb2 = fmaf(g[i], wr[i], pb2);
            pa1 = fmaf(-lam, wr[i + 1], pa1);
            pa2 = fmaf(-lam, wr[i], pa2);
            g[i] = lam;
         }
         float p[5] = {pb0, pb1, pb2, pa1, pa2};
#pragma unroll
         for (int k = 0; k < 5; k++) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) p[k] += __shfl_xor_sync(0xffffffffu, p[k], o);
         }
         if (lane == 0)
#pragma unroll
            for (int k = 0; k < 5; k++) sRed[s & 1][warp][k] = p[k];
      }
      // input gradient of the cascade (gradient w.r.t. the FIR output), coalesced store
#pragma unroll
      for (int i = 0; i < kL; i++) sIO[tid * kOutPad + i] = g[i];
      __syncthreads();
      if (tid == 0 && S > 0) {
         double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
         for (int w = 0; w < kBwdWarps; w++)
            for (int k = 0; k < 5; k++) acc[k] += (double) sRed[0][w][k];
         for (int k = 0; k < 5; k++) a.gpart[(long long) U.w * 5 + k] = acc[k];
      }
      for (int k = tid; k < n; k += kBwdThreads) a.g[c.xOff + segStart + k] = sIO[(k >> 4) * kOutPad + (k & 15)];
      // the last segment of the channel to finish sums the coefficient gradients in segment order
      if (S > 0) {
         __threadfence();
         __syncthreads();
         if (tid == 0) sLast = atomicAdd(a.chanDone + U.x, 1) == U.z - 1;
         __syncthreads();
         if (sLast) {
            __threadfence();
            const int r0 = U.w - (U.z - 1 - U.y) * S; // records of segment U.z - 1 (the channel's first ticket)
            for (int q = tid; q < 5 * S; q += kBwdThreads) {
               double acc = 0.0;
               for (int j = 0; j < U.z; j++) acc += __ldcg(a.gpart + (long long) (r0 + (U.z - 1 - j) * S) * 5 + q);
               a.gcoefs[c.cOff + q] = (float) acc;
            }
         }
      }
      __syncthreads(); // shared memory is reused by the next segment
   }
}

} // namespace

cudaError_t launchBankTables(const float *coefs, int totalStages, float *tables, cudaStream_t s)
{
   if (totalStages <= 0) return cudaSuccess;
   bank_tables_kernel<<<(totalStages + 127) / 128, 128, 0, s>>>(coefs, totalStages, tables);
   countLaunch();
   return cudaGetLastError();
}

cudaError_t launchBankForward(const BankLaunch &b, cudaStream_t s)
{
   if (b.nUnits <= 0) return cudaSuccess;
   const size_t dyn = (size_t) b.Smax * kBankTabFloats * sizeof(float);
   cudaError_t e = cudaFuncSetAttribute(bank_fwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn);
   if (e != cudaSuccess) return e;
   FwdArgs a{b.chans, b.units, b.tables, b.u, b.y, b.ckpt, b.recs, b.flags, b.ticket, b.err, b.waitLimit};
   bank_fwd_kernel<<<b.nUnits, kFwdThreads, dyn, s>>>(a);
   countLaunch();
   return cudaGetLastError();
}

size_t bankBackwardShared(int Smax, bool wInShared)
{
   return (size_t) Smax * kBankTabFloats * sizeof(float) +
          (wInShared ? (size_t) Smax * kWRows * kBwdThreads * sizeof(float) : 0);
}

bool bankBackwardFitsShared(int Smax) { return bankBackwardShared(Smax, true) <= kBankBwdSharedLimit; }

long long bankBackwardGlobalFloats(int Smax, int ctas) { return (long long) ctas * Smax * kWRows * kBwdThreads; }

cudaError_t launchBankBackward(const BankLaunch &b, int ctas, cudaStream_t s)
{
   if (b.nUnits <= 0) return cudaSuccess;
   const bool inShared = bankBackwardFitsShared(b.Smax);
   const size_t dyn = bankBackwardShared(b.Smax, inShared);
   cudaError_t e = cudaFuncSetAttribute(bank_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn);
   if (e != cudaSuccess) return e;
   BwdArgs a{b.chans, b.units, b.nUnits, b.tables, b.u, b.gy, b.ckpt, b.g, b.recs, b.flags, b.gpart,
             b.chanDone, b.ticket, b.gcoefs, b.err, b.waitLimit, b.wGlobal, inShared ? 1 : 0, b.Smax};
   bank_bwd_kernel<<<ctas, kBwdThreads, dyn, s>>>(a);
   countLaunch();
   return cudaGetLastError();
}

int bankBackwardCtas(int Smax, int nUnits)
{
   const bool inShared = bankBackwardFitsShared(Smax);
   const size_t dyn = bankBackwardShared(Smax, inShared);
   int dev = 0, sms = 148, perSm = 1;
   if (cudaGetDevice(&dev) == cudaSuccess) (void) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
   if (cudaFuncSetAttribute(bank_bwd_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn) ==
           cudaSuccess &&
       cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, bank_bwd_kernel, kBwdThreads, dyn) == cudaSuccess) {
      if (perSm < 1) perSm = 1;
   }
   else {
      (void) cudaGetLastError();
      perSm = 1;
   }
   const long long ctas = (long long) sms * perSm;
   return (int) (ctas < nUnits ? ctas : nUnits);
}

} // namespace dsplib
