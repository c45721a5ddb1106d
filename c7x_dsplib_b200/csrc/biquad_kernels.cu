// Cascade-biquad CUDA kernels for sm_100a.
//
// biquad_seq_kernel   one thread per channel, one sequential recursion per
//                     stage, operations in the order of the reference
//                     natural-C kernels (src/DSPLIB_cascadeBiquad/
//                     DSPLIB_cascadeBiquad_cn.cpp: DF2 :84-85, DF1 :230,
//                     TDF2 :386-388) with separately rounded float operations,
//                     so NATC results are bit-exact; the TI form follows
//                     DSPLIB_cascadeBiquad_tif_lStage_ci.cpp:204-214.
//
// biquad_scan_kernel  chunked parallel-in-time scan.  Lane = channel (32
//                     channels per CTA, so every time row is one coalesced
//                     128-byte access), warp = chunk of L consecutive samples,
//                     CTA = W chunks, cluster of K CTAs = one window of K*W*L
//                     samples.  For each stage:
//                       1. every chunk runs the stage recursion from a zero
//                          state, giving its end state e (FP32);
//                       2. each warp forms its chunk's true initial state
//                          from the end states of the chunks before it, by
//                          Horner's rule with M = A^L (A: the stage's
//                          one-sample state-transition matrix), lane =
//                          channel; across the CTAs of the cluster the last
//                          warp forms the CTA's span aggregates by a pairwise
//                          tree and pushes them into every CTA's shared memory
//                          (distributed shared memory), the warps form their
//                          prefixes while the cluster barrier completes, and
//                          one warp carries the window entry over the earlier
//                          CTAs' aggregates with Mc = A^(W*L) for all; the
//                          matrix powers are formed in FP64 and rounded once,
//                          the combination runs in FP32;
//                       3. every chunk reruns the recursion from its true
//                          initial state and its outputs become the next
//                          stage's input, kept in registers.
//                     The input is read once and the output written once.
//                     Windows of one cluster run in sequence, carrying the
//                     state across window boundaries.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdio>

#include "dsplib_internal.h"

namespace cg = cooperative_groups;

namespace dsplib {

namespace {

constexpr int kTifGroup = 7;

__device__ __forceinline__ int tifGroups(int S) { return S <= kTifGroup ? 1 : (S + kTifGroup - 1) / kTifGroup; }
__device__ __forceinline__ int tifPer(int S) { return S <= kTifGroup ? S : kTifGroup; }

// Coefficients of stage s for channel ch, from any of the accepted layouts.
// DF forms: {b0, b1, b2, a1, a2}.  TIF: {c0, c1, a12, a11} (storage order of
// DSPLIB_cascadeBiquad_utils.cpp:227-231), k[4] = group gain when s ends a group.
struct Coef {
   float k[5];
};

__device__ Coef loadCoef(const BiquadLaunch &a, int s, int ch)
{
   Coef c;
   if (a.form == DSPLIB_BIQUAD_TIF && a.optLayout) {
      const int S = a.S, G = tifGroups(S), per = tifPer(S);
      const bool last = (s % per == per - 1) || s == S - 1;
      const int g = s / per;
      if (a.nch) {
         for (int k = 0; k < 4; k++) c.k[k] = a.coef[((long long) k * S + s) * a.coefPitch + ch];
         c.k[4] = last ? a.coef[((long long) 4 * S + g) * a.coefPitch + ch] : 1.0f;
      }
      else {
         for (int k = 0; k < 4; k++) c.k[k] = a.coef[s * 4 + k];
         c.k[4] = last ? a.coef[4 * S + g] : 1.0f;
      }
      (void) G;
   }
   else if (a.optLayout && a.nch) {
      for (int k = 0; k < 5; k++) c.k[k] = a.coef[((long long) s * 5 + k) * a.coefPitch + ch];
   }
   else {
      const float *p = a.coef + (a.nch ? (long long) ch * a.S * 5 : 0) + s * 5;
      for (int k = 0; k < 5; k++) c.k[k] = p[k];
   }
   return c;
}

// ------------------------------------------------------------ sequential

template <int FORM> __global__ void __launch_bounds__(128) biquad_seq_kernel(BiquadLaunch a)
{
   const int ch = blockIdx.x * blockDim.x + threadIdx.x;
   if (ch >= a.C) return;
   constexpr int nv = FORM == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   for (int s = 0; s < a.S; s++) {
      const Coef cf = loadCoef(a, s, ch);
      float *st = a.state + (long long) (s * nv) * a.varPitch + ch;
      const float *in = s == 0 ? a.x + ch : a.y + ch;
      const long long ip = s == 0 ? a.inPitch : a.outPitch;
      float *out = a.y + ch;
      if (FORM == DSPLIB_BIQUAD_DF2) {
         const float b0 = cf.k[0], b1 = cf.k[1], b2 = cf.k[2], a1 = cf.k[3], a2 = cf.k[4];
         float w1 = st[0], w2 = st[a.varPitch];
         for (int t = 0; t < a.N; t++) {
            const float x = in[t * ip];
            const float w0 = __fsub_rn(__fsub_rn(x, __fmul_rn(a1, w1)), __fmul_rn(a2, w2));
            const float y = __fadd_rn(__fadd_rn(__fmul_rn(b0, w0), __fmul_rn(b1, w1)), __fmul_rn(b2, w2));
            w2 = w1;
            w1 = w0;
            out[t * a.outPitch] = y;
         }
         st[0] = w1;
         st[a.varPitch] = w2;
      }
      else if (FORM == DSPLIB_BIQUAD_DF1) {
         const float b0 = cf.k[0], b1 = cf.k[1], b2 = cf.k[2], a1 = cf.k[3], a2 = cf.k[4];
         float xd1 = st[0], xd2 = st[a.varPitch], yd1 = st[2 * a.varPitch], yd2 = st[3 * a.varPitch];
         for (int t = 0; t < a.N; t++) {
            const float x = in[t * ip];
            float y = __fadd_rn(__fmul_rn(b0, x), __fmul_rn(b1, xd1));
            y = __fadd_rn(y, __fmul_rn(b2, xd2));
            y = __fsub_rn(y, __fmul_rn(a1, yd1));
            y = __fsub_rn(y, __fmul_rn(a2, yd2));
            xd2 = xd1;
            xd1 = x;
            yd2 = yd1;
            yd1 = y;
            out[t * a.outPitch] = y;
         }
         st[0] = xd1;
         st[a.varPitch] = xd2;
         st[2 * a.varPitch] = yd1;
         st[3 * a.varPitch] = yd2;
      }
      else if (FORM == DSPLIB_BIQUAD_TDF2) {
         const float b0 = cf.k[0], b1 = cf.k[1], b2 = cf.k[2], a1 = cf.k[3], a2 = cf.k[4];
         float w1 = st[0], w2 = st[a.varPitch];
         for (int t = 0; t < a.N; t++) {
            const float x = in[t * ip];
            const float y = __fadd_rn(w1, __fmul_rn(x, b0));
            w1 = __fsub_rn(__fadd_rn(w2, __fmul_rn(x, b1)), __fmul_rn(a1, y));
            w2 = __fsub_rn(__fmul_rn(x, b2), __fmul_rn(a2, y));
            out[t * a.outPitch] = y;
         }
         st[0] = w1;
         st[a.varPitch] = w2;
      }
      else { // TIF, optimized layout
         const float c0 = cf.k[0], c1 = cf.k[1], a12 = cf.k[2], a11 = cf.k[3], gain = cf.k[4];
         float d0 = st[0], d1 = st[a.varPitch];
         for (int t = 0; t < a.N; t++) {
            const float x = in[t * ip];
            const float o = __fadd_rn(x, d0);
            const float t1 = __fadd_rn(__fmul_rn(x, c0), d1);
            const float t0 = __fmul_rn(a12, d0);
            d0 = __fadd_rn(__fmul_rn(a11, d0), t1);
            d1 = __fadd_rn(__fmul_rn(c1, x), t0);
            out[t * a.outPitch] = __fmul_rn(o, gain);
         }
         st[0] = d0;
         st[a.varPitch] = d1;
      }
   }
}

// ------------------------------------------------------------ scan

// 2x2 matrix [[a, b], [c, d]] in FP64.
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

// One-sample state transition (zero input) in the scan's state coordinates.
//   DF2  (w1, w2):  w1' = -a1 w1 - a2 w2,  w2' = w1
//   TDF2 (w1, w2):  y = w1,  w1' = w2 - a1 y,  w2' = -a2 y.  DF1 is run in
//        this transposed realization of the same section: its minimal state.
//   TIF  (d0, d1):  d0' = a11 d0 + d1,  d1' = a12 d0
template <int FORM> __device__ __forceinline__ M2 transition(const Coef &c)
{
   if (FORM == DSPLIB_BIQUAD_DF2) return {-(double) c.k[3], -(double) c.k[4], 1.0, 0.0};
   if (FORM == DSPLIB_BIQUAD_TIF) return {(double) c.k[3], 1.0, (double) c.k[2], 0.0};
   return {-(double) c.k[3], 1.0, -(double) c.k[4], 0.0};
}

// The stage recursion over v[0..len) from state st (FP32, fused multiply-add).
// WRITE = false computes only the end state.  DF1 uses the TDF2 recursion.
// For DF1 the last two stage inputs and outputs are kept for the final state.
// Each recursion is arranged so that one fused multiply-add per sample lies
// on the loop-carried dependency chain (the older state enters the inner term).
// FULL = true: len == L, no per-sample predicate.
template <int FORM, int L, bool WRITE, bool FULL>
__device__ __forceinline__ void runChunk(float (&v)[L], int len, const Coef &c, float2 &st, float4 *tail)
{
   if (FORM == DSPLIB_BIQUAD_DF2) {
      const float b0 = c.k[0], b1 = c.k[1], b2 = c.k[2], a1 = c.k[3], a2 = c.k[4];
      float w1 = st.x, w2 = st.y;
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (FULL || i < len) {
            const float w0 = fmaf(-a1, w1, fmaf(-a2, w2, v[i]));
            if (WRITE) v[i] = fmaf(b0, w0, fmaf(b1, w1, b2 * w2));
            w2 = w1;
            w1 = w0;
         }
      }
      st = make_float2(w1, w2);
   }
   else if (FORM == DSPLIB_BIQUAD_TIF) {
      const float c0 = c.k[0], c1 = c.k[1], a12 = c.k[2], a11 = c.k[3];
      float d0 = st.x, d1 = st.y;
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (FULL || i < len) {
            const float x = v[i];
            const float o = x + d0;
            const float nd0 = fmaf(a11, d0, fmaf(x, c0, d1));
            d1 = fmaf(c1, x, a12 * d0);
            d0 = nd0;
            if (WRITE) v[i] = o;
         }
      }
      st = make_float2(d0, d1);
   }
   else {
      // TDF2: y = b0 x + w1; w1' = w2 + b1 x - a1 y; w2' = b2 x - a2 y, with y
      // substituted so that w1' = -a1 w1 + (w2 + (b1 - a1 b0) x).
      const float b0 = c.k[0], a1 = c.k[3], a2 = c.k[4];
      const float c1 = (float) ((double) c.k[1] - (double) a1 * b0);
      const float c2 = (float) ((double) c.k[2] - (double) a2 * b0);
      float w1 = st.x, w2 = st.y;
      float u1 = 0.f, u2 = 0.f, y1 = 0.f, y2 = 0.f;
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (FULL || i < len) {
            const float x = v[i];
            if (WRITE) {
               const float y = fmaf(x, b0, w1);
               v[i] = y;
               if (FORM == DSPLIB_BIQUAD_DF1) {
                  u2 = u1;
                  u1 = x;
                  y2 = y1;
                  y1 = y;
               }
            }
            const float w1n = fmaf(-a1, w1, fmaf(x, c1, w2));
            w2 = fmaf(-a2, w1, x * c2);
            w1 = w1n;
         }
      }
      st = make_float2(w1, w2);
      if (FORM == DSPLIB_BIQUAD_DF1 && WRITE) *tail = make_float4(u1, u2, y1, y2);
   }
}

template <int FORM, int L, bool WRITE>
__device__ __forceinline__ void runChunkAny(float (&v)[L], int len, const Coef &c, float2 &st, float4 *tail)
{
   if (len == L) runChunk<FORM, L, WRITE, true>(v, len, c, st, tail);
   else runChunk<FORM, L, WRITE, false>(v, len, c, st, tail);
}

constexpr int kScanL = 32;      // samples per chunk
constexpr int kPad = 33;        // row pitch (double2) of the chunk x channel tables
constexpr int kMaxCluster = 16; // CTAs per cluster
constexpr int kPowTableBytes = 64 * 1024;

__host__ __device__ constexpr int ilog2c(int x) { return x <= 1 ? 0 : 1 + ilog2c(x / 2); }

// FP32 2x2 matrices and affine maps of the lane scan kernel.  Its matrix powers are
// formed in FP64 and rounded once; the scans themselves run in FP32: chunk transitions
// of stable sections contract, so their rounding stays at the level of the sequential
// FP32 recursion while the dependent chains are several times shorter than in FP64.
struct M2f {
   float a, b, c, d;
};

__device__ __forceinline__ float2 affinef(const M2f &m, float2 v, float2 e)
{
   return make_float2(fmaf(m.a, v.x, fmaf(m.b, v.y, e.x)), fmaf(m.c, v.x, fmaf(m.d, v.y, e.y)));
}

// Matrix powers kept per stage and channel: M^(2^k), M = A^L, for
// k = 0 .. log2(W) (the last one is the CTA span A^(W*L)).
template <int W> struct ScanShape {
   static constexpr int LOGW = ilog2c(W);
   static constexpr int NP = LOGW + 1;
};

struct ScanSmem {
   size_t E, Mine, Win, Pow, Cf, Next, total;
   bool powTable;
};

template <int W> __host__ __device__ inline ScanSmem scanLayout(int S)
{
   ScanSmem o;
   size_t off = 0;
   o.E = off;
   off += (size_t) W * kPad * sizeof(float2);
   o.Mine = off;
   off += (size_t) 32 * sizeof(float2);
   o.Win = off;
   off += (size_t) S * 32 * sizeof(float2);
   const size_t pow = (size_t) S * 32 * ScanShape<W>::NP * sizeof(M2f);
   o.powTable = pow <= (size_t) kPowTableBytes;
   o.Pow = off; // all stages' powers, or two buffers of one stage's (recomputed per stage) when too large
   off += o.powTable ? pow : (size_t) 2 * 32 * ScanShape<W>::NP * sizeof(M2f);
   o.Cf = off;
   off += (size_t) S * 32 * 5 * sizeof(float);
   o.Next = (off + 15) / 16 * 16; // next window's input, fetched during this one (prefetch launches)
   o.total = o.Next;
   return o;
}

// Shared memory of a scan launch: the tables, plus the next-window buffer when the
// input is device memory and spans more than one window, plus (clusters) the
// exchange buffer: two phases of every CTA's 32 chunk-span aggregates.
template <int W> inline size_t scanSmemBytes(const BiquadLaunch &a, int K)
{
   const ScanSmem lay = scanLayout<W>(a.S);
   const bool next = a.prefetch && (long long) a.N > (long long) K * W * kScanL;
   return lay.total + (next ? (size_t) kScanL * W * 32 * sizeof(float) : 0) +
          (K > 1 ? (size_t) 2 * K * 32 * sizeof(float2) : 0);
}

__device__ __forceinline__ void cpAsync4(float *dst, const float *src)
{
   const unsigned d = (unsigned) __cvta_generic_to_shared(dst);
   asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}

// Writes M^(2^k), k = 0 .. NP-1, of M = A^L to out[] (formed in FP64, rounded once).
template <int FORM, int W> __device__ __forceinline__ void stagePowersF(const Coef &c, M2f *out)
{
   M2 P = transition<FORM>(c);
#pragma unroll
   for (int r = 1; r < kScanL; r <<= 1) P = mmul(P, P);
   out[0] = {(float) P.a, (float) P.b, (float) P.c, (float) P.d};
#pragma unroll
   for (int k = 1; k < ScanShape<W>::NP; k++) {
      P = mmul(P, P);
      out[k] = {(float) P.a, (float) P.b, (float) P.c, (float) P.d};
   }
}

// Horner's rule acc <- M acc + e_i over i = 0 .. n-1 (n <= MAXN), e_i = src[i * stride].
// The loads are issued eight at a time ahead of the dependent multiply-adds, so the chain
// costs about one FMA latency pair per step rather than a shared-memory round trip.
template <int MAXN>
__device__ __forceinline__ float2 hornerF(const M2f &M, float2 acc, const float2 *src, int stride, int n)
{
#pragma unroll
   for (int g = 0; g < MAXN; g += 8) {
      if (g >= n) break;
      float2 e[8];
#pragma unroll
      for (int i = 0; i < 8; i++) e[i] = (g + i < n) ? src[(g + i) * stride] : make_float2(0.f, 0.f);
#pragma unroll
      for (int i = 0; i < 8; i++)
         if (g + i < n) acc = affinef(M, acc, e[i]);
   }
   return acc;
}

// M^n v for 0 <= n < 2^nb, with P[k] = M^(2^k).
__device__ __forceinline__ float2 powApplyF(const M2f *P, int n, int nb, float2 v)
{
   const float2 z = make_float2(0.0f, 0.0f);
#pragma unroll
   for (int k = 0; k < 5; k++)
      if (k < nb && ((n >> k) & 1)) v = affinef(P[k], v, z);
   return v;
}

template <int FORM, int W, bool CLUSTER>
__global__ void __launch_bounds__(W * 32, 16 / W) biquad_scan_kernel(BiquadLaunch a)
{
   constexpr int L = kScanL;
   constexpr int nv = FORM == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   constexpr int LOGW = ScanShape<W>::LOGW;
   constexpr int NP = ScanShape<W>::NP;
   extern __shared__ __align__(16) unsigned char smem[];
   const ScanSmem lay = scanLayout<W>(a.S);
   float2 *sE = (float2 *) (smem + lay.E);
   float2 *sMine = (float2 *) (smem + lay.Mine);
   float2 *sWin = (float2 *) (smem + lay.Win);
   M2f *sPow = (M2f *) (smem + lay.Pow);
   float *sCf = (float *) (smem + lay.Cf);
   float *sNext = (float *) (smem + lay.Next);

   const int lane = threadIdx.x & 31;
   const int w = threadIdx.x >> 5;
   const int ch = blockIdx.y * 32 + lane;
   const bool active = ch < a.C;
   int K = 1, rank = 0;
   if (CLUSTER) {
      cg::cluster_group cl = cg::this_cluster();
      K = (int) cl.num_blocks();
      rank = (int) cl.block_rank();
   }
   const long long windowLen = (long long) K * W * L;
   // Device-memory input over several windows: the next window's samples are copied into
   // shared memory (each thread its own slots) while this one is filtered.
   const bool usePrefetch = a.prefetch && a.N > windowLen;
   // [2][K][32]: the aggregates every CTA of the cluster pushed for this phase
   float2 *sAggIn = (float2 *) (smem + lay.Next + (usePrefetch ? (size_t) L * W * 32 * sizeof(float) : 0));

   // First window's input, issued before the table set-up so the loads overlap it.
   long long t0 = ((long long) rank * W + w) * L;
   int len = (active && t0 < a.N) ? (int) ((a.N - t0) < L ? (a.N - t0) : L) : 0;
   float v[L];
   {
      const float *xp = a.x + t0 * a.inPitch + ch;
      if (len == L) {
#pragma unroll
         for (int i = 0; i < L; i++) v[i] = xp[i * a.inPitch];
      }
      else {
#pragma unroll
         for (int i = 0; i < L; i++) v[i] = i < len ? xp[i * a.inPitch] : 0.0f;
      }
   }

   // Coefficients, matrix powers and the initial state (scan coordinates) per stage and channel.
   for (int s = w; s < a.S; s += W) {
      Coef c;
      if (active) c = loadCoef(a, s, ch);
      else
         for (int k = 0; k < 5; k++) c.k[k] = 0.0f;
      for (int k = 0; k < 5; k++) sCf[(s * 32 + lane) * 5 + k] = c.k[k];
      if (lay.powTable) stagePowersF<FORM, W>(c, sPow + (s * 32 + lane) * NP);
      float2 st0 = make_float2(0.0, 0.0);
      if (active) {
         const float *sp = a.state + (long long) (s * nv) * a.varPitch + ch;
         if (FORM == DSPLIB_BIQUAD_DF1) { // DF1 (xd1, xd2, yd1, yd2) -> transposed-form state
            const double xd1 = sp[0], xd2 = sp[a.varPitch], yd1 = sp[2 * a.varPitch], yd2 = sp[3 * a.varPitch];
            st0.x = c.k[1] * xd1 + c.k[2] * xd2 - c.k[3] * yd1 - c.k[4] * yd2;
            st0.y = c.k[2] * xd1 - c.k[4] * yd1;
         }
         else {
            st0 = make_float2(sp[0], sp[a.varPitch]);
         }
      }
      sWin[s * 32 + lane] = st0;
   }
   if (CLUSTER) cg::this_cluster().sync();
   else __syncthreads();

   int phase = 0;
   for (long long win0 = 0; win0 < a.N; win0 += windowLen) {
      if (win0 > 0) {
         t0 = win0 + ((long long) rank * W + w) * L;
         len = (active && t0 < a.N) ? (int) ((a.N - t0) < L ? (a.N - t0) : L) : 0;
         if (usePrefetch) {
            asm volatile("cp.async.wait_all;" ::: "memory");
#pragma unroll
            for (int i = 0; i < L; i++) v[i] = i < len ? sNext[i * (W * 32) + threadIdx.x] : 0.0f;
         }
         else {
            const float *xp = a.x + t0 * a.inPitch + ch;
            if (len == L) {
#pragma unroll
               for (int i = 0; i < L; i++) v[i] = xp[i * a.inPitch];
            }
            else {
#pragma unroll
               for (int i = 0; i < L; i++) v[i] = i < len ? xp[i * a.inPitch] : 0.0f;
            }
         }
      }
      if (usePrefetch && win0 + windowLen < a.N) {
         const long long tn = win0 + windowLen + ((long long) rank * W + w) * L;
         const int ln = (active && tn < a.N) ? (int) ((a.N - tn) < L ? (a.N - tn) : L) : 0;
         const float *xp = a.x + tn * a.inPitch + ch;
#pragma unroll
         for (int i = 0; i < L; i++)
            if (i < ln) cpAsync4(&sNext[i * (W * 32) + threadIdx.x], xp + i * a.inPitch);
         asm volatile("cp.async.commit_group;" ::: "memory");
      }
      for (int s = 0; s < a.S; s++) {
         Coef c;
#pragma unroll
         for (int k = 0; k < 5; k++) c.k[k] = sCf[(s * 32 + lane) * 5 + k];
         // Matrix powers of this stage for channel `lane`: the table, or (deep cascades) this
         // stage's powers formed by warp 0 into the buffer of this iteration's parity.  A buffer
         // is rewritten two iterations later, once every warp has passed the barrier between.
         const M2f *P;
         if (lay.powTable) {
            P = sPow + (s * 32 + lane) * NP;
         }
         else {
            P = sPow + ((phase & 1) * 32 + lane) * NP;
            if (w == 0) stagePowersF<FORM, W>(c, (M2f *) P);
         }
         // 1. zero-state end state of this chunk.  The window's entry state for this stage
         //    is read before the barrier: it is replaced after it.
         float2 e = make_float2(0.f, 0.f);
         runChunkAny<FORM, L, false>(v, len, c, e, nullptr);
         const float2 win = sWin[s * 32 + lane];
         sE[w * kPad + lane] = e;
         __syncthreads();

         // 2. chunk-boundary states, lane = channel, by Horner's rule over the chunks before
         //    this warp's with M = A^L: each warp needs only its own, so warps leave the scan
         //    (and start their reruns) at staggered times.
         const M2f M = P[0];
         float2 st;
         if (CLUSTER && K > 1) {
            float2 *in = sAggIn + (phase & 1) * (K * 32);
            if (w == W - 1) {
               // This CTA's aggregate (the end of its span from a zero entry state) by a
               // pairwise tree over the W chunk end states with P[k] = M^(2^k), pushed as one
               // coalesced 256-byte row into every CTA's exchange buffer.  After the cluster
               // barrier each CTA reads all K rows from its own shared memory.  Writes of phase
               // p + 2 into a row cannot overtake its reads of phase p: those precede this CTA's
               // arrival at the barrier of phase p + 1.
               float2 t[W];
#pragma unroll
               for (int i = 0; i < W; i++) t[i] = sE[i * kPad + lane];
#pragma unroll
               for (int k = 0; k < LOGW; k++) {
                  const M2f Pk = P[k];
#pragma unroll
                  for (int i = 0; i < (W >> (k + 1)); i++) t[i] = affinef(Pk, t[2 * i], t[2 * i + 1]);
               }
               for (int d = 0; d < K; d++) cg::this_cluster().map_shared_rank(in, d)[rank * 32 + lane] = t[0];
            }
            asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
            // the chunks before this warp's, from a zero state at the CTA's start, while the
            // other CTAs' aggregates arrive
            const float2 pre = hornerF<W>(M, make_float2(0.f, 0.f), sE + lane, kPad, w);
            asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
            // 3. entry state of this CTA, formed once by warp 0 and shared: the window entry
            //    carried over the aggregates of the CTAs before it with Mc = A^(W*L); over all
            //    K, the state at the window's end
            if (w == 0) {
               const M2f Mc = P[LOGW];
               const float2 mine = hornerF<kMaxCluster>(Mc, win, in + lane, 32, rank);
               sMine[lane] = mine;
               sWin[s * 32 + lane] = hornerF<kMaxCluster>(Mc, mine, in + rank * 32 + lane, 32, K - rank);
            }
            __syncthreads();
            // true initial state of this chunk: M^w * entry + prefix
            const float2 tv = powApplyF(P, w, LOGW, sMine[lane]);
            st = make_float2(tv.x + pre.x, tv.y + pre.y);
         }
         else {
            const float2 acc = hornerF<W>(M, win, sE + lane, kPad, w);
            st = acc;
            if (w == W - 1) sWin[s * 32 + lane] = affinef(M, acc, e); // state at the window's end
         }

         // 4. rerun from the true state, producing the stage output in place
         float4 tail = make_float4(0.f, 0.f, 0.f, 0.f);
         runChunkAny<FORM, L, true>(v, len, c, st, &tail);
         if (FORM == DSPLIB_BIQUAD_TIF && c.k[4] != 1.0f) {
            const float g = c.k[4];
#pragma unroll
            for (int i = 0; i < L; i++) v[i] *= g;
         }
         float *sp = a.state + (long long) (s * nv) * a.varPitch + ch;
         if (len > 0 && t0 + len == a.N) { // chunk holding the last sample: final state
            if (FORM == DSPLIB_BIQUAD_DF1) {
               // With a single sample the stage's old xd1 / yd1 shift into xd2 / yd2: read
               // them before they are overwritten (no other thread writes this stage's state).
               const float oxd1 = sp[0], oyd1 = sp[2 * a.varPitch];
               sp[0] = tail.x;
               sp[2 * a.varPitch] = tail.z;
               if (len >= 2) {
                  sp[a.varPitch] = tail.y;
                  sp[3 * a.varPitch] = tail.w;
               }
               else if (a.N == 1) {
                  sp[a.varPitch] = oxd1;
                  sp[3 * a.varPitch] = oyd1;
               }
            }
            else {
               sp[0] = st.x;
               sp[a.varPitch] = st.y;
            }
         }
         if (FORM == DSPLIB_BIQUAD_DF1 && len == L && t0 + L == a.N - 1) { // next chunk holds one sample
            sp[a.varPitch] = tail.x;
            sp[3 * a.varPitch] = tail.z;
         }
         phase++;
      }
      {
         float *yp = a.y + t0 * a.outPitch + ch;
         if (len == L) {
#pragma unroll
            for (int i = 0; i < L; i++) yp[i * a.outPitch] = v[i];
         }
         else {
#pragma unroll
            for (int i = 0; i < L; i++)
               if (i < len) yp[i * a.outPitch] = v[i];
         }
      }
   }
   // No remote access follows the last cluster barrier (pushes precede it), so CTAs
   // exit without another one.
}

// ------------------------------------------------------------ per-channel scan
//
// biquad_chan_kernel: for batches of few channels, where lane = channel would
// leave most of the GPU idle, one CTA per channel scans along time instead:
// lane = chunk of 16 samples, 512 chunks per CTA = one 8192-sample window,
// windows in sequence with the state carried.  Per stage: zero-state chunk end
// states, a warp-shuffle scan over 32 chunks (powers M^(2^k) of M = A^16), a
// scan over the 16 warp totals by warp 0 together with the window carry, then
// every chunk reruns from its true initial state.  Each sample is read and
// written once by the thread that owns its chunk (the channel's samples are a
// column of the time-major buffer, so no access pattern coalesces across a
// warp; the other channels of the same rows are read by the other CTAs out of L2).
constexpr int kChL = 16;
constexpr int kChWarps = 16;
constexpr int kChThreads = kChWarps * 32;
constexpr int kChWindow = kChThreads * kChL;
constexpr int kChPowers = 10; // M^(2^k), k = 0..9: M^512 spans a window
constexpr int kChanKernelMaxChannels = 16;
constexpr int kChanTuneMaxChannels = 128; // the autotuner may pick the per-channel kernel up to here
constexpr int kTuneChanKernel = 1;        // the autotuner's choice value for the per-channel kernel

size_t chanSmemBytes(int S) { return (size_t) S * (kChPowers * sizeof(M2) + sizeof(double2) + 5 * sizeof(float)); }

template <int FORM> __global__ void __launch_bounds__(kChThreads, 1) biquad_chan_kernel(BiquadLaunch a)
{
   constexpr int nv = FORM == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   __shared__ double2 sTot[2][kChWarps];
   extern __shared__ __align__(16) unsigned char chsm[];
   M2 *sPow = (M2 *) chsm;                                   // [S][kChPowers]
   double2 *sWin = (double2 *) (sPow + a.S * kChPowers);     // [S] state carried into the window
   float *sCf = (float *) (sWin + a.S);                      // [S][5]
   const int ch = blockIdx.x;
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;

   for (int s = tid; s < a.S; s += kChThreads) {
      const Coef c = loadCoef(a, s, ch);
#pragma unroll
      for (int k = 0; k < 5; k++) sCf[s * 5 + k] = c.k[k];
      M2 P = transition<FORM>(c);
#pragma unroll
      for (int r = 1; r < kChL; r <<= 1) P = mmul(P, P);
      sPow[s * kChPowers] = P;
      for (int k = 1; k < kChPowers; k++) {
         P = mmul(P, P);
         sPow[s * kChPowers + k] = P;
      }
      const float *sp = a.state + (long long) (s * nv) * a.varPitch + ch;
      double2 st0;
      if (FORM == DSPLIB_BIQUAD_DF1) { // DF1 (xd1, xd2, yd1, yd2) -> transposed-form state
         const double xd1 = sp[0], xd2 = sp[a.varPitch], yd1 = sp[2 * a.varPitch], yd2 = sp[3 * a.varPitch];
         st0.x = c.k[1] * xd1 + c.k[2] * xd2 - c.k[3] * yd1 - c.k[4] * yd2;
         st0.y = c.k[2] * xd1 - c.k[4] * yd1;
      }
      else {
         st0 = make_double2(sp[0], sp[a.varPitch]);
      }
      sWin[s] = st0;
   }
   __syncthreads();

   const double2 zero = make_double2(0.0, 0.0);
   int phase = 0;
   for (long long win0 = 0; win0 < a.N; win0 += kChWindow) {
      const long long t0 = win0 + (long long) tid * kChL;
      const int len = t0 < a.N ? (int) ((a.N - t0) < kChL ? (a.N - t0) : kChL) : 0;
      float v[kChL];
      {
         const float *xp = a.x + t0 * a.inPitch + ch;
#pragma unroll
         for (int i = 0; i < kChL; i++) v[i] = i < len ? xp[i * a.inPitch] : 0.0f;
      }
      for (int s = 0; s < a.S; s++, phase++) {
         Coef c;
#pragma unroll
         for (int k = 0; k < 5; k++) c.k[k] = sCf[s * 5 + k];
         const M2 *P = sPow + s * kChPowers;
         double2 *tot = sTot[phase & 1];
         // 1. zero-state end state of this chunk
         float2 e = make_float2(0.f, 0.f);
         runChunkAny<FORM, kChL, false>(v, len, c, e, nullptr);
         // 2. inclusive scan over the warp's 32 chunks
         double2 val = make_double2(e.x, e.y);
#pragma unroll
         for (int k = 0; k < 5; k++) {
            double2 o;
            o.x = __shfl_up_sync(0xffffffffu, val.x, 1 << k);
            o.y = __shfl_up_sync(0xffffffffu, val.y, 1 << k);
            if (lane >= (1 << k)) val = affine(P[k], o, val);
         }
         if (lane == 31) tot[warp] = val;
         __syncthreads();
         // 3. warp 0: entry state of every warp (M^(32 w) carry + totals of the warps before), new carry
         if (warp == 0) {
            double2 tv = lane < kChWarps ? tot[lane] : zero;
#pragma unroll
            for (int k = 0; k < 4; k++) {
               double2 o;
               o.x = __shfl_up_sync(0xffffffffu, tv.x, 1 << k);
               o.y = __shfl_up_sync(0xffffffffu, tv.y, 1 << k);
               if (lane >= (1 << k) && lane < kChWarps) tv = affine(P[5 + k], o, tv);
            }
            const double2 win = sWin[s];
            double2 before, last;
            before.x = __shfl_up_sync(0xffffffffu, tv.x, 1);
            before.y = __shfl_up_sync(0xffffffffu, tv.y, 1);
            last.x = __shfl_sync(0xffffffffu, tv.x, kChWarps - 1);
            last.y = __shfl_sync(0xffffffffu, tv.y, kChWarps - 1);
            if (lane < kChWarps) {
               double2 en = win;
#pragma unroll
               for (int k = 0; k < 4; k++)
                  if ((lane >> k) & 1) en = affine(P[5 + k], en, zero);
               if (lane > 0) en = make_double2(en.x + before.x, en.y + before.y);
               tot[lane] = en;
            }
            if (lane == 0) sWin[s] = affine(P[9], win, last);
         }
         __syncthreads();
         // 4. this chunk's initial state: M^lane entry(warp) + exclusive prefix within the warp
         double2 ex;
         ex.x = __shfl_up_sync(0xffffffffu, val.x, 1);
         ex.y = __shfl_up_sync(0xffffffffu, val.y, 1);
         if (lane == 0) ex = zero;
         double2 stv = tot[warp];
#pragma unroll
         for (int k = 0; k < 5; k++)
            if ((lane >> k) & 1) stv = affine(P[k], stv, zero);
         float2 st = make_float2((float) (stv.x + ex.x), (float) (stv.y + ex.y));
         float4 tail = make_float4(0.f, 0.f, 0.f, 0.f);
         runChunkAny<FORM, kChL, true>(v, len, c, st, &tail);
         if (FORM == DSPLIB_BIQUAD_TIF && c.k[4] != 1.0f) {
            const float g = c.k[4];
#pragma unroll
            for (int i = 0; i < kChL; i++) v[i] *= g;
         }
         float *sp = a.state + (long long) (s * nv) * a.varPitch + ch;
         if (len > 0 && t0 + len == a.N) { // chunk holding the last sample: final state
            if (FORM == DSPLIB_BIQUAD_DF1) {
               const float oxd1 = sp[0], oyd1 = sp[2 * a.varPitch]; // read before overwritten
               sp[0] = tail.x;
               sp[2 * a.varPitch] = tail.z;
               if (len >= 2) {
                  sp[a.varPitch] = tail.y;
                  sp[3 * a.varPitch] = tail.w;
               }
               else if (a.N == 1) {
                  sp[a.varPitch] = oxd1;
                  sp[3 * a.varPitch] = oyd1;
               }
            }
            else {
               sp[0] = st.x;
               sp[a.varPitch] = st.y;
            }
         }
         if (FORM == DSPLIB_BIQUAD_DF1 && len == kChL && t0 + kChL == a.N - 1) { // next chunk holds one sample
            sp[a.varPitch] = tail.x;
            sp[3 * a.varPitch] = tail.z;
         }
      }
      float *yp = a.y + t0 * a.outPitch + ch;
#pragma unroll
      for (int i = 0; i < kChL; i++)
         if (i < len) yp[i * a.outPitch] = v[i];
   }
}

// Largest power-of-two cluster <= want that can be resident (<= 8 portable, 16 opt-in).
template <int FORM, int W> int pickCluster(int want, size_t smemBytes)
{
   static int cached[17] = {0};
   if (want > W) want = W;
   if (want > kMaxCluster) want = kMaxCluster;
   int K = 1;
   while (K * 2 <= want) K *= 2;
   if (K <= 1) return 1;
   if (cached[K]) return cached[K];
   auto fn = biquad_scan_kernel<FORM, W, true>;
   int chosen = 1;
   for (int k = K; k >= 2; k >>= 1) {
      if (k > 8 && cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
         (void) cudaGetLastError();
         continue;
      }
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(k, 1);
      cfg.blockDim = dim3(W * 32);
      cfg.dynamicSmemBytes = smemBytes;
      cudaLaunchAttribute attr;
      attr.id = cudaLaunchAttributeClusterDimension;
      attr.val.clusterDim.x = k;
      attr.val.clusterDim.y = 1;
      attr.val.clusterDim.z = 1;
      cfg.attrs = &attr;
      cfg.numAttrs = 1;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) == cudaSuccess && n >= 1) {
         chosen = k;
         break;
      }
      (void) cudaGetLastError();
   }
   cached[K] = chosen;
   return chosen;
}

template <int FORM, int W> cudaError_t launchScanShape(const BiquadLaunch &a, int want, cudaStream_t s)
{
   const ScanSmem lay = scanLayout<W>(a.S);
   const int groups = (a.C + 31) / 32;
   dim3 block(W * 32);
   cudaError_t e;
   auto fn1 = biquad_scan_kernel<FORM, W, false>;
   auto fnK = biquad_scan_kernel<FORM, W, true>;
   // the largest footprint this launch can take (tables + next-window buffer)
   const size_t maxBytes = lay.total + (a.prefetch ? (size_t) kScanL * W * 32 * sizeof(float) : 0) +
                           (size_t) 2 * kMaxCluster * 32 * sizeof(float2);
   static bool attrSet = false;
   static size_t attrBytes = 0;
   if (!attrSet || attrBytes < maxBytes) {
      if ((e = cudaFuncSetAttribute(fn1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) maxBytes)) != cudaSuccess)
         return e;
      if ((e = cudaFuncSetAttribute(fnK, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) maxBytes)) != cudaSuccess)
         return e;
      attrSet = true;
      attrBytes = maxBytes;
   }
   const int K = want > 1 ? pickCluster<FORM, W>(want, maxBytes) : 1;
   const size_t bytes = scanSmemBytes<W>(a, K);
   dim3 grid(K, groups);
   if (K == 1) {
      fn1<<<grid, block, bytes, s>>>(a);
   }
   else {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = grid;
      cfg.blockDim = block;
      cfg.dynamicSmemBytes = bytes;
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = K;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      if ((e = cudaLaunchKernelEx(&cfg, fnK, a)) != cudaSuccess) return e;
   }
   countLaunch();
   return cudaGetLastError();
}

// Per-channel kernel: one CTA per channel, shared memory for the stage tables.
template <int FORM> cudaError_t launchChanForm(const BiquadLaunch &a, cudaStream_t s)
{
   const size_t smem = chanSmemBytes(a.S);
   if (smem > 48 * 1024) {
      const cudaError_t e =
          cudaFuncSetAttribute(biquad_chan_kernel<FORM>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
      if (e != cudaSuccess) return e;
   }
   biquad_chan_kernel<FORM><<<a.C, kChThreads, smem, s>>>(a);
   countLaunch();
   return cudaGetLastError();
}

// Shape choice, from timings of 1 .. 4096 channels x 8192 samples x 4 stages on B200:
//  * up to 16 channels, lane = channel leaves most lanes idle: one CTA per channel
//    scanning along time;
//  * otherwise 32 channels per CTA (W = 16 warps: one CTA per SM at 128 registers),
//    and time split over a cluster of K CTAs: the largest power of two <= 16 that keeps
//    groups x K <= 128 CTAs resident in one wave; clusters of 16 are only taken while at
//    most 7 of them are needed (no more are co-resident).  Fewer windows per CTA beat
//    more CTAs once a second wave would be needed.
// The autotuner's choice, where it has one for this problem class, replaces the rule:
// 8 or 16 warps per CTA (windows of 256 or 512 samples) and up to 16 CTAs per cluster.
template <int FORM> cudaError_t launchScanForm(const BiquadLaunch &a, cudaStream_t s)
{
   if (a.C <= kChanKernelMaxChannels || a.tuneChoice == kTuneChanKernel) return launchChanForm<FORM>(a, s);
   if (a.tuneChoice > 0) {
      const int W = a.tuneChoice / 100, K = a.tuneChoice % 100;
      if (W == 8 && K >= 1) return launchScanShape<FORM, 8>(a, K, s);
      if (W == 16 && K >= 1) return launchScanShape<FORM, 16>(a, K, s);
   }
   const int groups = (a.C + 31) / 32;
   const long long chunks = (a.N + kScanL - 1) / kScanL;
   int K = 1;
   while (K < 16 && (long long) K * 2 * 16 <= chunks && groups * K * 2 <= 128 && !(K * 2 == 16 && groups > 7))
      K *= 2;
   return launchScanShape<FORM, 16>(a, K, s);
}

template <int FORM> cudaError_t launchSeqForm(const BiquadLaunch &a, cudaStream_t s)
{
   biquad_seq_kernel<FORM><<<(a.C + 127) / 128, 128, 0, s>>>(a);
   countLaunch();
   return cudaGetLastError();
}

} // namespace

cudaError_t launchBiquadSequential(const BiquadLaunch &a, cudaStream_t s)
{
   switch (a.form) {
   case DSPLIB_BIQUAD_DF1: return launchSeqForm<DSPLIB_BIQUAD_DF1>(a, s);
   case DSPLIB_BIQUAD_DF2: return launchSeqForm<DSPLIB_BIQUAD_DF2>(a, s);
   case DSPLIB_BIQUAD_TDF2: return launchSeqForm<DSPLIB_BIQUAD_TDF2>(a, s);
   case DSPLIB_BIQUAD_TIF: return a.optLayout ? launchSeqForm<DSPLIB_BIQUAD_TIF>(a, s) : cudaErrorInvalidValue;
   }
   return cudaErrorInvalidValue;
}

// Deepest cascade whose coefficient and carry tables fit the scan kernel's
// shared memory beside the next-window buffer and the cluster exchange rows
// (28 B per stage and channel: 160 stages take 222 KB of the 227 KB); deeper
// cascades use the sequential kernel.
int biquadScanMaxStages() { return 160; }

std::string biquadTuneKey(const BiquadLaunch &a)
{
   if (!a.optLayout || a.C <= kChanKernelMaxChannels || a.S > biquadScanMaxStages() || a.N <= 0) return std::string();
   char buf[160];
   snprintf(buf, sizeof(buf), "bq_scan|form=%d|S=%d|nch=%d|ch=2^%d|N=2^%d|sms=%d", a.form, a.S, a.nch,
            tuneClass(a.C), tuneClass(a.N), deviceSms());
   return buf;
}

std::vector<int> biquadTuneCandidates(const BiquadLaunch &a)
{
   std::vector<int> c;
   if (biquadTuneKey(a).empty()) return c;
   // a few dozen channels: one CTA per channel along time (more SMs than one cluster) is a candidate
   if (a.C <= kChanTuneMaxChannels) c.push_back(kTuneChanKernel);
   const long long chunks = (a.N + kScanL - 1) / kScanL;
   for (int W : {8, 16})
      for (int K = 1; K <= (W < kMaxCluster ? W : kMaxCluster); K *= 2)
         if (K == 1 || (long long) K * W <= chunks) c.push_back(100 * W + K);
   return c;
}

cudaError_t launchBiquadScan(const BiquadLaunch &a, cudaStream_t s)
{
   if (a.S > biquadScanMaxStages()) return launchBiquadSequential(a, s);
   switch (a.form) {
   case DSPLIB_BIQUAD_DF1: return launchScanForm<DSPLIB_BIQUAD_DF1>(a, s);
   case DSPLIB_BIQUAD_DF2: return launchScanForm<DSPLIB_BIQUAD_DF2>(a, s);
   case DSPLIB_BIQUAD_TDF2: return launchScanForm<DSPLIB_BIQUAD_TDF2>(a, s);
   case DSPLIB_BIQUAD_TIF: return launchScanForm<DSPLIB_BIQUAD_TIF>(a, s);
   }
   return cudaErrorInvalidValue;
}

} // namespace dsplib
