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
//                       2. chunk-boundary states are combined with
//                          M = A^L (A: the stage's one-sample state-transition
//                          matrix) inside the CTA and with Mc = A^(W*L) across
//                          the CTAs of the cluster through distributed shared
//                          memory; A^L and the combination run in FP64;
//                       3. every chunk reruns the recursion from its true
//                          initial state and its outputs become the next
//                          stage's input, kept in registers.
//                     The input is read once and the output written once.
//                     Windows of one cluster run in sequence, carrying the
//                     state across window boundaries.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

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

template <int FORM> struct Form {
   static constexpr int D = FORM == DSPLIB_BIQUAD_DF1 ? 4 : 2;
};

// One-sample state transition (zero input) of each form, as a D x D matrix
// (row-major): state' = A * state.
template <int FORM> __device__ void transition(const Coef &c, double *A)
{
   if (FORM == DSPLIB_BIQUAD_DF2) { // (w1, w2): w1' = -a1 w1 - a2 w2, w2' = w1
      A[0] = -(double) c.k[3];
      A[1] = -(double) c.k[4];
      A[2] = 1.0;
      A[3] = 0.0;
   }
   else if (FORM == DSPLIB_BIQUAD_TDF2) { // (w1, w2): y = w1; w1' = w2 - a1 y; w2' = -a2 y
      A[0] = -(double) c.k[3];
      A[1] = 1.0;
      A[2] = -(double) c.k[4];
      A[3] = 0.0;
   }
   else if (FORM == DSPLIB_BIQUAD_TIF) { // (d0, d1): d0' = a11 d0 + d1; d1' = a12 d0
      A[0] = (double) c.k[3];
      A[1] = 1.0;
      A[2] = (double) c.k[2];
      A[3] = 0.0;
   }
   else { // DF1 (xd1, xd2, yd1, yd2): xd1' = 0, xd2' = xd1, yd1' = b1 xd1 + b2 xd2 - a1 yd1 - a2 yd2, yd2' = yd1
      for (int i = 0; i < 16; i++) A[i] = 0.0;
      A[1 * 4 + 0] = 1.0;
      A[2 * 4 + 0] = (double) c.k[1];
      A[2 * 4 + 1] = (double) c.k[2];
      A[2 * 4 + 2] = -(double) c.k[3];
      A[2 * 4 + 3] = -(double) c.k[4];
      A[3 * 4 + 2] = 1.0;
   }
}

template <int D> __device__ void matSquare(double *M)
{
   double R[D * D];
#pragma unroll
   for (int i = 0; i < D; i++)
#pragma unroll
      for (int j = 0; j < D; j++) {
         double acc = 0.0;
#pragma unroll
         for (int k = 0; k < D; k++) acc = fma(M[i * D + k], M[k * D + j], acc);
         R[i * D + j] = acc;
      }
#pragma unroll
   for (int i = 0; i < D * D; i++) M[i] = R[i];
}

// p = M p + e
template <int D> __device__ __forceinline__ void affine(const double *M, double *p, const double *e)
{
   double r[D];
#pragma unroll
   for (int i = 0; i < D; i++) {
      double acc = e[i];
#pragma unroll
      for (int k = 0; k < D; k++) acc = fma(M[i * D + k], p[k], acc);
      r[i] = acc;
   }
#pragma unroll
   for (int i = 0; i < D; i++) p[i] = r[i];
}

// Run the stage recursion over v[0..len) from state st (FP32, fused
// multiply-add).  WRITE = false computes only the end state.
template <int FORM, int L, bool WRITE>
__device__ __forceinline__ void runChunk(float (&v)[L], int len, const Coef &c, float *st)
{
   if (FORM == DSPLIB_BIQUAD_DF2) {
      const float b0 = c.k[0], b1 = c.k[1], b2 = c.k[2], a1 = c.k[3], a2 = c.k[4];
      float w1 = st[0], w2 = st[1];
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (i < len) {
            const float w0 = fmaf(-a2, w2, fmaf(-a1, w1, v[i]));
            if (WRITE) v[i] = fmaf(b2, w2, fmaf(b1, w1, b0 * w0));
            w2 = w1;
            w1 = w0;
         }
      }
      st[0] = w1;
      st[1] = w2;
   }
   else if (FORM == DSPLIB_BIQUAD_TDF2) {
      const float b0 = c.k[0], b1 = c.k[1], b2 = c.k[2], a1 = c.k[3], a2 = c.k[4];
      float w1 = st[0], w2 = st[1];
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (i < len) {
            const float x = v[i];
            const float y = fmaf(x, b0, w1);
            w1 = fmaf(-a1, y, fmaf(x, b1, w2));
            w2 = fmaf(-a2, y, x * b2);
            if (WRITE) v[i] = y;
         }
      }
      st[0] = w1;
      st[1] = w2;
   }
   else if (FORM == DSPLIB_BIQUAD_TIF) {
      const float c0 = c.k[0], c1 = c.k[1], a12 = c.k[2], a11 = c.k[3];
      float d0 = st[0], d1 = st[1];
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (i < len) {
            const float x = v[i];
            const float o = x + d0;
            const float nd0 = fmaf(a11, d0, fmaf(x, c0, d1));
            d1 = fmaf(c1, x, a12 * d0);
            d0 = nd0;
            if (WRITE) v[i] = o;
         }
      }
      st[0] = d0;
      st[1] = d1;
   }
   else {
      const float b0 = c.k[0], b1 = c.k[1], b2 = c.k[2], a1 = c.k[3], a2 = c.k[4];
      float xd1 = st[0], xd2 = st[1], yd1 = st[2], yd2 = st[3];
#pragma unroll
      for (int i = 0; i < L; i++) {
         if (i < len) {
            const float x = v[i];
            const float y = fmaf(-a2, yd2, fmaf(-a1, yd1, fmaf(b2, xd2, fmaf(b1, xd1, b0 * x))));
            xd2 = xd1;
            xd1 = x;
            yd2 = yd1;
            yd1 = y;
            if (WRITE) v[i] = y;
         }
      }
      st[0] = xd1;
      st[1] = xd2;
      st[2] = yd1;
      st[3] = yd2;
   }
}

constexpr int kScanW = 16; // warps (chunks) per CTA
constexpr int kScanL = 32; // samples per chunk

struct ScanSmem {
   // byte offsets inside dynamic shared memory
   size_t M, Mc, E, Agg, In, Win, Cf, total;
};

__host__ __device__ inline ScanSmem scanLayout(int S, int D)
{
   ScanSmem o;
   size_t off = 0;
   o.M = off;
   off += (size_t) S * 32 * D * D * sizeof(double);
   o.Mc = off;
   off += (size_t) S * 32 * D * D * sizeof(double);
   o.E = off;
   off += (size_t) kScanW * 32 * D * sizeof(double);
   o.Agg = off;
   off += (size_t) 2 * 32 * D * sizeof(double);
   o.In = off;
   off += (size_t) 32 * D * sizeof(double);
   o.Win = off;
   off += (size_t) S * 32 * D * sizeof(double);
   o.Cf = off;
   off += (size_t) S * 32 * 5 * sizeof(float);
   o.total = off;
   return o;
}

template <int FORM, bool CLUSTER>
__global__ void __launch_bounds__(kScanW * 32, 1) biquad_scan_kernel(BiquadLaunch a)
{
   constexpr int D = Form<FORM>::D;
   constexpr int W = kScanW;
   constexpr int L = kScanL;
   constexpr int nv = FORM == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   extern __shared__ __align__(16) unsigned char smem[];
   const ScanSmem lay = scanLayout(a.S, D);
   double *sM = (double *) (smem + lay.M);
   double *sMc = (double *) (smem + lay.Mc);
   double *sE = (double *) (smem + lay.E);
   double *sAgg = (double *) (smem + lay.Agg);
   double *sIn = (double *) (smem + lay.In);
   double *sWin = (double *) (smem + lay.Win);
   float *sCf = (float *) (smem + lay.Cf);

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

   // Per stage and lane: coefficients, M = A^L, Mc = A^(W*L), initial state.
   for (int s = w; s < a.S; s += W) {
      Coef c;
      if (active) c = loadCoef(a, s, ch);
      else
         for (int k = 0; k < 5; k++) c.k[k] = 0.0f;
      for (int k = 0; k < 5; k++) sCf[(s * 32 + lane) * 5 + k] = c.k[k];
      double A[D * D];
      transition<FORM>(c, A);
      for (int r = 1; r < L; r <<= 1) matSquare<D>(A);
      for (int i = 0; i < D * D; i++) sM[(s * 32 + lane) * D * D + i] = A[i];
      for (int r = 1; r < W; r <<= 1) matSquare<D>(A);
      for (int i = 0; i < D * D; i++) sMc[(s * 32 + lane) * D * D + i] = A[i];
      for (int i = 0; i < D; i++)
         sWin[(s * 32 + lane) * D + i] = active ? (double) a.state[(long long) (s * nv + i) * a.varPitch + ch] : 0.0;
   }
   if (CLUSTER) cg::this_cluster().sync();
   else __syncthreads();

   const long long windowLen = (long long) K * W * L;
   int phase = 0;
   for (long long win0 = 0; win0 < a.N; win0 += windowLen) {
      const long long t0 = win0 + ((long long) rank * W + w) * L;
      int len = 0;
      if (active && t0 < a.N) len = (int) ((a.N - t0) < L ? (a.N - t0) : L);
      float v[L];
#pragma unroll
      for (int i = 0; i < L; i++) v[i] = i < len ? a.x[(t0 + i) * a.inPitch + ch] : 0.0f;

      for (int s = 0; s < a.S; s++) {
         Coef c;
#pragma unroll
         for (int k = 0; k < 5; k++) c.k[k] = sCf[(s * 32 + lane) * 5 + k];
         const double *M = sM + (s * 32 + lane) * D * D;
         // 1. zero-state end state of this chunk
         float e[D];
#pragma unroll
         for (int i = 0; i < D; i++) e[i] = 0.0f;
         runChunk<FORM, L, false>(v, len, c, e);
#pragma unroll
         for (int i = 0; i < D; i++) sE[(w * 32 + lane) * D + i] = (double) e[i];
         __syncthreads();
         // 2a. CTA aggregate: state at the end of this CTA's span starting from zero
         double *agg = sAgg + (phase & 1) * 32 * D;
         if (w == W - 1) {
            double p[D];
#pragma unroll
            for (int i = 0; i < D; i++) p[i] = 0.0;
            for (int j = 0; j < W; j++) affine<D>(M, p, sE + (j * 32 + lane) * D);
#pragma unroll
            for (int i = 0; i < D; i++) agg[lane * D + i] = p[i];
         }
         if (CLUSTER) cg::this_cluster().sync();
         else __syncthreads();
         // 2b. combine the cluster's aggregates in order: state entering this
         // CTA, and the state at the end of the window (next window's carry).
         if (w == 0) {
            const double *Mc = sMc + (s * 32 + lane) * D * D;
            double cur[D], mine[D];
#pragma unroll
            for (int i = 0; i < D; i++) cur[i] = sWin[(s * 32 + lane) * D + i];
            for (int q = 0; q < K; q++) {
               if (q == rank)
#pragma unroll
                  for (int i = 0; i < D; i++) mine[i] = cur[i];
               double eq[D];
               if (CLUSTER && q != rank) {
                  const double *remote = cg::this_cluster().map_shared_rank(agg, q);
#pragma unroll
                  for (int i = 0; i < D; i++) eq[i] = remote[lane * D + i];
               }
               else {
#pragma unroll
                  for (int i = 0; i < D; i++) eq[i] = agg[lane * D + i];
               }
               affine<D>(Mc, cur, eq);
            }
#pragma unroll
            for (int i = 0; i < D; i++) {
               sIn[lane * D + i] = mine[i];
               sWin[(s * 32 + lane) * D + i] = cur[i];
            }
         }
         __syncthreads();
         // 2c. this chunk's initial state
         double p[D];
#pragma unroll
         for (int i = 0; i < D; i++) p[i] = sIn[lane * D + i];
         for (int j = 0; j < w; j++) affine<D>(M, p, sE + (j * 32 + lane) * D);
         // 3. rerun from the true state, producing the stage output in place
         float st[D];
#pragma unroll
         for (int i = 0; i < D; i++) st[i] = (float) p[i];
         runChunk<FORM, L, true>(v, len, c, st);
         if (FORM == DSPLIB_BIQUAD_TIF) {
            const float g = c.k[4];
#pragma unroll
            for (int i = 0; i < L; i++) v[i] *= g;
         }
         if (len > 0 && t0 + len == a.N) { // chunk holding the last sample: final state
#pragma unroll
            for (int i = 0; i < D; i++) a.state[(long long) (s * nv + i) * a.varPitch + ch] = st[i];
         }
         phase++;
         __syncthreads();
      }
#pragma unroll
      for (int i = 0; i < L; i++)
         if (i < len) a.y[(t0 + i) * a.outPitch + ch] = v[i];
   }
   // Keep every CTA's shared memory alive until the cluster's last remote read.
   if (CLUSTER) cg::this_cluster().sync();
}

template <int FORM> cudaError_t launchScanForm(const BiquadLaunch &a, cudaStream_t s)
{
   constexpr int D = Form<FORM>::D;
   const ScanSmem lay = scanLayout(a.S, D);
   const long long cta = (long long) kScanW * kScanL;
   int K = (int) ((a.N + cta - 1) / cta);
   if (K > 8) K = 8;
   if (K < 1) K = 1;
   dim3 grid(K, (a.C + 31) / 32);
   dim3 block(kScanW * 32);
   cudaError_t e;
   if (K == 1) {
      auto fn = biquad_scan_kernel<FORM, false>;
      if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) lay.total)) != cudaSuccess)
         return e;
      fn<<<grid, block, lay.total, s>>>(a);
   }
   else {
      auto fn = biquad_scan_kernel<FORM, true>;
      if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) lay.total)) != cudaSuccess)
         return e;
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = grid;
      cfg.blockDim = block;
      cfg.dynamicSmemBytes = lay.total;
      cfg.stream = s;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = K;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      if ((e = cudaLaunchKernelEx(&cfg, fn, a)) != cudaSuccess) return e;
   }
   countLaunch();
   return cudaGetLastError();
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

// Largest stage count whose scan tables fit in shared memory; deeper
// cascades use the sequential kernel.
static int scanMaxStages(int form) { return form == DSPLIB_BIQUAD_DF1 ? 16 : 32; }

cudaError_t launchBiquadScan(const BiquadLaunch &a, cudaStream_t s)
{
   if (a.S > scanMaxStages(a.form)) return launchBiquadSequential(a, s);
   switch (a.form) {
   case DSPLIB_BIQUAD_DF1: return launchScanForm<DSPLIB_BIQUAD_DF1>(a, s);
   case DSPLIB_BIQUAD_DF2: return launchScanForm<DSPLIB_BIQUAD_DF2>(a, s);
   case DSPLIB_BIQUAD_TDF2: return launchScanForm<DSPLIB_BIQUAD_TDF2>(a, s);
   case DSPLIB_BIQUAD_TIF: return launchScanForm<DSPLIB_BIQUAD_TIF>(a, s);
   }
   return cudaErrorInvalidValue;
}

} // namespace dsplib
