// Cascade of direct-form-II biquads of the batched filter bank, forward and
// adjoint, split along time into 512-sample units that warps filter
// independently, with no wait between CTAs and no CTA barrier.
//
// A unit is one warp; each lane owns a chunk of 16 consecutive samples.  Per
// stage the chunk is filtered from a zero state (the only serial pass), the
// chunk end states are combined by a warp scan of the affine maps
// s -> M s + e (M = A^16 and its powers, A the stage's 2x2 companion matrix,
// formed in FP64 and rounded once; the unit's entry state joins the first
// chunk's end state before the scan), and the true output follows without a
// serial chain: w[i] = w_zs[i] + alpha_i w1 + beta_i w2 with (alpha_i, beta_i)
// the first row of A^(i+1) and (w1, w2) the chunk's initial state, then
// y[i] = b0 w[i] + b1 w[i-1] + b2 w[i-2].
//
// Units are chained through the whole cascade at once.  With the state of
// all S stages at a unit's start as one 2S-vector z, the state at its end is
// Phi z + e, where e is the end state when every stage starts the unit from
// zero and Phi = A_c^512, A_c the cascade's 2S x 2S one-step transition (block
// lower-triangular: stage p's output drives stage p + 1).  So:
//   pass 1 (bank_unit_kernel<AGG>): every unit, all stages from a zero state:
//           e, 2 floats per stage;
//   pass 2 (bank_chain_fast_kernel up to 16 stages, bank_chain_kernel beyond):
//           per channel, z_0 = 0, z_{j+1} = Phi z_j + e_j, j over the
//           channel's units (in two levels through Phi^32 over groups of 32
//           units in FP32, or one unit after another in FP64); z_j is stored
//           (2 floats per unit and stage): the checkpoints;
//   pass 3 (bank_unit_kernel<OUT>): every unit again from its checkpoint: y.
// The adjoint is the same cascade run backwards in time with the stages in
// reverse order (v[t] = g[t] - a1 v[t+1] - a2 v[t+2], lambda[t] = b0 v[t] +
// b1 v[t+1] + b2 v[t+2]: g the stage's output gradient, lambda its input
// gradient), chained the same way from the channel's end; its last pass
// (bank_adjoint_kernel) recomputes each unit's forward from the forward
// checkpoints, keeping every stage's internal sequence w_s in shared memory,
// and accumulates the coefficient gradients
//     dL/db_i = sum_t g[t] w[t-i],   dL/da_i = -sum_t lambda[t] w[t-i]
// in FP32 per unit, then in FP64 per channel in a fixed order (bank_coef_kernel):
// bitwise repeatable.
#include <cuda_runtime.h>

#include "dsplib_internal.h"
#include "scan_common.cuh"

namespace dsplib {
namespace {

using scan::M2;
using scan::M2f;

constexpr int kL = 16;          // samples per chunk (lane)
constexpr int kUnit = 32 * kL;  // samples per unit (warp): 512
constexpr int kWarps = 4;       // units per CTA
constexpr int kThreads = 32 * kWarps;
constexpr int kOutPad = kL + 1; // padded shared row per chunk (conflict-free staging)
constexpr int kUnitLog2 = 9;    // Phi = A_c^(2^9)
constexpr int kChainFastStages = 16; // cascades the FP32 register chain takes

static_assert(kUnit == kBankSpan, "unit size");

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

__device__ __forceinline__ float2 shflDown(float2 v, int d)
{
   v.x = __shfl_down_sync(0xffffffffu, v.x, d);
   v.y = __shfl_down_sync(0xffffffffu, v.y, d);
   return v;
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

// ------------------------------------------------------------------ cascade transitions

// Lower block-triangular 2S x 2S matrix in 2x2 blocks (p, q), q <= p, block index
// p (p + 1) / 2 + q, each block 4 doubles row-major.
__host__ __device__ inline int blk(int p, int q) { return p * (p + 1) / 2 + q; }

// Processing position p -> stage: forward p, adjoint S - 1 - p.
__device__ __forceinline__ int stageAt(int p, int S, bool adj) { return adj ? S - 1 - p : p; }

// Phi = A_c^512 for one channel and direction, one CTA: A_c in shared memory, nine
// squarings C(p,q) = sum_{m=q..p} B(p,m) B(m,q) between two shared buffers; then
// Phi^32.  Per channel: Phi forward, Phi adjoint, Phi^32 forward, Phi^32 adjoint.
__global__ void __launch_bounds__(128) bank_transition_kernel(const RaggedChan *chans, const float *coefs,
                                                              double *phi)
{
   extern __shared__ double dynT[];
   const RaggedChan c = chans[blockIdx.x];
   const bool adj = blockIdx.y != 0;
   const int S = c.S;
   if (S == 0) return;
   const int nb = S * (S + 1) / 2;
   double *B = dynT, *C = dynT + 4 * nb;
   const float *cf = coefs + c.cOff;
   for (int b = threadIdx.x; b < nb; b += blockDim.x) {
      int p = 0;
      while (blk(p + 1, 0) <= b) p++;
      const int q = b - blk(p, 0);
      const int sp = stageAt(p, S, adj);
      double *o = B + 4 * b;
      if (q == p) {
         o[0] = -(double) cf[5 * sp + 3];
         o[1] = -(double) cf[5 * sp + 4];
         o[2] = 1.0;
         o[3] = 0.0;
      }
      else {
         // stage q's state reaches stage p's input through the direct terms b0 of the stages between
         const int sq = stageAt(q, S, adj);
         const double b0 = cf[5 * sq], b1 = cf[5 * sq + 1], b2 = cf[5 * sq + 2];
         double d0 = b1 - b0 * (double) cf[5 * sq + 3], d1 = b2 - b0 * (double) cf[5 * sq + 4];
         for (int m = q + 1; m < p; m++) {
            const double g = cf[5 * stageAt(m, S, adj)];
            d0 *= g;
            d1 *= g;
         }
         o[0] = d0;
         o[1] = d1;
         o[2] = 0.0;
         o[3] = 0.0;
      }
   }
   __syncthreads();
   for (int it = 0; it < kUnitLog2; it++) {
      for (int b = threadIdx.x; b < nb; b += blockDim.x) {
         int p = 0;
         while (blk(p + 1, 0) <= b) p++;
         const int q = b - blk(p, 0);
         double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
         for (int m = q; m <= p; m++) {
            const double *x = B + 4 * blk(p, m), *y = B + 4 * blk(m, q);
            r0 = fma(x[0], y[0], fma(x[1], y[2], r0));
            r1 = fma(x[0], y[1], fma(x[1], y[3], r1));
            r2 = fma(x[2], y[0], fma(x[3], y[2], r2));
            r3 = fma(x[2], y[1], fma(x[3], y[3], r3));
         }
         double *o = C + 4 * b;
         o[0] = r0;
         o[1] = r1;
         o[2] = r2;
         o[3] = r3;
      }
      __syncthreads();
      double *t = B;
      B = C;
      C = t;
   }
   double *dst = phi + c.phiOff + (adj ? 4LL * nb : 0);
   for (int i = threadIdx.x; i < 4 * nb; i += blockDim.x) dst[i] = B[i];
   // five more squarings: Phi^32, the transition over a group of 32 units
   for (int it = 0; it < 5; it++) {
      for (int b = threadIdx.x; b < nb; b += blockDim.x) {
         int p = 0;
         while (blk(p + 1, 0) <= b) p++;
         const int q = b - blk(p, 0);
         double r0 = 0.0, r1 = 0.0, r2 = 0.0, r3 = 0.0;
         for (int m = q; m <= p; m++) {
            const double *x = B + 4 * blk(p, m), *y = B + 4 * blk(m, q);
            r0 = fma(x[0], y[0], fma(x[1], y[2], r0));
            r1 = fma(x[0], y[1], fma(x[1], y[3], r1));
            r2 = fma(x[2], y[0], fma(x[3], y[2], r2));
            r3 = fma(x[2], y[1], fma(x[3], y[3], r3));
         }
         double *o = C + 4 * b;
         o[0] = r0;
         o[1] = r1;
         o[2] = r2;
         o[3] = r3;
      }
      __syncthreads();
      double *t = B;
      B = C;
      C = t;
   }
   dst = phi + c.phiOff + 8LL * nb + (adj ? 4LL * nb : 0);
   for (int i = threadIdx.x; i < 4 * nb; i += blockDim.x) dst[i] = B[i];
}

// Per channel (one warp): z_0 = 0, checkpoint z_j, z_{j+1} = Phi z_j + e_j over the
// channel's units (adjoint: from the last unit back).  z in FP64; cascades of more than
// 16 stages (those of up to 16 take bank_chain_fast_kernel).
__global__ void __launch_bounds__(32) bank_chain_kernel(const RaggedChan *chans, const int *order, const double *phi,
                                                        const float2 *agg, float2 *ckpt, int adj)
{
   extern __shared__ double dynC[];
   const RaggedChan c = chans[order[blockIdx.x]];
   const int S = c.S, lane = threadIdx.x;
   if (S <= kChainFastStages) return; // bank_chain_fast_kernel
   const int nb = S * (S + 1) / 2, n2 = 2 * S;
   double *P = dynC, *z = dynC + 4 * nb;
   const double *src = phi + c.phiOff + (adj ? 4LL * nb : 0);
   for (int i = lane; i < 4 * nb; i += 32) P[i] = src[i];
   for (int r = lane; r < n2; r += 32) z[r] = 0.0;
   __syncwarp();
   const int units = (c.Lu + kUnit - 1) / kUnit;
   for (int k = 0; k < units; k++) {
      const int j = adj ? units - 1 - k : k;
      const long long base = c.ckOff + (long long) j * S;
      for (int p = lane; p < S; p += 32) ckpt[base + p] = make_float2((float) z[2 * p], (float) z[2 * p + 1]);
      if (k + 1 == units) break;
      double nz[4];
      for (int i = 0; i < 4; i++) {
         const int r = lane + 32 * i;
         if (r >= n2) break;
         const int p = r >> 1, row = r & 1;
         const float2 e = agg[base + p];
         double acc0 = row ? e.y : e.x, acc1 = 0.0;
         for (int q = 0; q <= p; q++) {
            const double *x = P + 4 * blk(p, q) + 2 * row;
            acc0 = fma(x[0], z[2 * q], acc0);
            acc1 = fma(x[1], z[2 * q + 1], acc1);
         }
         nz[i] = acc0 + acc1;
      }
      __syncwarp();
      for (int i = 0; i < 4; i++) {
         const int r = lane + 32 * i;
         if (r < n2) z[r] = nz[i];
      }
      __syncwarp();
   }
}

// The same chain for cascades of up to 16 stages (2S <= 32), in FP32 (the transitions
// rounded once from their FP64 products), in two levels so that its depth is about
// 2 x 32 + units / 32 steps instead of one step per unit: each warp of the CTA runs
// groups of 32 units from a zero state (group aggregates), warp 0 chains the groups
// with Phi^32, then every group runs again from its true start and writes the
// checkpoints.  In a step, lane r holds state component r and row r of the
// transition in registers; z is broadcast by shuffles.  Group states sit in shared
// memory for channels of up to 48 groups, in the caller's buffer beyond.
constexpr int kChainWarps = 8;
constexpr int kChainGroup = 32;
constexpr int kChainSharedGroups = 48;

// Row r of a transition (lane r's) at rows[r * kRowPad + k], zero beyond n2 and above the
// block diagonal: in shared memory rather than registers, which keeps the kernel's register
// count low enough for four CTAs per SM (the rows are read conflict-free: lane r, column q
// sits in bank (r + q) mod 32).
constexpr int kRowPad = 2 * kChainFastStages + 1;
__device__ __forceinline__ void loadRows(float *rows, const double *P, int n2, int tid, int nthreads)
{
   constexpr int n = 2 * kChainFastStages * kRowPad;
   for (int i0 = tid; i0 < n; i0 += 4 * nthreads) { // four loads in flight per thread
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; u++) {
         const int i = i0 + u * nthreads, r = i / kRowPad, k = i % kRowPad;
         const int p = r >> 1, q = k >> 1;
         v[u] = (i < n && r < n2 && k < n2 && q <= p) ? (float) P[4 * blk(p, q) + 2 * (r & 1) + (k & 1)] : 0.0f;
      }
#pragma unroll
      for (int u = 0; u < 4; u++)
         if (i0 + u * nthreads < n) rows[i0 + u * nthreads] = v[u];
   }
}

// z' = row . z + e (lane r: component r), z broadcast from lanes 0 .. n2 - 1.
__device__ __forceinline__ float chainStep(const float *row, float z, float e, int n2)
{
   float a0 = e, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
#pragma unroll
   for (int q = 0; q < 2 * kChainFastStages; q += 4) {
      if (q >= n2) break;
      a0 = fmaf(row[q], __shfl_sync(0xffffffffu, z, q), a0);
      a1 = fmaf(row[q + 1], __shfl_sync(0xffffffffu, z, q + 1), a1);
      a2 = fmaf(row[q + 2], __shfl_sync(0xffffffffu, z, q + 2), a2);
      a3 = fmaf(row[q + 3], __shfl_sync(0xffffffffu, z, q + 3), a3);
   }
   return (a0 + a1) + (a2 + a3);
}

__global__ void __launch_bounds__(kChainWarps * 32) bank_chain_fast_kernel(const RaggedChan *chans, const int *order,
                                                                           const double *phi, const float2 *agg,
                                                                           float2 *ckpt, float *groupBuf, int adj)
{
   __shared__ float sE[kChainWarps][kChainGroup * 2 * kChainFastStages]; // a group's aggregates, per warp
   __shared__ float sG[kChainSharedGroups * 2 * kChainFastStages];       // group states
   __shared__ float sRow[2][2 * kChainFastStages * kRowPad];             // Phi and Phi^32
   const RaggedChan c = chans[order[blockIdx.x]];
   const int S = c.S, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   if (S == 0 || S > kChainFastStages) return;
   const int n2 = 2 * S, nb = S * (S + 1) / 2;
   const int units = (c.Lu + kUnit - 1) / kUnit, groups = (units + kChainGroup - 1) / kChainGroup;
   float *G = groups <= kChainSharedGroups ? sG : groupBuf + c.grpOff;
   const float *ag = (const float *) (agg + c.ckOff);
   float *ck = (float *) (ckpt + c.ckOff);
   // unit of step k of group g (processing order), and that group's units in memory order
   auto unitOf = [&](int g, int k) { return adj ? units - 1 - (g * kChainGroup + k) : g * kChainGroup + k; };
   auto stageGroup = [&](int g, int gn) {
      const int j0 = adj ? units - g * kChainGroup - gn : g * kChainGroup;
      const float *src = ag + (long long) j0 * n2;
      const int n = gn * n2;
      __syncwarp();
      for (int q0 = lane; q0 < n; q0 += 4 * 32) { // four loads in flight per lane
         float r[4];
#pragma unroll
         for (int u = 0; u < 4; u++)
            if (q0 + 32 * u < n) r[u] = src[q0 + 32 * u];
#pragma unroll
         for (int u = 0; u < 4; u++)
            if (q0 + 32 * u < n) sE[warp][q0 + 32 * u] = r[u];
      }
      __syncwarp();
      return j0;
   };
   loadRows(sRow[0], phi + c.phiOff + (adj ? 4LL * nb : 0), n2, threadIdx.x, blockDim.x);
   loadRows(sRow[1], phi + c.phiOff + 8LL * nb + (adj ? 4LL * nb : 0), n2, threadIdx.x, blockDim.x);
   __syncthreads();
   const float *row = sRow[0] + lane * kRowPad;
   // 1. group aggregates from a zero state (the last group's is not needed)
   for (int g = warp; g + 1 < groups; g += kChainWarps) {
      const int j0 = stageGroup(g, kChainGroup);
      float z = 0.0f;
      for (int k = 0; k < kChainGroup; k++)
         z = chainStep(row, z, lane < n2 ? sE[warp][(unitOf(g, k) - j0) * n2 + lane] : 0.0f, n2);
      if (lane < n2) G[g * n2 + lane] = z;
   }
   __syncthreads();
   // 2. true group starts: Z_0 = 0, Z_{g+1} = Phi^32 Z_g + E_g
   if (warp == 0) {
      const float *rowQ = sRow[1] + lane * kRowPad;
      float Z = 0.0f;
      for (int g = 0; g < groups; g++) {
         const float E = (lane < n2 && g + 1 < groups) ? G[g * n2 + lane] : 0.0f;
         __syncwarp();
         if (lane < n2) G[g * n2 + lane] = Z;
         if (g + 1 < groups) Z = chainStep(rowQ, Z, E, n2);
      }
   }
   __syncthreads();
   // 3. every group from its true start: the checkpoints
   for (int g = warp; g < groups; g += kChainWarps) {
      const int gn = min(kChainGroup, units - g * kChainGroup);
      const int j0 = stageGroup(g, gn);
      float z = lane < n2 ? G[g * n2 + lane] : 0.0f;
      for (int k = 0; k < gn; k++) {
         const int j = unitOf(g, k);
         if (lane < n2) ck[(long long) j * n2 + lane] = z;
         if (k + 1 < gn) z = chainStep(row, z, lane < n2 ? sE[warp][(j - j0) * n2 + lane] : 0.0f, n2);
      }
   }
}

// ------------------------------------------------------------------ unit passes

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

// The chunk of an unaligned packed row (x, y, gradients), through the warp's staging
// area so that every access of the warp covers 32 consecutive samples.  fetchPacked
// issues the unit's coalesced loads (sample t0 + lane + 32 j in r[j]); stagePacked turns
// them into the lane's chunk, so that a kernel can put other work between the two.
__device__ __forceinline__ void fetchPacked(float (&r)[kL], const float *row, int t0, int n, int lane)
{
#pragma unroll
   for (int j = 0; j < kL; j++) {
      const int k = lane + 32 * j;
      r[j] = t0 + k < n ? row[t0 + k] : 0.0f;
   }
}
__device__ __forceinline__ void stagePacked(float (&v)[kL], const float (&r)[kL], float *stage, int lane)
{
#pragma unroll
   for (int j = 0; j < kL; j++) {
      const int k = lane + 32 * j;
      stage[(k >> 4) * kOutPad + (k & 15)] = r[j];
   }
   __syncwarp();
#pragma unroll
   for (int i = 0; i < kL; i++) v[i] = stage[lane * kOutPad + i];
   __syncwarp();
}

__device__ __forceinline__ void storePacked(const float (&v)[kL], float *row, int t0, int n, float *stage, int lane)
{
#pragma unroll
   for (int i = 0; i < kL; i++) stage[lane * kOutPad + i] = v[i];
   __syncwarp();
   for (int k = lane; k < kUnit && t0 + k < n; k += 32) row[t0 + k] = stage[(k >> 4) * kOutPad + (k & 15)];
   __syncwarp();
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

// The same in reverse time: v[i] = g[i] - a1 v[i+1] - a2 v[i+2]; end state (v[0], v[1]).
__device__ __forceinline__ float2 zeroStatePassRev(const float (&g)[kL], float (&v)[kL], float a1, float a2)
{
   float p1 = 0.0f, p2 = 0.0f;
#pragma unroll
   for (int i = kL - 1; i >= 0; i--) {
      v[i] = fmaf(-a1, p1, fmaf(-a2, p2, g[i]));
      p2 = p1;
      p1 = v[i];
   }
   return make_float2(v[0], v[1]);
}

// Initial state of this lane's chunk, forward time: M^lane entry + the scan of the lanes
// before.  The first chunk's end state takes the unit's entry (M entry + its zero-state end)
// before the scan, which then carries it to every lane with the chunks' own contributions.
// Returns the inclusive scan in *incl (the unit's aggregate in the last lane when ZERO_ENTRY).
template <bool ZERO_ENTRY = false>
__device__ __forceinline__ float2 chunkStateUp(float2 end, float2 entry, const float *tb, int lane, float2 *incl)
{
   float2 val = end;
   if (!ZERO_ENTRY && lane == 0) val = scan::affine(tabP(tb, 0), entry, val);
#pragma unroll
   for (int k = 0; k < 5; k++) {
      const float2 o = scan::shflUp(val, 1 << k, 32);
      if (lane >= (1 << k)) val = scan::affine(tabP(tb, k), o, val);
   }
   float2 ex = scan::shflUp(val, 1, 32);
   if (lane == 0) ex = ZERO_ENTRY ? make_float2(0.0f, 0.0f) : entry;
   *incl = val;
   return ex;
}

// Reverse time: M^(31 - lane) entry + the scan of the lanes after (lane 31 holds the chunk
// processed first).
template <bool ZERO_ENTRY = false>
__device__ __forceinline__ float2 chunkStateDown(float2 end, float2 entry, const float *tb, int lane, float2 *incl)
{
   float2 val = end;
   if (!ZERO_ENTRY && lane == 31) val = scan::affine(tabP(tb, 0), entry, val);
#pragma unroll
   for (int k = 0; k < 5; k++) {
      const float2 o = shflDown(val, 1 << k);
      if (lane + (1 << k) < 32) val = scan::affine(tabP(tb, k), o, val);
   }
   float2 ex = shflDown(val, 1);
   if (lane == 31) ex = ZERO_ENTRY ? make_float2(0.0f, 0.0f) : entry;
   *incl = val;
   return ex;
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

// Reverse time, from (v[16], v[17]): lambda[i] = b0 v[i] + b1 v[i+1] + b2 v[i+2].
__device__ __forceinline__ void correctAndOutputRev(float (&v)[kL], float (&lam)[kL], const float *tb, float v16,
                                                    float v17)
{
   const float b0 = tb[0], b1 = tb[1], b2 = tb[2];
   float n1 = v16, n2 = v17;
#pragma unroll
   for (int i = kL - 1; i >= 0; i--) {
      const float2 ab = *(const float2 *) (tb + kTabAB + 2 * (kL - 1 - i));
      const float vt = fmaf(ab.x, v16, fmaf(ab.y, v17, v[i]));
      lam[i] = fmaf(b0, vt, fmaf(b1, n1, b2 * n2));
      v[i] = vt;
      n2 = n1;
      n1 = vt;
   }
}

// A unit's per-stage states, read once: lane l holds stage l in lo and stage l + 32 in hi
// (up to 64 stages); entryAt broadcasts stage p.
struct UnitStates {
   float2 lo, hi;
};
__device__ __forceinline__ UnitStates loadStates(const float2 *src, int S, int lane)
{
   UnitStates u;
   u.lo = lane < S ? src[lane] : make_float2(0.0f, 0.0f);
   u.hi = lane + 32 < S ? src[lane + 32] : make_float2(0.0f, 0.0f);
   return u;
}
__device__ __forceinline__ float2 entryAt(const UnitStates &u, int p)
{
   return scan::shflIdx(p < 32 ? u.lo : u.hi, p & 31);
}

struct UnitArgs {
   const RaggedChan *chans;
   const int2 *units; // (channel, unit index within the channel)
   int nUnits;
   int Smax;
   const float *tables;
   const float *in;   // forward: FIR output plane; adjoint aggregates: output gradient (packed)
   float *out;        // OUT: y (packed, tail zeros)
   float2 *agg;       // AGG: unit aggregates, 2 floats per stage (processing order)
   const float2 *ckpt;
   // OUT_MSE: loss gradient gy = scale (y - target) on the valid samples, the unit's
   // sum of (y - target)^2 in lossPart[unit], and the adjoint's unit aggregates in aggA
   const float *target;
   float *gy;
   double *lossPart;
   float2 *aggA;
   float scale;
};

// Copy the channel's stage tables into the warp's slice of shared memory, four loads
// per lane in flight before their stores (up to 6 stages in one round).
__device__ __forceinline__ void loadTables(float *dst, const float *tables, const RaggedChan &c, int lane)
{
   const float4 *src = (const float4 *) (tables + (c.cOff / 5) * kBankTabFloats);
   const int n4 = c.S * (kBankTabFloats / 4);
   for (int i0 = lane; i0 < n4; i0 += 4 * 32) {
      float4 r[4];
#pragma unroll
      for (int j = 0; j < 4; j++)
         if (i0 + 32 * j < n4) r[j] = src[i0 + 32 * j];
#pragma unroll
      for (int j = 0; j < 4; j++)
         if (i0 + 32 * j < n4) ((float4 *) dst)[i0 + 32 * j] = r[j];
   }
   __syncwarp();
}

// Forward passes: AGG = from a zero state, write the unit aggregate of every stage;
// OUT = from the checkpoints, write y.  ADJ_AGG: adjoint aggregates over the output
// gradient (reverse time, stages in reverse order).
enum UnitMode { UNIT_AGG = 0, UNIT_OUT = 1, UNIT_ADJ_AGG = 2, UNIT_OUT_MSE = 3 };

// The adjoint's zero-entry pass over a unit (reverse time, stages in reverse order):
// g holds the output gradient on entry, the unit aggregate of every stage goes to agg.
__device__ __forceinline__ void adjointAggregates(float (&g)[kL], const float *sTab, int S, float2 *agg, int lane)
{
   for (int p = 0; p < S; p++) {
      const float *tb = sTab + (S - 1 - p) * kBankTabFloats;
      float w[kL];
      float2 incl;
      const float2 st =
          chunkStateDown<true>(zeroStatePassRev(g, w, tb[3], tb[4]), make_float2(0.0f, 0.0f), tb, lane, &incl);
      correctAndOutputRev(w, g, tb, st.x, st.y);
      if (lane == 0) agg[p] = incl;
   }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads) bank_unit_kernel(UnitArgs a)
{
   extern __shared__ float4 dynU[];
   __shared__ float sStage[kWarps][32 * kOutPad];
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   const int ui = blockIdx.x * kWarps + warp;
   if (ui >= a.nUnits) return;
   float *sTab = (float *) dynU + (size_t) warp * a.Smax * kBankTabFloats;
   const int2 U = a.units[ui];
   const RaggedChan c = a.chans[U.x];
   const int S = c.S, Lu = c.Lu, t0 = U.y * kUnit;
   const long long base = c.ckOff + (long long) U.y * S;
   constexpr bool OUT = MODE == UNIT_OUT || MODE == UNIT_OUT_MSE;
   // the unit's entry states and input are requested before the tables' copy waits on its own loads
   UnitStates ent = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f)};
   if (OUT) ent = loadStates(a.ckpt + base, S, lane);
   float v[kL], tg[kL];
   if (MODE == UNIT_ADJ_AGG) {
      fetchPacked(tg, a.in + c.xOff, t0, Lu, lane);
      loadTables(sTab, a.tables, c, lane);
      stagePacked(v, tg, sStage[warp], lane);
      adjointAggregates(v, sTab, S, a.agg + base, lane);
      return;
   }
   loadChunk(v, a.in + c.pOff, t0 + lane * kL, Lu);
   loadTables(sTab, a.tables, c, lane);
   for (int p = 0; p < S; p++) {
      const float *tb = sTab + p * kBankTabFloats;
      float w[kL];
      const float2 entry = OUT ? entryAt(ent, p) : make_float2(0.0f, 0.0f);
      float2 incl;
      const float2 st = OUT ? chunkStateUp(zeroStatePass(v, w, tb[3], tb[4]), entry, tb, lane, &incl)
                            : chunkStateUp<true>(zeroStatePass(v, w, tb[3], tb[4]), entry, tb, lane, &incl);
      correctAndOutput(w, v, tb, st.x, st.y);
      if (MODE == UNIT_AGG && lane == 31) a.agg[base + p] = incl;
   }
   if (OUT) {
      storePacked(v, a.out + c.xOff, t0, Lu, sStage[warp], lane);
      if (t0 + kUnit >= Lu)
         for (int t = Lu + lane; t < c.L; t += 32) a.out[c.xOff + t] = 0.0f;
   }
   if (MODE == UNIT_OUT_MSE) {
      // the target is read here, not with the unit's other loads: held across the stages
      // it costs 16 registers a thread and the occupancy they buy (measured 1 % slower)
      fetchPacked(tg, a.target + c.xOff, t0, Lu, lane);
      stagePacked(tg, tg, sStage[warp], lane);
      double sq = 0.0;
#pragma unroll
      for (int i = 0; i < kL; i++) {
         const bool valid = t0 + lane * kL + i < Lu;
         const float d = v[i] - tg[i];
         v[i] = valid ? a.scale * d : 0.0f;
         if (valid) sq += (double) d * d;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
      if (lane == 0) a.lossPart[ui] = sq;
      storePacked(v, a.gy + c.xOff, t0, Lu, sStage[warp], lane);
      if (t0 + kUnit >= Lu)
         for (int t = Lu + lane; t < c.L; t += 32) a.gy[c.xOff + t] = 0.0f;
      adjointAggregates(v, sTab, S, a.aggA + base, lane);
   }
}

struct AdjArgs {
   const RaggedChan *chans;
   const int2 *units;
   int nUnits;
   int Smax;
   const float *tables;
   const float *u;       // FIR output plane
   const float *gy;      // output gradient (packed)
   const float2 *ckptF;  // forward checkpoints
   const float2 *ckptA;  // adjoint checkpoints (processing order)
   float *g;             // gradient w.r.t. the FIR output (packed)
   float *part;          // 5 coefficient-gradient sums per unit and stage
   int first;            // this launch's first unit (a bucket of one stage count)
};

// Stage sequences of one unit in shared memory: per stage (the last excepted, which
// stays in registers) 16 rows of 32 lanes, so that the lanes of the warp touch
// distinct banks.  One warp per CTA: the sequences are the bulk of the CTA's
// shared memory, and single-warp CTAs pack the SM most tightly.
__global__ void __launch_bounds__(32) bank_adjoint_kernel(AdjArgs a)
{
   extern __shared__ float4 dynA[];
   const int lane = threadIdx.x;
   float *sTab = (float *) dynA;
   const int2 U = a.units[a.first + blockIdx.x];
   const RaggedChan c = a.chans[U.x];
   float *W = sTab + (size_t) c.S * kBankTabFloats; // the launch sized shared memory for c.S stages
   // The staging rows of the packed gradient loads and stores share the stage sequences'
   // space: the output gradient is read before the sequences are written, the input
   // gradient stored after the last of them was read (at least 32 x 17 floats: adjointShared).
   float *sStage = W;
   const int S = c.S, Lu = c.Lu, t0 = U.y * kUnit;
   const long long base = c.ckOff + (long long) U.y * S;
   const UnitStates entF = loadStates(a.ckptF + base, S, lane), entA = loadStates(a.ckptA + base, S, lane);
   float v[kL], w[kL], g[kL];
   loadChunk(v, a.u + c.pOff, t0 + lane * kL, Lu);
   fetchPacked(w, a.gy + c.xOff, t0, Lu, lane);
   loadTables(sTab, a.tables, c, lane);
   stagePacked(g, w, sStage, lane);
   // 1. the forward of this unit from its checkpoints; every stage's sequence kept
   for (int s = 0; s < S; s++) {
      const float *tb = sTab + s * kBankTabFloats;
      float2 incl;
      const float2 st = chunkStateUp(zeroStatePass(v, w, tb[3], tb[4]), entryAt(entF, s), tb, lane, &incl);
      correctAndOutput(w, v, tb, st.x, st.y);
      if (s + 1 < S) {
         float *Ws = W + s * kL * 32 + lane;
#pragma unroll
         for (int i = 0; i < kL; i++) Ws[i * 32] = w[i];
      }
   }
   // 2. the stages' adjoints, last stage first, in reverse time
   for (int p = 0; p < S; p++) {
      const int s = S - 1 - p;
      const float *tb = sTab + s * kBankTabFloats;
      float vz[kL], lam[kL];
      float2 incl;
      const float2 st = chunkStateDown(zeroStatePassRev(g, vz, tb[3], tb[4]), entryAt(entA, p), tb, lane, &incl);
      correctAndOutputRev(vz, lam, tb, st.x, st.y);
      // forward sequence of this stage: wr[i + 2] = w[i]; w[-1], w[-2] are the previous
      // lane's last two samples (lane 0: the unit's checkpoint state)
      float wr[kL + 2];
      if (p > 0) {
         const float *Ws = W + s * kL * 32 + lane;
#pragma unroll
         for (int i = 0; i < kL; i++) wr[i + 2] = Ws[i * 32];
      }
      else {
#pragma unroll
         for (int i = 0; i < kL; i++) wr[i + 2] = w[i];
      }
      wr[1] = __shfl_up_sync(0xffffffffu, wr[kL + 1], 1);
      wr[0] = __shfl_up_sync(0xffffffffu, wr[kL], 1);
      {
         const float2 e = entryAt(entF, s);
         if (lane == 0) {
            wr[1] = e.x;
            wr[0] = e.y;
         }
      }
      float pr[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
#pragma unroll
      for (int i = 0; i < kL; i++) {
         pr[0] = fmaf(g[i], wr[i + 2], pr[0]);
         pr[1] = fmaf(g[i], wr[i + 1], pr[1]);
         pr[2] = fmaf(g[i], wr[i], pr[2]);
         pr[3] = fmaf(-lam[i], wr[i + 1], pr[3]);
         pr[4] = fmaf(-lam[i], wr[i], pr[4]);
         g[i] = lam[i];
      }
      // the five sums over the warp by halving: at each step a lane keeps half of its
      // values and adds the partner's copy of them; lane 4 k ends with sum k (9 shuffles)
      const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
      float q[4], q2[2];
#pragma unroll
      for (int j = 0; j < 4; j++) {
         const float lo = pr[j], hi = j == 0 ? pr[4] : 0.0f;
         q[j] = (b4 ? hi : lo) + __shfl_xor_sync(0xffffffffu, b4 ? lo : hi, 16);
      }
#pragma unroll
      for (int j = 0; j < 2; j++) q2[j] = (b3 ? q[j + 2] : q[j]) + __shfl_xor_sync(0xffffffffu, b3 ? q[j] : q[j + 2], 8);
      float r = (b2 ? q2[1] : q2[0]) + __shfl_xor_sync(0xffffffffu, b2 ? q2[0] : q2[1], 4);
      r += __shfl_xor_sync(0xffffffffu, r, 2);
      r += __shfl_xor_sync(0xffffffffu, r, 1);
      const int k = lane >> 2;
      if ((lane & 3) == 0 && k < 5) a.part[(base + s) * 5 + k] = r;
   }
   __syncwarp(); // every lane's last read of the stage sequences precedes the staging writes
   storePacked(g, a.g + c.xOff, t0, Lu, sStage, lane);
}

// Coefficient gradients of one channel (one CTA, coefficients spread over its warps): per
// coefficient, lane l adds the partial sums of units l, l + 32, ... in FP64, in that order,
// four loads in flight, then a fixed butterfly adds the lanes' sums (bitwise repeatable).
constexpr int kCoefWarps = 8;
__global__ void __launch_bounds__(32 * kCoefWarps) bank_coef_kernel(const RaggedChan *chans, const float *part,
                                                                    float *gcoefs)
{
   const RaggedChan c = chans[blockIdx.x];
   const int S = c.S, units = (c.Lu + kUnit - 1) / kUnit, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   for (int q = warp; q < 5 * S; q += kCoefWarps) {
      const float *pq = part + c.ckOff * 5 + q;
      const long long st = 5LL * S; // one unit's partial sums
      double acc = 0.0;
      int j = lane;
      for (; j + 96 < units; j += 128) {
         const float v0 = pq[j * st], v1 = pq[(j + 32) * st], v2 = pq[(j + 64) * st], v3 = pq[(j + 96) * st];
         acc += (double) v0;
         acc += (double) v1;
         acc += (double) v2;
         acc += (double) v3;
      }
      for (; j < units; j += 32) acc += (double) pq[j * st];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) gcoefs[c.cOff + q] = (float) acc;
   }
}

} // namespace

long long bankTransitionDoubles(int S) { return 8LL * S * (S + 1); } // Phi and Phi^32, both directions

cudaError_t launchBankTables(const RaggedChan *chans, int C, const float *coefs, int totalStages, int Smax,
                             float *tables, double *phi, cudaStream_t s)
{
   if (totalStages <= 0) return cudaSuccess;
   bank_tables_kernel<<<(totalStages + 127) / 128, 128, 0, s>>>(coefs, totalStages, tables);
   const size_t dyn = (size_t) 8 * Smax * (Smax + 1) / 2 * sizeof(double);
   cudaError_t e = cudaFuncSetAttribute(bank_transition_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn);
   if (e != cudaSuccess) return e;
   // one warp per (channel, direction) while the block count is small (up to 36 blocks of
   // 2 x 2 for 8 stages): the squarings' barriers then cost a warp, not four
   bank_transition_kernel<<<dim3(C, 2), Smax <= 8 ? 32 : 128, dyn, s>>>(chans, coefs, phi);
   countLaunch(2);
   return cudaGetLastError();
}

static size_t unitShared(int Smax) { return (size_t) kWarps * Smax * kBankTabFloats * sizeof(float); }
static size_t adjointShared(int Smax)
{
   const size_t seq = (size_t) (Smax > 0 ? Smax - 1 : 0) * kL * 32, stage = (size_t) 32 * kOutPad;
   return ((size_t) Smax * kBankTabFloats + (seq > stage ? seq : stage)) * sizeof(float);
}

template <int MODE> static cudaError_t launchUnits(const UnitArgs &a, cudaStream_t s)
{
   const size_t dyn = unitShared(a.Smax);
   cudaError_t e = cudaFuncSetAttribute(bank_unit_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dyn);
   if (e != cudaSuccess) return e;
   bank_unit_kernel<MODE><<<(a.nUnits + kWarps - 1) / kWarps, kThreads, dyn, s>>>(a);
   countLaunch();
   return cudaGetLastError();
}

cudaError_t launchBankForward(const BankLaunch &b, cudaStream_t s)
{
   if (b.nUnits <= 0) return cudaSuccess;
   UnitArgs a{b.chans, b.units, b.nUnits, b.Smax, b.tables, b.u, nullptr, b.aggF, nullptr};
   cudaError_t e = launchUnits<UNIT_AGG>(a, s);
   if (e != cudaSuccess) return e;
   const size_t dynC = (size_t) (4 * b.Smax * (b.Smax + 1) / 2 + 2 * b.Smax) * sizeof(double);
   if ((e = cudaFuncSetAttribute(bank_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dynC)) !=
       cudaSuccess)
      return e;
   bank_chain_fast_kernel<<<b.C, kChainWarps * 32, 0, s>>>(b.chans, b.chainOrder, b.phi, b.aggF, b.ckptF, b.groupF, 0);
   countLaunch();
   if (b.Smax > kChainFastStages) {
      bank_chain_kernel<<<b.C, 32, dynC, s>>>(b.chans, b.chainOrder, b.phi, b.aggF, b.ckptF, 0);
      countLaunch();
   }
   a.out = b.y;
   a.ckpt = b.ckptF;
   if (b.target) {
      a.target = b.target;
      a.gy = b.gyOut;
      a.lossPart = b.lossPart;
      a.aggA = b.aggA;
      a.scale = b.scale;
      return launchUnits<UNIT_OUT_MSE>(a, s);
   }
   return launchUnits<UNIT_OUT>(a, s);
}

cudaError_t launchBankBackward(const BankLaunch &b, cudaStream_t s)
{
   if (b.nUnits <= 0) return cudaSuccess;
   cudaError_t e = cudaSuccess;
   if (!b.aggReady) {
      UnitArgs a{b.chans, b.units, b.nUnits, b.Smax, b.tables, b.gy, nullptr, b.aggA, nullptr};
      if ((e = launchUnits<UNIT_ADJ_AGG>(a, s)) != cudaSuccess) return e;
   }
   const size_t dynC = (size_t) (4 * b.Smax * (b.Smax + 1) / 2 + 2 * b.Smax) * sizeof(double);
   if ((e = cudaFuncSetAttribute(bank_chain_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) dynC)) !=
       cudaSuccess)
      return e;
   bank_chain_fast_kernel<<<b.C, kChainWarps * 32, 0, s>>>(b.chans, b.chainOrder, b.phi, b.aggA, b.ckptA, b.groupA, 1);
   countLaunch();
   if (b.Smax > kChainFastStages) {
      bank_chain_kernel<<<b.C, 32, dynC, s>>>(b.chans, b.chainOrder, b.phi, b.aggA, b.ckptA, 1);
      countLaunch();
   }
   if ((e = cudaFuncSetAttribute(bank_adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int) adjointShared(b.Smax))) != cudaSuccess)
      return e;
   AdjArgs d{b.chans, b.units, b.nUnits, b.Smax, b.tables, b.u, b.gy, b.ckptF, b.ckptA, b.g, b.part, 0};
   // One launch per stage count, each with the shared memory its cascades need, spread over
   // the caller's stream and the auxiliary ones so that CTAs of different buckets share the
   // SMs (and no launch waits for another's tail).
   const int lanes = 1 + b.nAux;
   if (b.nAux > 0) {
      if ((e = cudaEventRecord(b.fork, s)) != cudaSuccess) return e;
      for (int i = 0; i < b.nAux; i++)
         if ((e = cudaStreamWaitEvent(b.aux[i], b.fork, 0)) != cudaSuccess) return e;
   }
   for (int k = 0; k < b.nBuckets; k++) {
      d.first = b.bucketStart[k];
      const int n = b.bucketStart[k + 1] - b.bucketStart[k];
      if (n <= 0) continue;
      const cudaStream_t st = (k % lanes) == 0 ? s : b.aux[(k % lanes) - 1];
      bank_adjoint_kernel<<<n, 32, adjointShared(b.bucketS[k]), st>>>(d);
      countLaunch();
   }
   for (int i = 0; i < b.nAux; i++) {
      if ((e = cudaEventRecord(b.join[i], b.aux[i])) != cudaSuccess) return e;
      if ((e = cudaStreamWaitEvent(s, b.join[i], 0)) != cudaSuccess) return e;
   }
   bank_coef_kernel<<<b.C, 32 * kCoefWarps, 0, s>>>(b.chans, b.part, b.gcoefs);
   countLaunch();
   return cudaGetLastError();
}

} // namespace dsplib
