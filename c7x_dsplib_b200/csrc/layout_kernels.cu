// Layout kernels for sm_100a: DSPLIB_interleave / DSPLIB_deinterleave (a strided
// matrix transpose) and DSPLIB_addNCh (sum of stacked inputs).
//
// transpose_kernel<E>  out[(i * strideOutBytes) / E + j] = in[i + strideInElems * j]
//                      for i < W (input columns), j < H (input rows), E-byte elements.
//                      A CTA moves a tile of TJ input rows x TI input columns (TJ * TI =
//                      1024, powers of two) through shared memory: it reads the tile row
//                      by row (consecutive threads on consecutive columns) and writes it
//                      output row by output row (consecutive threads on consecutive j), so
//                      both sides are coalesced, with 16-byte accesses wherever rows allow.  The tile follows the matrix's shape: a
//                      two-channel interleave (H = 2) uses 2 x 512 tiles, a two-channel
//                      deinterleave (W = 2) 512 x 2 tiles, large matrices 32 x 32.
// addnch_kernel<F>     out[row * sO + col] = ((0 + x_0) + x_1) + ... in input order, one CTA
//                      per 1024-sample row segment, four columns per thread (each layer's
//                      loads are coalesced and independent).
// Both are pure data movement bound by HBM bandwidth.
#include <cuda_runtime.h>

#include <cstdint>

#include "dsplib_internal.h"

namespace dsplib {

namespace {

constexpr int kThreads = 256;
constexpr int kTile = 1024;

template <int E> struct Word;
template <> struct Word<1> { using T = uint8_t; };
template <> struct Word<2> { using T = uint16_t; };
template <> struct Word<4> { using T = uint32_t; };
template <> struct Word<8> { using T = unsigned long long; };

// Tile (TJ x TI) of the transpose: CTA (blockIdx.x = column tile, blockIdx.y strides over
// row tiles).  Element idx of the load phase is (r, c) = (idx / TI, idx % TI); element idx
// of the store phase is (output row r2, column c2) = (idx / TJ, idx % TJ).  With vecIn /
// vecOut a thread moves V = 16 / E consecutive idx as one 16-byte access: the host sets
// the flag only when such a run is contiguous and aligned in memory (a run inside one row,
// or rows packed back to back with the tile spanning whole rows); runs that cross the
// matrix edge fall back to element accesses.
template <int E>
__global__ void __launch_bounds__(kThreads) transpose_kernel(const typename Word<E>::T *__restrict__ in,
                                                             typename Word<E>::T *__restrict__ out, long long W,
                                                             long long H, long long sInE, long long sOutB, int logTI,
                                                             int logTJ, int vecIn, int vecOut)
{
   using T = typename Word<E>::T;
   constexpr int V = 16 / E;
   __shared__ T tile[2 * kTile]; // TJ rows of TI + 1 elements: TJ * (TI + 1) = 1024 + TJ <= 2048
   const int TI = 1 << logTI, TJ = 1 << logTJ, pitch = TI + 1;
   const long long i0 = (long long) blockIdx.x << logTI;
   for (long long jt = blockIdx.y; (jt << logTJ) < H; jt += gridDim.y) {
      const long long j0 = jt << logTJ;
      if (vecIn) {
         for (int idx = threadIdx.x * V; idx < kTile; idx += kThreads * V) {
            const int rl = (idx + V - 1) >> logTI, cl = (idx + V - 1) & (TI - 1);
            const int r = idx >> logTI, c = idx & (TI - 1);
            if (j0 + rl < H && i0 + cl < W) {
               const uint4 v = __ldcs((const uint4 *) (in + (j0 + r) * sInE + i0 + c));
               const T *e = (const T *) &v;
#pragma unroll
               for (int k = 0; k < V; k++) tile[((idx + k) >> logTI) * pitch + ((idx + k) & (TI - 1))] = e[k];
            }
            else {
#pragma unroll
               for (int k = 0; k < V; k++) {
                  const int rk = (idx + k) >> logTI, ck = (idx + k) & (TI - 1);
                  if (j0 + rk < H && i0 + ck < W) tile[rk * pitch + ck] = in[(j0 + rk) * sInE + i0 + ck];
               }
            }
         }
      }
      else {
         for (int idx = threadIdx.x; idx < kTile; idx += kThreads) {
            const int r = idx >> logTI, c = idx & (TI - 1);
            if (j0 + r < H && i0 + c < W) tile[r * pitch + c] = in[(j0 + r) * sInE + i0 + c];
         }
      }
      __syncthreads();
      if (vecOut) {
         for (int idx = threadIdx.x * V; idx < kTile; idx += kThreads * V) {
            const int rl = (idx + V - 1) >> logTJ, cl = (idx + V - 1) & (TJ - 1);
            const int r = idx >> logTJ, c = idx & (TJ - 1);
            if (i0 + rl < W && j0 + cl < H) {
               uint4 v;
               T *e = (T *) &v;
#pragma unroll
               for (int k = 0; k < V; k++) e[k] = tile[((idx + k) & (TJ - 1)) * pitch + ((idx + k) >> logTJ)];
               __stcs((uint4 *) (out + ((i0 + r) * sOutB) / E + j0 + c), v);
            }
            else {
#pragma unroll
               for (int k = 0; k < V; k++) {
                  const int rk = (idx + k) >> logTJ, ck = (idx + k) & (TJ - 1);
                  if (i0 + rk < W && j0 + ck < H) out[((i0 + rk) * sOutB) / E + j0 + ck] = tile[ck * pitch + rk];
               }
            }
         }
      }
      else {
         for (int idx = threadIdx.x; idx < kTile; idx += kThreads) {
            const int r = idx >> logTJ, c = idx & (TJ - 1); // r: output row (i), c: j
            if (i0 + r < W && j0 + c < H) out[((i0 + r) * sOutB) / E + j0 + c] = tile[c * pitch + r];
         }
      }
      __syncthreads();
   }
}

// Few channels (K <= 4), packed on the interleaved side: no shared memory.  Interleave
// (H = K rows of W samples -> W rows of K): a thread takes V = 16 / E consecutive columns,
// loads one 16-byte vector from each of the K rows and writes the K * V interleaved
// elements as K 16-byte vectors (consecutive threads write consecutive 16K-byte spans).
// Deinterleave (W = K columns, H rows) is the mirror image.  Columns (rows) past the last
// whole vector are left to transpose_kernel.
template <int E, int K>
__global__ void __launch_bounds__(kThreads) interleave_k_kernel(const typename Word<E>::T *__restrict__ in,
                                                                typename Word<E>::T *__restrict__ out,
                                                                long long groups, long long sInE)
{
   using T = typename Word<E>::T;
   constexpr int V = 16 / E;
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g = (long long) blockIdx.x * kThreads + threadIdx.x; g < groups; g += stride) {
      uint4 a[K], b[K];
#pragma unroll
      for (int j = 0; j < K; j++) a[j] = __ldcs((const uint4 *) (in + j * sInE + g * V));
      const T *src = (const T *) a;
      T *dst = (T *) b;
#pragma unroll
      for (int q = 0; q < K * V; q++) dst[q] = src[(q % K) * V + q / K]; // out (i, j) = in (j, i)
#pragma unroll
      for (int j = 0; j < K; j++) __stcs((uint4 *) (out + g * V * K) + j, b[j]);
   }
}

template <int E, int K>
__global__ void __launch_bounds__(kThreads) deinterleave_k_kernel(const typename Word<E>::T *__restrict__ in,
                                                                  typename Word<E>::T *__restrict__ out,
                                                                  long long groups, long long sOutE)
{
   using T = typename Word<E>::T;
   constexpr int V = 16 / E;
   const long long stride = (long long) gridDim.x * kThreads;
   for (long long g = (long long) blockIdx.x * kThreads + threadIdx.x; g < groups; g += stride) {
      uint4 a[K], b[K];
#pragma unroll
      for (int j = 0; j < K; j++) a[j] = __ldcs((const uint4 *) (in + g * V * K) + j);
      const T *src = (const T *) a;
      T *dst = (T *) b;
#pragma unroll
      for (int q = 0; q < K * V; q++) dst[q] = src[(q % V) * K + q / V]; // out row q / V, column q % V
#pragma unroll
      for (int i = 0; i < K; i++) __stcs((uint4 *) (out + i * sOutE + g * V), b[i]);
   }
}

template <typename F> __device__ __forceinline__ F addRn(F a, F b);
template <> __device__ __forceinline__ float addRn(float a, float b) { return __fadd_rn(a, b); }
template <> __device__ __forceinline__ double addRn(double a, double b) { return __dadd_rn(a, b); }

template <typename F>
__global__ void __launch_bounds__(kThreads) addnch_kernel(const F *__restrict__ in, F *__restrict__ out,
                                                          long long samples, long long tilesPerRow, long long tiles,
                                                          int inputs, long long sY, long long sZ, long long sO)
{
   for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
      const long long row = t / tilesPerRow, c0 = (t % tilesPerRow) * kTile;
      F acc[4];
      bool ok[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
         acc[k] = F(0);
         ok[k] = c0 + threadIdx.x + k * kThreads < samples;
      }
      const F *p = in + row * sY + c0 + threadIdx.x;
      for (int l = 0; l < inputs; l++) {
#pragma unroll
         for (int k = 0; k < 4; k++)
            if (ok[k]) acc[k] = addRn(acc[k], p[(long long) l * sZ + k * kThreads]);
      }
#pragma unroll
      for (int k = 0; k < 4; k++)
         if (ok[k]) out[row * sO + c0 + threadIdx.x + k * kThreads] = acc[k];
   }
}

int waveBlocks(long long tiles)
{
   static int sms = 0;
   if (sms == 0) {
      int dev = 0;
      if (cudaGetDevice(&dev) != cudaSuccess ||
          cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
         sms = 148;
   }
   const long long cap = (long long) sms * 8;
   return (int) (tiles < 1 ? 1 : (tiles > cap ? cap : tiles));
}

int log2ceil(long long v)
{
   int l = 0;
   while ((1LL << l) < v) l++;
   return l;
}

} // namespace

cudaError_t launchTiled(const TransposeLaunch &a, cudaStream_t s);

template <int E, int K> void launchFewK(const TransposeLaunch &a, bool inter, long long groups, cudaStream_t s)
{
   using T = typename Word<E>::T;
   const long long blocks = (groups + kThreads - 1) / kThreads;
   const int grid = waveBlocks(blocks);
   if (inter)
      interleave_k_kernel<E, K><<<grid, kThreads, 0, s>>>((const T *) a.in, (T *) a.out, groups, a.sInE);
   else
      deinterleave_k_kernel<E, K><<<grid, kThreads, 0, s>>>((const T *) a.in, (T *) a.out, groups, a.sOutB / E);
   countLaunch();
}

template <int E> void launchFewE(const TransposeLaunch &a, bool inter, int K, long long groups, cudaStream_t s)
{
   switch (K) {
   case 2: launchFewK<E, 2>(a, inter, groups, s); break;
   case 3: launchFewK<E, 3>(a, inter, groups, s); break;
   default: launchFewK<E, 4>(a, inter, groups, s); break;
   }
}

cudaError_t launchTranspose(const TransposeLaunch &a, cudaStream_t s)
{
   if (a.W <= 0 || a.H <= 0) return cudaSuccess;
   {
      // 2-4 channels packed on the interleaved side, 16-byte aligned rows on the other side
      const long long E = a.elt, V = 16 / E;
      const bool aligned = ((uintptr_t) a.in & 15u) == 0 && ((uintptr_t) a.out & 15u) == 0;
      const bool inter = a.H >= 2 && a.H <= 4 && a.W >= V && a.sOutB == a.H * E && (a.sInE * E) % 16 == 0;
      const bool deinter = a.W >= 2 && a.W <= 4 && a.H >= V && a.sInE == a.W && a.sOutB % 16 == 0;
      if (aligned && (inter || deinter)) {
         const int K = (int) (inter ? a.H : a.W);
         const long long n = inter ? a.W : a.H, groups = n / V, done = groups * V;
         switch (a.elt) {
         case 1: launchFewE<1>(a, inter, K, groups, s); break;
         case 2: launchFewE<2>(a, inter, K, groups, s); break;
         case 4: launchFewE<4>(a, inter, K, groups, s); break;
         default: launchFewE<8>(a, inter, K, groups, s); break;
         }
         if (done == n) return cudaGetLastError();
         // the last partial vector's columns (rows) through the tiled kernel
         TransposeLaunch r = a;
         if (inter) {
            r.in = (const char *) a.in + done * E;
            r.out = (char *) a.out + done * a.sOutB;
            r.W = a.W - done;
         }
         else {
            r.in = (const char *) a.in + done * a.sInE * E;
            r.out = (char *) a.out + done * E;
            r.H = a.H - done;
         }
         return launchTiled(r, s);
      }
   }
   return launchTiled(a, s);
}

cudaError_t launchTiled(const TransposeLaunch &a, cudaStream_t s)
{
   // tile shape: the smaller side gets up to 32 (its next power of two), the other the rest of 1024
   int logTI, logTJ;
   if (a.H <= a.W) {
      logTJ = log2ceil(a.H) < 5 ? log2ceil(a.H) : 5;
      logTI = 10 - logTJ;
   }
   else {
      logTI = log2ceil(a.W) < 5 ? log2ceil(a.W) : 5;
      logTJ = 10 - logTI;
   }
   const long long TI = 1LL << logTI, TJ = 1LL << logTJ, V = 16 / a.elt, E = a.elt;
   const long long tilesI = (a.W + TI - 1) >> logTI;
   const long long tilesJ = (a.H + TJ - 1) >> logTJ;
   if (tilesI > 0x7fffffffLL) return cudaErrorInvalidValue;
   // 16-byte runs: inside one row (row pitch a multiple of 16 bytes), or over rows packed back
   // to back that the tile spans whole
   const bool inAligned = ((uintptr_t) a.in & 15u) == 0, outAligned = ((uintptr_t) a.out & 15u) == 0;
   const int vecIn = inAligned && ((TI >= V && (a.sInE * E) % 16 == 0) || (TI < V && a.sInE == a.W && TI == a.W));
   const int vecOut = outAligned && ((TJ >= V && a.sOutB % 16 == 0) || (TJ < V && a.sOutB == a.H * E && TJ == a.H));
   const dim3 grid((unsigned) tilesI, (unsigned) (tilesJ < 65535 ? tilesJ : 65535));
   switch (a.elt) {
   case 1:
      transpose_kernel<1><<<grid, kThreads, 0, s>>>((const uint8_t *) a.in, (uint8_t *) a.out, a.W, a.H, a.sInE,
                                                    a.sOutB, logTI, logTJ, vecIn, vecOut);
      break;
   case 2:
      transpose_kernel<2><<<grid, kThreads, 0, s>>>((const uint16_t *) a.in, (uint16_t *) a.out, a.W, a.H, a.sInE,
                                                    a.sOutB, logTI, logTJ, vecIn, vecOut);
      break;
   case 4:
      transpose_kernel<4><<<grid, kThreads, 0, s>>>((const uint32_t *) a.in, (uint32_t *) a.out, a.W, a.H, a.sInE,
                                                    a.sOutB, logTI, logTJ, vecIn, vecOut);
      break;
   case 8:
      transpose_kernel<8><<<grid, kThreads, 0, s>>>((const unsigned long long *) a.in, (unsigned long long *) a.out,
                                                    a.W, a.H, a.sInE, a.sOutB, logTI, logTJ, vecIn, vecOut);
      break;
   default: return cudaErrorInvalidValue;
   }
   countLaunch();
   return cudaGetLastError();
}

cudaError_t launchAddNCh(const AddNChLaunch &a, cudaStream_t s)
{
   if (a.samples <= 0 || a.channels <= 0) return cudaSuccess;
   const long long tilesPerRow = (a.samples + kTile - 1) / kTile;
   const long long tiles = tilesPerRow * a.channels;
   const int grid = waveBlocks(tiles);
   if (a.isDouble)
      addnch_kernel<double><<<grid, kThreads, 0, s>>>((const double *) a.in, (double *) a.out, a.samples, tilesPerRow,
                                                      tiles, a.inputs, a.sY, a.sZ, a.sO);
   else
      addnch_kernel<float><<<grid, kThreads, 0, s>>>((const float *) a.in, (float *) a.out, a.samples, tilesPerRow,
                                                     tiles, a.inputs, a.sY, a.sZ, a.sO);
   countLaunch();
   return cudaGetLastError();
}

} // namespace dsplib
