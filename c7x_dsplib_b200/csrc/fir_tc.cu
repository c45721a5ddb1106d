// Tensor-core (tcgen05) FIR kernels for sm_100a.
//
// FIR as a Toeplitz contraction.  One tile = 2048 consecutive outputs of one
// channel, computed by M = 128 rows x N = 16 phases:
//     D[a][b] = sum_m A[a][m] * B[m][b] = y[j0 + 16a + b]
//     A[a][m] = x[j0 + 16a + m]            (data, Hankel: row a starts 16 samples after row a-1)
//     B[m][b] = g[m - b], g[c] = h[T-1-c]  (taps band, zero outside 0 <= m-b < T)
// with K = T + 15 rounded up to the MMA depth.  For 8-bit operands a 16-byte
// core-matrix row holds exactly 16 samples, so the Hankel matrix A is read by
// the tensor core straight from the raw signal segment in shared memory: the
// no-swizzle K-major descriptor with row pitch 16 B, LBO = 16 B (next 16
// samples) and SBO = 128 B (next 8 rows) makes consecutive rows overlap.  No
// expanded copy of the signal is ever written.  The taps band B (16 x K) is
// built once per CTA and channel.  Accumulators live in TMEM and are drained
// by 4 warps with tcgen05.ld (thread a receives the 16 consecutive outputs of
// row a, so the stores are contiguous).
//
// int8:  one s8 x s8 product, int32 accumulator.
// int16: x = 256*xh + xl, g = 256*gh + gl (xh, gh signed bytes; xl, gl
//        unsigned bytes); y = 65536*hh + 256*(hl + lh) + ll, each term an
//        exact int32 kind::i8 accumulation, recombined exactly in 64 bits.
//        Modulo 2^16 the hh term vanishes, so the natural-C (wrap) mode
//        issues three products instead of four.
// Output stage: wrap (natural-C semantics) or Q mode (round half up, shift,
// saturate), both exact.
#include <cuda_runtime.h>

#include "dsplib_internal.h"
#include "tc_common.cuh"

namespace dsplib {

__device__ int g_firTcError; // set when a bounded wait for the tensor core gives up

namespace {

constexpr int kRows = 128;
constexpr int kPhases = 16;
constexpr int kTile = kRows * kPhases; // outputs per tile
constexpr int kThreads = 128;
constexpr int kMaxTapsTc = 2048;

__host__ __device__ inline int bandK(int T) { return ((T + 15 + 31) / 32) * 32; }

template <typename T> struct IntLimits;
template <> struct IntLimits<int8_t> { static constexpr long long lo = -128, hi = 127; };
template <> struct IntLimits<int16_t> { static constexpr long long lo = -32768, hi = 32767; };

template <typename T, int QMODE>
__device__ __forceinline__ T outStage(long long acc, int shift)
{
   if (!QMODE) return (T) acc; // modulo 2^bits
   if (shift > 0) acc = (acc + (1LL << (shift - 1))) >> shift;
   if (acc < IntLimits<T>::lo) acc = IntLimits<T>::lo;
   if (acc > IntLimits<T>::hi) acc = IntLimits<T>::hi;
   return (T) acc;
}

template <typename T, int QMODE>
__global__ void __launch_bounds__(kThreads) fir_int_tc_kernel(FirLaunch a, int tilesPerCta)
{
   constexpr bool SPLIT = sizeof(T) == 2;
   constexpr uint32_t kCols = SPLIT ? 64 : 32; // TMEM columns (accumulators of 16 columns each)
   const int T_ = a.T;
   const int Kt = bandK(T_);
   const int seg = kTile + Kt; // signal samples one tile reads (bytes per byte-plane)
   extern __shared__ __align__(128) unsigned char sm[];
   uint64_t *mbar = (uint64_t *) sm;
   uint32_t *tslot = (uint32_t *) (sm + 8);
   unsigned char *B0 = sm + 16;
   unsigned char *B1 = B0 + (size_t) Kt * 16;
   unsigned char *A0 = B0 + (size_t) Kt * 16 * (SPLIT ? 2 : 1);
   unsigned char *A1 = A0 + seg;

   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   if (warp == 0) tc::tmemAlloc(tslot, kCols);
   if (tid == 0) tc::mbarInit(mbar, 1);
   tc::fenceBeforeSync();
   __syncthreads();
   tc::fenceAfterSync();
   const uint32_t tmem = *tslot;

   const int nt = (a.outSize + kTile - 1) / kTile;
   const long long inExtent = (long long) a.outSize + T_ - 1;
   uint32_t iter = 0;
   bool failed = false;
   for (int l = blockIdx.y; l < a.batch && !failed; l += gridDim.y) {
      const T *x = (const T *) a.x + (long long) l * a.inPitch;
      const T *h = (const T *) a.h + (long long) l * a.filtPitch;
      T *y = (T *) a.y + (long long) l * a.outPitch;
      // Taps band, K-major no-swizzle: byte (q*256 + i*128 + r*16 + e) holds B[m = 16q + e][b = 8i + r].
      for (int idx = tid; idx < Kt * 16; idx += kThreads) {
         const int q = idx >> 8, rem = idx & 255;
         const int b = ((rem >> 7) << 3) + ((rem >> 4) & 7);
         const int m = (q << 4) + (rem & 15);
         const int c = m - b;
         const int g = (c >= 0 && c < T_) ? (int) h[T_ - 1 - c] : 0;
         if (SPLIT) {
            B0[idx] = (unsigned char) (g >> 8);
            B1[idx] = (unsigned char) (g & 0xFF);
         }
         else {
            B0[idx] = (unsigned char) g;
         }
      }
      const int t0 = blockIdx.x * tilesPerCta;
      const int t1 = min(nt, t0 + tilesPerCta);
      for (int t = t0; t < t1; t++) {
         const long long j0 = (long long) t * kTile;
         // Signal segment of this tile (zero past the row's extent).
         const T *xs = x + j0;
         const bool full = j0 + seg <= inExtent;
         if (!SPLIT && full && (((uintptr_t) xs) & 15) == 0) {
            for (int k = tid; k < seg / 16; k += kThreads) ((int4 *) A0)[k] = ((const int4 *) xs)[k];
         }
         else {
            for (int k = tid; k < seg; k += kThreads) {
               const int v = (full || j0 + k < inExtent) ? (int) xs[k] : 0;
               if (SPLIT) {
                  A0[k] = (unsigned char) (v >> 8);
                  A1[k] = (unsigned char) (v & 0xFF);
               }
               else {
                  A0[k] = (unsigned char) v;
               }
            }
         }
         tc::fenceProxyAsync();
         __syncthreads();
         if (tid == 0) {
            tc::fenceAfterSync();
            const uint32_t a0 = tc::smemAddr(A0), a1 = tc::smemAddr(A1);
            const uint32_t b0 = tc::smemAddr(B0), b1 = tc::smemAddr(B1);
            for (int kk = 0; kk < Kt / 32; kk++) {
               const uint64_t dA0 = tc::descNoSwizzle(a0 + 32 * kk, 16, 128);
               const uint64_t dB0 = tc::descNoSwizzle(b0 + 512 * kk, 256, 128);
               if (!SPLIT) {
                  tc::mmaI8(tmem, dA0, dB0, tc::idesc(2, 1, 1, kRows, kPhases), kk > 0);
               }
               else {
                  const uint64_t dA1 = tc::descNoSwizzle(a1 + 32 * kk, 16, 128);
                  const uint64_t dB1 = tc::descNoSwizzle(b1 + 512 * kk, 256, 128);
                  if (QMODE) tc::mmaI8(tmem, dA0, dB0, tc::idesc(2, 1, 1, kRows, kPhases), kk > 0); // hi*hi
                  tc::mmaI8(tmem + 16, dA0, dB1, tc::idesc(2, 1, 0, kRows, kPhases), kk > 0);       // hi*lo
                  tc::mmaI8(tmem + 16, dA1, dB0, tc::idesc(2, 0, 1, kRows, kPhases), true);         // lo*hi
                  tc::mmaI8(tmem + 32, dA1, dB1, tc::idesc(2, 0, 0, kRows, kPhases), kk > 0);       // lo*lo
               }
            }
            tc::commit(mbar);
         }
         const bool done = tc::mbarWait(mbar, iter & 1);
         if (!done && tid == 0) atomicExch(&g_firTcError, 1);
         failed = __syncthreads_or(!done) != 0;
         iter++;
         tc::fenceAfterSync();
         if (!failed) {
            // Drain: warp w owns TMEM lanes 32w..32w+31 = rows a; 16 consecutive outputs per row.
            const uint32_t lanes = (uint32_t) (warp * 32) << 16;
            uint32_t acc[3][16];
            tc::tmemLoad16(tmem + lanes, acc[0]);
            if (SPLIT) {
               tc::tmemLoad16(tmem + lanes + 16, acc[1]);
               tc::tmemLoad16(tmem + lanes + 32, acc[2]);
            }
            tc::tmemWaitLoad();
            const int row = warp * 32 + lane;
            const long long jr = j0 + (long long) row * kPhases;
            __align__(16) T out[16];
#pragma unroll
            for (int b = 0; b < 16; b++) {
               long long v;
               if (!SPLIT) {
                  v = (int) acc[0][b];
               }
               else if (QMODE) {
                  v = ((long long) (int) acc[0][b] << 16) + ((long long) (int) acc[1][b] << 8) +
                      (long long) (int) acc[2][b];
               }
               else {
                  v = (long long) (int) (((uint32_t) acc[1][b] << 8) + (uint32_t) acc[2][b]);
               }
               out[b] = outStage<T, QMODE>(v, a.shift);
            }
            T *yr = y + jr;
            if (jr + 16 <= a.outSize && (((uintptr_t) yr) & 15) == 0) {
               if (SPLIT) {
                  ((int4 *) yr)[0] = *(int4 *) &out[0];
                  ((int4 *) yr)[1] = *(int4 *) &out[8];
               }
               else {
                  *(int4 *) yr = *(int4 *) &out[0];
               }
            }
            else {
#pragma unroll
               for (int b = 0; b < 16; b++)
                  if (jr + b < a.outSize) yr[b] = out[b];
            }
         }
         tc::fenceBeforeSync();
         __syncthreads();
         if (failed) break;
      }
   }
   __syncthreads();
   if (warp == 0) tc::tmemFree(tmem, kCols);
}

template <typename T, int QMODE> cudaError_t launchIntTc(const FirLaunch &a, cudaStream_t s)
{
   constexpr bool SPLIT = sizeof(T) == 2;
   const int Kt = bandK(a.T);
   const size_t smem = 16 + (size_t) Kt * 16 * (SPLIT ? 2 : 1) + (size_t) (kTile + Kt) * (SPLIT ? 2 : 1);
   auto fn = fir_int_tc_kernel<T, QMODE>;
   cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
   if (e != cudaSuccess) return e;
   const int nt = (a.outSize + kTile - 1) / kTile;
   // Enough CTAs for several waves on 148 SMs while reusing the taps band across tiles.
   int tpc = 1;
   while (tpc < 8 && (long long) ((nt + tpc * 2 - 1) / (tpc * 2)) * a.batch >= 148 * 8) tpc *= 2;
   dim3 grid((nt + tpc - 1) / tpc, a.batch < 65535 ? a.batch : 65535);
   fn<<<grid, kThreads, smem, s>>>(a, tpc);
   countLaunch();
   return cudaGetLastError();
}

} // namespace

bool firIntTcSupported(const FirLaunch &a)
{
   return (a.dtype == DSPLIB_INT8 || a.dtype == DSPLIB_INT16) && a.T >= 1 && a.T <= kMaxTapsTc && a.outSize > 0;
}

cudaError_t launchFirIntTc(const FirLaunch &a, bool qmode, cudaStream_t s)
{
   if (a.dtype == DSPLIB_INT8) return qmode ? launchIntTc<int8_t, 1>(a, s) : launchIntTc<int8_t, 0>(a, s);
   if (a.dtype == DSPLIB_INT16) return qmode ? launchIntTc<int16_t, 1>(a, s) : launchIntTc<int16_t, 0>(a, s);
   return cudaErrorInvalidValue;
}

int firTcErrorFlag(bool clear)
{
   int v = 0;
   if (cudaMemcpyFromSymbol(&v, g_firTcError, sizeof(int)) != cudaSuccess) return -1;
   if (clear && v) {
      int z = 0;
      cudaMemcpyToSymbol(g_firTcError, &z, sizeof(int));
   }
   return v;
}

cudaError_t launchFirBf16x3(const FirLaunch &a, cudaStream_t s)
{
   (void) a;
   (void) s;
   return cudaErrorNotSupported;
}

} // namespace dsplib
