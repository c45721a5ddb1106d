// Tensor-core (tcgen05) FIR kernels for sm_100a.
//
// FIR as a Toeplitz contraction.  A tile of consecutive outputs of one channel
// is computed by an M = 128 (rows) x N (phases) accumulator in TMEM:
//     D[a][b] = sum_m A[a][m] * B[m][b] = y[j0 + P*a + b]
//     A[a][m] = x[j0 + P*a + m]            (data, Hankel: row a starts P samples after row a-1)
//     B[m][b] = g[m - b], g[c] = h[T-1-c]  (taps band, zero outside 0 <= m-b < T)
// The Hankel matrix A is never expanded: the shared-memory descriptors make
// consecutive rows overlap inside the raw signal segment.
//
// int8/int16 (kind::i8, P = 16, N = 16, tile 2048): an 8-bit core-matrix row
//   is 16 bytes = 16 samples, so the no-swizzle K-major descriptor with
//   LBO = 16 B and SBO = 128 B reads row a at byte 16a of the segment.
//   int8: one s8 x s8 product.  int16: x = 256*xh + xl, g = 256*gh + gl (xh, gh
//   signed bytes, xl, gl unsigned); y = 65536*hh + 256*(hl + lh) + ll, each an
//   exact int32 kind::i8 accumulation recombined exactly in 64 bits; modulo
//   2^16 the hh term vanishes, so the wrap mode issues three products.
//   Output stage: wrap (natural-C) or Q mode (round half up, shift, saturate).
//
// float (split-BF16x3, kind::f16, P = 64, N = 128, tile 8192): each operand is
//   split into BF16 hi + lo (lo = bf16(v - hi)); the signal planes are stored
//   as consecutive 128-byte blocks of 64 samples in the 128-byte-swizzle
//   K-major layout, whose 8-row atoms have a 128-byte row pitch, so with the
//   descriptor starting at block kb row a reads block a + kb.  B rows 0..63
//   hold g_hi by phase, rows 64..127 g_lo:
//     MMA 1: D[:, 0:128] += A_hi x B        (x_hi*g_hi | x_hi*g_lo)
//     MMA 2: D[:, 0:128] += A_lo x B        (x_lo*g_hi | x_lo*g_lo)
//     y[j0 + 64a + b] = D[a][b] + D[a][64 + b]
//   The three products hi*hi, hi*lo, lo*hi leave the lo*lo term (2^-16 of each
//   product) out, 1.25e-5 of the peak output on the 256-tap FIR workload; the
//   fourth rides in the same MMA (N = 128 instead of 64 for the lo plane) at no
//   measurable cost here (the tile loop is not MMA-bound) and brings it to 8.7e-6.
//
// Each CTA owns consecutive tiles of one channel: the taps are staged into
// shared memory once and the band built from there; the next tile's signal is
// staged into the second buffer while the tensor core works on the current
// one.  The integer kernel is persistent: one wave of CTAs strides over the
// (channel, tile range) work items, keeps a band of shared taps for all of them
// and fetches each item's first segment during the previous item's last tile.
// All waits on the tensor core are bounded; on expiry the kernel sets the error word it
// was given (the calling handle's or plan's), frees its TMEM and exits.
#include <algorithm>
#include <cstdio>

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "dsplib_internal.h"
#include "tc_common.cuh"

namespace dsplib {

// Set the error word of the call (mapped page-locked host memory; a plain store, since
// atomics on host memory are not available on every system).
__device__ __forceinline__ void raiseError(int *err)
{
   if (err) *(volatile int *) err = 1;
}

namespace {

constexpr int kRows = 128;

// ------------------------------------------------------------------ integer

constexpr int kPhases = 16;
constexpr int kTile = kRows * kPhases;
constexpr int kThreads = 128;
constexpr int kMaxTapsTc = 2048;

__host__ __device__ inline int bandK(int T) { return ((T + 15 + 31) / 32) * 32; }

template <typename T> struct IntLimits;
template <> struct IntLimits<int8_t> { static constexpr long long lo = -128, hi = 127; };
template <> struct IntLimits<int16_t> { static constexpr long long lo = -32768, hi = 32767; };

// int8: |acc| <= 2048 * 2^14 fits 32 bits, so the output stage stays in 32-bit arithmetic.
template <int QMODE> __device__ __forceinline__ int8_t outStage8(int acc, int shift)
{
   if (!QMODE) return (int8_t) acc; // modulo 2^8
   if (shift > 0) acc = (acc + (1 << (shift - 1))) >> shift;
   return (int8_t) max(-128, min(127, acc));
}

// Four int8 Q-mode outputs (round half up, shift, saturate) packed into one word, byte k =
// output k: two saturating pack conversions instead of a clamp per output and byte moves.
__device__ __forceinline__ uint32_t outStage8x4(int v0, int v1, int v2, int v3, int shift)
{
   if (shift > 0) {
      const int r = 1 << (shift - 1);
      v0 = (v0 + r) >> shift, v1 = (v1 + r) >> shift, v2 = (v2 + r) >> shift, v3 = (v3 + r) >> shift;
   }
   uint32_t hi, d;
   asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, 0;" : "=r"(hi) : "r"(v3), "r"(v2));
   asm("cvt.pack.sat.s8.s32.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(v1), "r"(v0), "r"(hi));
   return d;
}

// Two int16 Q-mode outputs packed into one word (low half = v0): round half up and shift in
// 64 bits, narrow to 32 bits with saturation, then one saturating pack conversion.
__device__ __forceinline__ uint32_t outStage16x2(long long v0, long long v1, int shift)
{
   if (shift > 0) {
      const long long r = 1LL << (shift - 1);
      v0 = (v0 + r) >> shift, v1 = (v1 + r) >> shift;
   }
   int w0, w1;
   uint32_t d;
   asm("cvt.sat.s32.s64 %0, %1;" : "=r"(w0) : "l"(v0));
   asm("cvt.sat.s32.s64 %0, %1;" : "=r"(w1) : "l"(v1));
   asm("cvt.pack.sat.s16.s32 %0, %1, %2;" : "=r"(d) : "r"(w1), "r"(w0));
   return d;
}

template <typename T, int QMODE>
__device__ __forceinline__ T outStage(long long acc, int shift)
{
   if (!QMODE) return (T) acc; // modulo 2^bits
   if (shift > 0) acc = (acc + (1LL << (shift - 1))) >> shift;
   if (acc < IntLimits<T>::lo) acc = IntLimits<T>::lo;
   if (acc > IntLimits<T>::hi) acc = IntLimits<T>::hi;
   return (T) acc;
}

// One 16-byte vector (16 / sizeof(T) samples) of the segment starting at xs, the
// samples at or beyond `avail` read as zero: whole vectors load as one access, the one
// vector that straddles the row end element by element.
template <typename T> __device__ __forceinline__ int4 loadSegVec(const T *xs, long long k, long long avail)
{
   constexpr int per = 16 / sizeof(T);
   const long long s0 = k * per;
   if (s0 + per <= avail) return ((const int4 *) xs)[k];
   __align__(16) T tmp[per];
#pragma unroll
   for (int e = 0; e < per; e++) tmp[e] = (s0 + e < avail) ? xs[s0 + e] : (T) 0;
   return *(const int4 *) tmp;
}

// Write one 16-byte vector of samples into the byte plane(s): int8 -> A0; int16 ->
// A0 = high (signed) bytes, A1 = low (unsigned) bytes.
template <typename T>
__device__ __forceinline__ void putSegVec(const int4 &v, int k, unsigned char *A0, unsigned char *A1)
{
   if (sizeof(T) == 1) {
      ((int4 *) A0)[k] = v;
   }
   else {
      const int16_t *e = (const int16_t *) &v;
      __align__(8) unsigned char hb[8], lb[8];
#pragma unroll
      for (int i = 0; i < 8; i++) {
         hb[i] = (unsigned char) (e[i] >> 8);
         lb[i] = (unsigned char) (e[i] & 0xFF);
      }
      ((uint2 *) A0)[k] = *(uint2 *) hb;
      ((uint2 *) A1)[k] = *(uint2 *) lb;
   }
}

// Stage seg samples of xs (row positions j0 .. j0 + seg - 1, zero from inExtent on) into
// the byte plane(s).  16-byte vectors when xs is aligned, samples otherwise.
template <typename T>
__device__ __forceinline__ void intStage(const T *xs, long long j0, long long inExtent, int seg, unsigned char *A0,
                                         unsigned char *A1, int tid)
{
   constexpr bool SPLIT = sizeof(T) == 2;
   constexpr int per = 16 / sizeof(T); // samples per 16-byte vector
   const long long avail = inExtent - j0;
   if ((((uintptr_t) xs) & 15) == 0) {
      for (int k = tid; k < seg / per; k += kThreads) putSegVec<T>(loadSegVec<T>(xs, k, avail), k, A0, A1);
   }
   else {
      for (int k = tid; k < seg; k += kThreads) {
         const int v = (k < avail) ? (int) xs[k] : 0;
         if (SPLIT) {
            A0[k] = (unsigned char) (v >> 8);
            A1[k] = (unsigned char) (v & 0xFF);
         }
         else {
            A0[k] = (unsigned char) v;
         }
      }
   }
}

// Write n consecutive outputs dst[0..n) of one tile from shared memory, where
// the tile's 16-byte chunk ci (bytes 16ci .. 16ci+15 of the output run) sits at
// byte offset cpos(ci) of stage.  The accumulator drain leaves one output row
// per lane, so storing straight from registers would make every lane of a warp
// hit a different row (one memory transaction per lane and instruction); from
// shared memory a warp writes contiguous 16-byte vectors instead.  The vectors
// are aligned to the destination: when dst is not 16-byte aligned (row pitches
// such as N - T + 1 elements), each vector is assembled from two stage chunks
// with a funnel shift, and a head and tail of scalar stores cover the ends.
template <typename T, typename ChunkPos>
__device__ __forceinline__ void storeTile(T *dst, int n, const unsigned char *stage, ChunkPos cpos, int tid,
                                          int nthreads)
{
   auto elem = [&](int k) {
      const int byte = k * (int) sizeof(T);
      return *(const T *) (stage + cpos(byte >> 4) + (byte & 15));
   };
   const int hb = (16 - (int) ((uintptr_t) dst & 15)) & 15; // bytes before the first 16-byte boundary
   const int head = min(n, hb / (int) sizeof(T));
   const int nvec = (n - head) * (int) sizeof(T) / 16;
   if (tid < head) dst[tid] = elem(tid);
   const int q = hb >> 2, r = (hb & 3) * 8;
   unsigned char *dv = (unsigned char *) dst + hb;
   for (int v = tid; v < nvec; v += nthreads) {
      const uint4 a = *(const uint4 *) (stage + cpos(v));
      uint4 o = a;
      if (hb) {
         const uint4 b = *(const uint4 *) (stage + cpos(v + 1));
         uint32_t w0, w1, w2, w3, w4;
         switch (q) { // uniform across the CTA
         case 0: w0 = a.x, w1 = a.y, w2 = a.z, w3 = a.w, w4 = b.x; break;
         case 1: w0 = a.y, w1 = a.z, w2 = a.w, w3 = b.x, w4 = b.y; break;
         case 2: w0 = a.z, w1 = a.w, w2 = b.x, w3 = b.y, w4 = b.z; break;
         default: w0 = a.w, w1 = b.x, w2 = b.y, w3 = b.z, w4 = b.w; break;
         }
         o.x = __funnelshift_r(w0, w1, r);
         o.y = __funnelshift_r(w1, w2, r);
         o.z = __funnelshift_r(w2, w3, r);
         o.w = __funnelshift_r(w3, w4, r);
      }
      *(uint4 *) (dv + 16 * v) = o;
   }
   for (int k = head + nvec * (16 / (int) sizeof(T)) + tid; k < n; k += nthreads) dst[k] = elem(k);
}

template <typename T, int QMODE>
__global__ void __launch_bounds__(kThreads, sizeof(T) == 2 ? 6 : 8) fir_int_tc_kernel(FirLaunch a, int tilesPerCta)
{
   constexpr bool SPLIT = sizeof(T) == 2;
   constexpr uint32_t kCols = SPLIT ? 64 : 32; // TMEM columns (accumulators of 16 columns each)
   const int T_ = a.T;
   const int Kt = bandK(T_);
   const int seg = kTile + Kt;            // samples one tile reads (multiple of 32)
   const int nplane = SPLIT ? 2 : 1;
   extern __shared__ __align__(128) unsigned char sm[];
   uint64_t *mbar = (uint64_t *) sm;
   uint32_t *tslot = (uint32_t *) (sm + 8);
   // Reversed taps g[c] = h[T-1-c] as bytes (int16: high and low byte planes) at
   // byte 16 + c of gb0 / gb1, zero elsewhere: one 32-bit word per thread to build.
   const int gbWords = (Kt + 20) / 4;
   uint32_t *gb0 = (uint32_t *) (sm + 16);
   uint32_t *gb1 = gb0 + gbWords;
   unsigned char *B0 = sm + 16 + ((gbWords * 4 * nplane + 15) & ~15);
   unsigned char *B1 = B0 + (size_t) Kt * 16;
   unsigned char *Abase = B0 + (size_t) Kt * 16 * nplane;
   // A[buf][plane]: seg bytes each
   auto A = [&](int buf, int plane) { return Abase + (size_t) (buf * nplane + plane) * seg; };
   T *ostage = (T *) (Abase + (size_t) 2 * nplane * seg); // one tile of outputs, row-major

   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   if (warp == 0) tc::tmemAlloc(tslot, kCols);
   if (tid == 0) tc::mbarInit(mbar, 1);
   tc::fenceBeforeSync();
   __syncthreads();
   tc::fenceAfterSync();
   const uint32_t tmem = *tslot;

   const int nt = (a.outSize + kTile - 1) / kTile;
   const long long inExtent = (long long) a.outSize + T_ - 1;
   // Work item = tiles [part * tilesPerCta, ...) of one channel; CTAs stride over the items
   // (persistent: the taps band of shared taps is built once per CTA, and each item's first
   // segment is fetched during the previous item's last tile).
   const int nParts = (nt + tilesPerCta - 1) / tilesPerCta;
   const long long nItems = (long long) a.batch * nParts;
   uint32_t iter = 0;
   bool failed = false;
   int bandOf = -1; // channel whose taps the band holds
   int buf = 0;
   long long item = blockIdx.x;
   if (item < nItems) {
      const int l = (int) (item / nParts), t0 = (int) (item % nParts) * tilesPerCta;
      intStage<T>((const T *) a.x + (long long) l * a.inPitch + (long long) t0 * kTile, (long long) t0 * kTile,
                  inExtent, seg, A(0, 0), A(0, 1), tid);
   }
   for (; item < nItems && !failed; item += gridDim.x) {
      const int l = (int) (item / nParts);
      const int t0 = (int) (item % nParts) * tilesPerCta;
      const int t1 = min(nt, t0 + tilesPerCta);
      const T *x = (const T *) a.x + (long long) l * a.inPitch;
      T *y = (T *) a.y + (long long) l * a.outPitch;
      if (bandOf < 0 || (a.filtPitch != 0 && bandOf != l)) {
         const T *h = (const T *) a.h + (long long) l * a.filtPitch;
         __syncthreads(); // the previous band's last MMAs are complete (waited) before it changes
         for (int wd = tid; wd < gbWords; wd += kThreads) {
            uint32_t w0 = 0, w1 = 0;
#pragma unroll
            for (int j = 0; j < 4; j++) {
               const int c = 4 * wd + j - 16;
               const int g = (c >= 0 && c < T_) ? (int) h[T_ - 1 - c] : 0;
               if (SPLIT) {
                  w0 |= (uint32_t) ((g >> 8) & 0xFF) << (8 * j);
                  w1 |= (uint32_t) (g & 0xFF) << (8 * j);
               }
               else {
                  w0 |= (uint32_t) (g & 0xFF) << (8 * j);
               }
            }
            gb0[wd] = w0;
            if (SPLIT) gb1[wd] = w1;
         }
         __syncthreads();
         // Taps band, K-major no-swizzle: 16-byte chunk ch = 16q + 8i + r (byte 16 ch) holds
         // B[m = 16q + e][b = 8i + r] = g[16q + e - 8i - r], e < 16: bytes gb[16 + 16q - 8i - r + e],
         // gathered from five words with funnel shifts.
         for (int ch = tid; ch < Kt; ch += kThreads) {
            const int base = 16 + 16 * (ch >> 4) - 8 * ((ch >> 3) & 1) - (ch & 7);
            const int w = base >> 2, sh = (base & 3) * 8;
#pragma unroll
            for (int pl = 0; pl < (SPLIT ? 2 : 1); pl++) {
               const uint32_t *gb = pl ? gb1 : gb0;
               const uint32_t v0 = gb[w], v1 = gb[w + 1], v2 = gb[w + 2], v3 = gb[w + 3], v4 = gb[w + 4];
               uint4 o;
               o.x = __funnelshift_r(v0, v1, sh);
               o.y = __funnelshift_r(v1, v2, sh);
               o.z = __funnelshift_r(v2, v3, sh);
               o.w = __funnelshift_r(v3, v4, sh);
               *(uint4 *) ((pl ? B1 : B0) + 16 * ch) = o;
            }
         }
         bandOf = l;
      }
      for (int t = t0; t < t1; t++) {
         const long long j0 = (long long) t * kTile;
         tc::fenceProxyAsync();
         __syncthreads(); // segment[buf] and band written; previous accumulators drained
         if (tid == 0) {
            tc::fenceAfterSync();
            const uint32_t a0 = tc::smemAddr(A(buf, 0)), a1 = tc::smemAddr(A(buf, 1));
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
         // Fetch the next segment (this item's next tile, or the next item's first) into
         // registers now; it is written to shared memory after this tile's drain, so the
         // load latency hides behind the MMAs and the drain.
         constexpr int kPre = SPLIT ? 5 : 3; // 16-byte vectors per thread: (2048 + 2080) * sizeof(T) / 16 / 128
         int4 pre[kPre];
         const T *xn = nullptr;
         long long jn = 0;
         if (t + 1 < t1) {
            xn = x;
            jn = j0 + kTile;
         }
         else if (item + gridDim.x < nItems) {
            const long long ni = item + gridDim.x;
            xn = (const T *) a.x + (long long) (ni / nParts) * a.inPitch;
            jn = (long long) (ni % nParts) * tilesPerCta * kTile;
         }
         const bool preVec = xn != nullptr && ((((uintptr_t) (xn + jn)) & 15) == 0);
         const int nvec = seg * (int) sizeof(T) / 16;
         if (preVec) {
#pragma unroll
            for (int i = 0; i < kPre; i++) {
               const int k = tid + i * kThreads;
               if (k < nvec) pre[i] = loadSegVec<T>(xn + jn, k, inExtent - jn);
            }
         }
         const bool done = tc::mbarWait(mbar, iter & 1);
         if (!done && tid == 0) raiseError(a.err);
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
            __align__(16) T out[16];
            if (SPLIT && QMODE) {
               uint32_t w[8];
#pragma unroll
               for (int b = 0; b < 16; b += 2) {
                  const long long v0 = ((long long) (int) acc[0][b] << 16) + ((long long) (int) acc[1][b] << 8) +
                                       (long long) (int) acc[2][b];
                  const long long v1 = ((long long) (int) acc[0][b + 1] << 16) +
                                       ((long long) (int) acc[1][b + 1] << 8) + (long long) (int) acc[2][b + 1];
                  w[b / 2] = outStage16x2(v0, v1, a.shift);
               }
               *(uint4 *) &out[0] = make_uint4(w[0], w[1], w[2], w[3]);
               *(uint4 *) &out[8] = make_uint4(w[4], w[5], w[6], w[7]);
            }
            if (!SPLIT && QMODE) {
               uint4 w;
               w.x = outStage8x4((int) acc[0][0], (int) acc[0][1], (int) acc[0][2], (int) acc[0][3], a.shift);
               w.y = outStage8x4((int) acc[0][4], (int) acc[0][5], (int) acc[0][6], (int) acc[0][7], a.shift);
               w.z = outStage8x4((int) acc[0][8], (int) acc[0][9], (int) acc[0][10], (int) acc[0][11], a.shift);
               w.w = outStage8x4((int) acc[0][12], (int) acc[0][13], (int) acc[0][14], (int) acc[0][15], a.shift);
               *(uint4 *) &out[0] = w;
            }
#pragma unroll
            for (int b = 0; b < 16; b++) {
               long long v;
               if (!SPLIT) {
                  if (!QMODE) out[b] = (T) outStage8<QMODE>((int) acc[0][b], a.shift);
                  continue;
               }
               if (QMODE) continue; // packed above
               v = (long long) (int) (((uint32_t) acc[1][b] << 8) + (uint32_t) acc[2][b]);
               out[b] = outStage<T, QMODE>(v, a.shift);
            }
            int4 *os = (int4 *) (ostage + row * kPhases);
            os[0] = *(int4 *) &out[0];
            if (SPLIT) os[1] = *(int4 *) &out[8];
         }
         tc::fenceBeforeSync();
         if (failed) break;
         __syncthreads(); // the output tile is complete in shared memory
         storeTile<T>(y + j0, (int) min((long long) kTile, (long long) a.outSize - j0),
                      (const unsigned char *) ostage, [](int ci) { return ci * 16; }, tid, kThreads);
         if (preVec) {
            unsigned char *N0 = A(buf ^ 1, 0), *N1 = A(buf ^ 1, 1);
#pragma unroll
            for (int i = 0; i < kPre; i++) {
               const int k = tid + i * kThreads;
               if (k < nvec) putSegVec<T>(pre[i], k, N0, N1);
            }
         }
         else if (xn != nullptr) {
            intStage<T>(xn + jn, jn, inExtent, seg, A(buf ^ 1, 0), A(buf ^ 1, 1), tid); // unaligned row
         }
         buf ^= 1;
      }
   }
   __syncthreads();
   if (warp == 0) tc::tmemFree(tmem, kCols);
}

// Tiles per CTA (the built-in rule, when the autotuner has no entry): a whole channel
// when there are enough channels to fill the GPU several times over, else split so that
// at least ~2 waves of CTAs exist.
inline int tilesPerCtaFor(int nt, int batch, int ctasPerSm)
{
   const long long sms = deviceSms() > 0 ? deviceSms() : 148;
   int tpc = nt;
   while (tpc > 1 && (long long) ((nt + tpc - 1) / tpc) * batch < sms * ctasPerSm * 2) tpc = (tpc + 1) / 2;
   return tpc;
}

template <typename T> constexpr int intLaunchBound() { return sizeof(T) == 2 ? 6 : 8; }

template <typename T, int QMODE> cudaError_t launchIntTc(const FirLaunch &a, cudaStream_t s)
{
   constexpr bool SPLIT = sizeof(T) == 2;
   const int Kt = bandK(a.T);
   const int nplane = SPLIT ? 2 : 1;
   const size_t gbBytes = (size_t) ((Kt + 20) / 4) * 4 * nplane;
   const size_t smem = 16 + ((gbBytes + 15) & ~(size_t) 15) + (size_t) Kt * 16 * nplane +
                       2 * (size_t) nplane * (kTile + Kt) + (size_t) kTile * sizeof(T);
   auto fn = fir_int_tc_kernel<T, QMODE>;
   cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
   if (e != cudaSuccess) return e;
   const int nt = (a.outSize + kTile - 1) / kTile;
   const int tpc = a.tuneTpc > 0 ? (a.tuneTpc < nt ? a.tuneTpc : nt) : tilesPerCtaFor(nt, a.batch, 8);
   const long long items = (long long) a.batch * ((nt + tpc - 1) / tpc);
   // persistent: one wave of resident CTAs striding over the work items (CTAs per SM: the
   // autotuner's choice or the launch bound, fewer when shared memory runs out first)
   const int bySmem = (int) ((228u * 1024u) / (smem + 1024u));
   const int want = a.tunePerSm > 0 ? a.tunePerSm : intLaunchBound<T>();
   const int perSm = want < bySmem ? want : bySmem;
   const int sms = deviceSms() > 0 ? deviceSms() : 148;
   const long long wave = (long long) (perSm > 0 ? perSm : 1) * sms;
   const int grid = (int) (items < wave ? items : wave);
   FirLaunch k = a;
   // int8: |acc| <= 2048 * 2^14 = 2^25, so every shift from 27 up rounds to zero, as 31
   // (the largest the 32-bit output stage can take) does.
   if (!SPLIT && k.shift > 31) k.shift = 31;
   fn<<<grid, kThreads, smem, s>>>(k, tpc);
   countLaunch();
   return cudaGetLastError();
}

// ------------------------------------------------------------------ split-BF16x3

constexpr int kBfPhases = 64;
constexpr int kBfTile = kRows * kBfPhases;
constexpr int kBfMaxTaps = kFirBfMaxTaps;
static_assert(kBfTile == kFirBfTile, "ragged run tiles and kernel tiles must agree");
constexpr int kBfThreads = 512;
constexpr int kBfPadLeft = 64; // zero taps ahead of the reversed taps (phase offsets)

__host__ __device__ constexpr int bfK(int T) { return ((63 + T + 15) / 16) * 16; }
__host__ __device__ constexpr int bfBlocks(int T) { return kRows + (bfK(T) + 63) / 64; }
// 16-byte plane chunks staged per thread by bfStage
constexpr int kBfChunksPerThread = (bfBlocks(kBfMaxTaps) * 8 + kBfThreads - 1) / kBfThreads;
__host__ __device__ constexpr int bfTapSlots(int T) { return kBfPadLeft + bfK(T) + 8; }

__device__ __forceinline__ void splitBf16(float v, uint16_t &hi, uint16_t &lo)
{
   const __nv_bfloat16 h = __float2bfloat16_rn(v);
   const __nv_bfloat16 l = __float2bfloat16_rn(v - __bfloat162float(h));
   hi = __bfloat16_as_ushort(h);
   lo = __bfloat16_as_ushort(l);
}

// The same for two values at once, packed (a in the low half): one paired conversion
// per plane, rounding each value exactly as splitBf16 does.
__device__ __forceinline__ void splitBf16x2(float a, float b, uint32_t &hi, uint32_t &lo)
{
   const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
   const __nv_bfloat162 l = __floats2bfloat162_rn(a - __low2float(h), b - __high2float(h));
   hi = *(const uint32_t *) &h;
   lo = *(const uint32_t *) &l;
}

// Stage one tile's signal planes: sample i of the tile (64 per 128-byte block
// k = i / 64) goes to block k, 16-byte chunk c = (i % 64) / 8 stored at
// k*128 + ((c ^ (k & 7)) * 16), as hi and lo BF16.  Sample i is input index
// q0 + i of x, zero outside [0, inLen).  All loads of a thread are issued
// before any conversion so they overlap.
__device__ __forceinline__ void bfStage(const float *x, long long q0, long long inLen, int nb, unsigned char *Ahi,
                                        unsigned char *Alo, int tid)
{
   float f[kBfChunksPerThread][8];
   // chunk starts are 8 floats apart, so all share one misalignment (in floats)
   const int mis = (int) ((((uintptr_t) (x + q0)) >> 2) & 3);
#pragma unroll
   for (int u = 0; u < kBfChunksPerThread; u++) {
      const int cidx = tid + u * kBfThreads;
      if (cidx < nb * 8) {
         const long long q = q0 + (long long) (cidx >> 3) * 64 + (cidx & 7) * 8;
         if (mis == 0 && q >= 0 && q + 8 <= inLen) {
            *(float4 *) &f[u][0] = *(const float4 *) (x + q);
            *(float4 *) &f[u][4] = *(const float4 *) (x + q + 4);
         }
         else if (mis != 0 && q - mis >= 0 && q - mis + 12 <= inLen) {
            // three aligned vectors around the chunk, then pick its 8 samples
            const float4 a = *(const float4 *) (x + q - mis);
            const float4 b = *(const float4 *) (x + q - mis + 4);
            const float4 cc = *(const float4 *) (x + q - mis + 8);
            const float w[12] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, cc.x, cc.y, cc.z, cc.w};
#pragma unroll
            for (int e = 0; e < 8; e++) f[u][e] = mis == 1 ? w[1 + e] : (mis == 2 ? w[2 + e] : w[3 + e]);
         }
         else {
#pragma unroll
            for (int e = 0; e < 8; e++) f[u][e] = (q + e >= 0 && q + e < inLen) ? x[q + e] : 0.0f;
         }
      }
   }
#pragma unroll
   for (int u = 0; u < kBfChunksPerThread; u++) {
      const int cidx = tid + u * kBfThreads;
      if (cidx < nb * 8) {
         const int k = cidx >> 3, c = cidx & 7;
         uint4 hv, lv;
         splitBf16x2(f[u][0], f[u][1], hv.x, lv.x);
         splitBf16x2(f[u][2], f[u][3], hv.y, lv.y);
         splitBf16x2(f[u][4], f[u][5], hv.z, lv.z);
         splitBf16x2(f[u][6], f[u][7], hv.w, lv.w);
         const int off = k * 128 + ((c ^ (k & 7)) << 4);
         *(uint4 *) (Ahi + off) = hv;
         *(uint4 *) (Alo + off) = lv;
      }
   }
}

// Raw FP32 tiles (nb blocks of 64 samples) are bulk-copied by the TMA engine
// when the whole tile lies inside the input and is 16-byte aligned, then split
// in shared memory; other tiles (row edges, unaligned rows) are staged by the
// threads straight into the planes (bfStage).
// Split a raw tile into the signal planes: sample i (64 per 128-byte block
// k = i / 64) goes to block k, 16-byte chunk c = (i % 64) / 8 stored at
// k*128 + ((c ^ (k & 7)) * 16), as hi and lo BF16.  Sample i is raw[mis + i]
// (mis < 4: the bulk copy started at the 16-byte boundary below the tile).  A
// thread takes 4 samples (consecutive lanes, consecutive addresses) and writes
// half a chunk of each plane.
__device__ __forceinline__ void bfSplit(const float *raw, int mis, int nb, unsigned char *Ahi, unsigned char *Alo,
                                        int tid)
{
   for (int f = tid; f < nb * 16; f += kBfThreads) {
      float4 v;
      if (mis == 0) v = ((const float4 *) raw)[f];
      else {
         const float *p = raw + mis + 4 * f;
         v = make_float4(p[0], p[1], p[2], p[3]);
      }
      const int k = f >> 4, c = (f >> 1) & 7, half = f & 1;
      uint2 hv, lv;
      splitBf16x2(v.x, v.y, hv.x, lv.x);
      splitBf16x2(v.z, v.w, hv.y, lv.y);
      const int off = k * 128 + ((c ^ (k & 7)) << 4) + half * 8;
      *(uint2 *) (Ahi + off) = hv;
      *(uint2 *) (Alo + off) = lv;
   }
}

// A run of consecutive output tiles [t0, t1) of one channel:
//     y[j] = sum_{c<T} x[inShift + j + c] * g(c),  x zero outside [0, inLen),
//     g(c) = h[T-1-c] (reverse = 1: DSPLIB_fir correlation order) or h[c] (reverse = 0).
struct BfRun {
   const float *x;
   const float *h;
   float *y;
   long long inShift, inLen;
   int outLen, T, reverse, t0, t1;
   int *err; // error word for an expired bounded wait
};

// Shared memory for taps up to Tmax: two sets of hi/lo signal planes (tile t is
// split into set t % 2 while the tensor core reads the other; a drained tile's set
// also stages its output), a ring of raw FP32 tiles fetched by the TMA engine ahead
// of their split (up to two when they fit beside the band, none for the longest
// taps: those tiles are staged by the threads straight from global memory), the
// taps band and the split taps.  Two accumulators of 128 TMEM columns each.
//
// Warp roles: warps 0-15 (the workers) build the band, split tiles into the planes
// and drain the accumulators; warp 16 issues the MMAs.  The issuing thread may stall
// in tcgen05.mma while the tensor core is busy, so it has a warp of its own.
// Handshakes: planesFull[b] (a worker arrives once plane set b holds a tile and
// accumulator b is free) and mmaDone[b] (tcgen05.commit once the MMAs reading set b
// and writing accumulator b completed); the workers synchronise among themselves on
// named barrier 1.
constexpr size_t kBfSmemLimit = 227 * 1024;
constexpr uint32_t kBfTmemCols = 256;
constexpr int kBfWorkers = kBfThreads;         // worker threads (16 warps)
constexpr int kBfBlock = kBfWorkers + 32;      // + the MMA warp
constexpr uint32_t kBfBar = 1;                 // the workers' named barrier
// Layout for taps up to T (the batched kernels lay out shared memory per run, for that
// run's taps, in an allocation of kBfSmemLimit): the barriers and the TMEM slot in the
// first 1024 bytes, then the plane sets, the raw ring, the band and the split taps.
__host__ __device__ constexpr size_t bfPlaneBytes(int T) { return (size_t) ((bfBlocks(T) * 128 + 1023) & ~1023); }
// a raw tile and the up to 3 samples before it (copies start on a 16-byte boundary),
// padded to 128 bytes so that the band behind the ring keeps its 128-byte alignment
__host__ __device__ constexpr size_t bfRawBytes(int T) { return (size_t) bfBlocks(T) * 256 + 128; }
__host__ __device__ constexpr size_t bfSmemBytesFor(int T, int stages)
{
   return 2048 + 4 * bfPlaneBytes(T) + stages * bfRawBytes(T) + (size_t) bfK(T) * 256 + 4 * (size_t) bfTapSlots(T);
}
__host__ __device__ inline int bfStages(int T)
{
   return bfSmemBytesFor(T, 2) <= kBfSmemLimit ? 2 : (bfSmemBytesFor(T, 1) <= kBfSmemLimit ? 1 : 0);
}
__host__ __device__ inline size_t bfSmemBytes(int T) { return bfSmemBytesFor(T, bfStages(T)); }
static_assert(bfSmemBytesFor(kBfMaxTaps, 0) <= kBfSmemLimit, "two plane sets and the longest band fit");

struct BfSmem {
   unsigned char *sets; // plane set b: hi at sets + 2 b planeBytes, lo planeBytes further (1024-byte aligned)
   size_t planeBytes;
   float *raw;          // stages x rawFloats
   int rawFloats, stages;
   unsigned char *Bt;
   uint16_t *gHi, *gLo;
   uint64_t *mbar, *planesFull, *full; // MMA completion and plane-set readiness per accumulator; raw tiles
   uint32_t *tslot;
   __device__ float *slot(int k) const { return raw + (size_t) k * rawFloats; }
   __device__ unsigned char *hi(int b) const { return sets + (size_t) (2 * b) * planeBytes; }
   __device__ unsigned char *lo(int b) const { return sets + (size_t) (2 * b + 1) * planeBytes; }
};

__device__ __forceinline__ BfSmem bfSmemLayout(unsigned char *smraw, int T)
{
   BfSmem L;
   unsigned char *sm = (unsigned char *) (((uintptr_t) smraw + 1023) & ~(uintptr_t) 1023);
   L.mbar = (uint64_t *) sm;
   L.planesFull = L.mbar + 2;
   L.full = L.planesFull + 2;
   L.tslot = (uint32_t *) (L.full + 2);
   const size_t pb = bfPlaneBytes(T);
   L.stages = bfStages(T);
   L.planeBytes = pb;
   L.sets = sm + 1024;
   L.raw = (float *) (L.sets + 4 * pb);
   L.rawFloats = (int) (bfRawBytes(T) / 4);
   L.Bt = (unsigned char *) L.raw + (size_t) L.stages * bfRawBytes(T);
   L.gHi = (uint16_t *) (L.Bt + (size_t) bfK(T) * 256); // split taps with zero padding
   L.gLo = L.gHi + bfTapSlots(T);
   return L;
}

// The workers' barrier phases and copies in flight, carried across the runs of one CTA.
struct BfPipe {
   uint32_t tiles = 0;   // tiles split so far: tile n uses plane set and accumulator n % 2
   uint32_t mmaPar = 0;  // mmaDone phase, one bit per accumulator
   uint32_t par = 0;     // raw-tile barrier phase, one bit per stage
   uint32_t pending = 0; // stages with a bulk copy issued and not yet waited for
};

// The MMA thread's state.
struct BfIssuer {
   uint32_t tiles = 0;
   uint32_t pfPar = 0;          // planesFull phase, one bit per accumulator
   uint32_t commits0 = 0, commits1 = 0; // commits per accumulator
};

// Workers: wait for the MMAs of accumulator b (bounded; thread 0 waits, the barrier
// releases the rest).
__device__ __forceinline__ bool bfWaitMma(const BfSmem &L, BfPipe &pp, int b, int *err, int tid)
{
   const bool done = tid == 0 ? tc::mbarWait(L.mbar + b, (pp.mmaPar >> b) & 1) : true;
   pp.mmaPar ^= 1u << b;
   if (!done && tid == 0) raiseError(err);
   return !tc::namedSyncOr(kBfBar, kBfWorkers, !done);
}

// Workers: drain accumulator b (output tile t of run r, its MMAs complete) through
// plane set b into y.
__device__ __forceinline__ void bfDrain(const BfRun &r, const BfSmem &L, uint32_t tmem, int b, int t, int tid)
{
   const int warp = tid >> 5, lane = tid & 31;
   tc::fenceAfterSync();
   const long long j0 = (long long) t * kBfTile;
   unsigned char *stage = L.hi(b); // the set spans both planes: 2 * planeBytes >= 32 KB
   {
      // Warp w drains TMEM lane quadrant w % 4 (rows a) and output quarter qt = w / 4
      // (16 phases): y[j0 + 64a + 16*qt + b] = D[a][16*qt + b] + D[a][64 + 16*qt + b].
      const int quad = warp & 3, qt = warp >> 2, half = qt >> 1;
      const uint32_t acc = tmem + (uint32_t) b * 128 + ((uint32_t) (quad * 32) << 16);
      const int row = quad * 32 + lane;
      // 16-byte chunk v4 of row half (row, half) rotated to slot (v4 + row) & 7 so that
      // eight consecutive rows store to distinct banks.  Two passes of 8 columns keep
      // the register footprint small.
      float *os = (float *) stage + row * kBfPhases + half * 32;
#pragma unroll
      for (int h8 = 0; h8 < 2; h8++) {
         uint32_t a[8], c[8];
         tc::tmemLoad8(acc + qt * 16 + h8 * 8, a);
         tc::tmemLoad8(acc + 64 + qt * 16 + h8 * 8, c);
         tc::tmemWaitLoad();
#pragma unroll
         for (int v = 0; v < 2; v++) {
            const int v4 = (qt & 1) * 4 + h8 * 2 + v;
            float4 o;
            o.x = __uint_as_float(a[4 * v + 0]) + __uint_as_float(c[4 * v + 0]);
            o.y = __uint_as_float(a[4 * v + 1]) + __uint_as_float(c[4 * v + 1]);
            o.z = __uint_as_float(a[4 * v + 2]) + __uint_as_float(c[4 * v + 2]);
            o.w = __uint_as_float(a[4 * v + 3]) + __uint_as_float(c[4 * v + 3]);
            *(float4 *) (os + (((v4 + row) & 7) << 2)) = o;
         }
      }
   }
   tc::fenceBeforeSync();
   tc::namedSync(kBfBar, kBfWorkers); // the output tile is complete in shared memory; the accumulator is free
   storeTile<float>(r.y + j0, (int) min((long long) kBfTile, (long long) r.outLen - j0), (const unsigned char *) stage,
                    [](int ci) {
                       const int row = ci >> 4, half = (ci >> 3) & 1, v4 = ci & 7;
                       return (row * kBfPhases + half * 32 + (((v4 + row) & 7) << 2)) * 4;
                    },
                    tid, kBfWorkers);
   tc::namedSync(kBfBar, kBfWorkers); // the staged output has left plane set b: it may be split into again
}

// Workers: build the taps band of run r, then split its tiles into alternate plane
// sets (handing each to the MMA warp) and drain tile t - 1 while tile t's MMAs run.
// Returns false when a bounded wait gave up.
__device__ __forceinline__ bool bfWork(const BfRun &r, const BfSmem &L, uint32_t tmem, BfPipe &pp, int tid)
{
   const int T_ = r.T;
   const int Kt = bfK(T_);
   const int nb = bfBlocks(T_);
   const int slots = bfTapSlots(T_);
   const int S = L.stages;
   auto q0 = [&](int t) { return r.inShift + (long long) t * kBfTile; };
   // Blocks of tile t the MMAs read for its valid output rows (a short last tile needs
   // fewer; the rows beyond are computed from stale planes and never stored).
   auto blocksOf = [&](int t) {
      const int outs = (int) min((long long) kBfTile, (long long) r.outLen - (long long) t * kBfTile);
      return min(nb, (outs + kBfPhases - 1) / kBfPhases + (Kt + 63) / 64);
   };
   // samples between the 16-byte boundary at or below the tile's first input and that input
   auto misOf = [&](int t) { return (int) ((((long long) ((uintptr_t) r.x >> 2)) + q0(t)) & 3); };
   auto bytesOf = [&](int t) { return (uint32_t) blocksOf(t) * 256u + (misOf(t) ? 16u : 0u); };
   // The raw window of tile t is [w0, w0 + bytes / 4), w0 = q - mis on a 16-byte boundary.
   // The bulk copy takes its part inside the input, [lo, hi), both ends on 16-byte
   // boundaries (window offsets multiples of 4 samples); the threads write the rest:
   // the up to 3 samples beside each end and the zeros outside the input.
   auto bulkLo = [&](int t) {
      const long long w0 = q0(t) - misOf(t);
      return w0 >= 0 ? w0 : w0 + ((-w0 + 3) & ~3LL);
   };
   auto bulkHi = [&](int t) {
      const long long w0 = q0(t) - misOf(t), end = min(w0 + (long long) (bytesOf(t) / 4), r.inLen);
      return w0 + ((end - w0) & ~3LL);
   };
   auto bulkOk = [&](int t) { return S > 0 && bulkHi(t) > bulkLo(t); };
   auto fetch = [&](int t, int k) {
      const long long w0 = q0(t) - misOf(t), lo = bulkLo(t), hi = bulkHi(t);
      tc::mbarExpectTx(L.full + k, (uint32_t) (hi - lo) * 4u);
      tc::bulkLoad(L.slot(k) + (lo - w0), r.x + lo, (uint32_t) (hi - lo) * 4u, L.full + k);
   };
   // the window's samples outside the bulk range: input values or zeros beyond it
   auto fixEdges = [&](int t, int k) {
      const long long w0 = q0(t) - misOf(t), lo = bulkLo(t), hi = bulkHi(t);
      const int W = (int) (bytesOf(t) / 4);
      float *raw = L.slot(k);
      for (int i = tid; i < (int) (lo - w0); i += kBfWorkers) {
         const long long q = w0 + i;
         raw[i] = (q >= 0 && q < r.inLen) ? r.x[q] : 0.0f;
      }
      for (int i = (int) (hi - w0) + tid; i < W; i += kBfWorkers) {
         const long long q = w0 + i;
         raw[i] = (q >= 0 && q < r.inLen) ? r.x[q] : 0.0f;
      }
   };
   // The first raw tiles are fetched while the taps band is built.  (Every MMA of the
   // previous run completed: its last tile was drained.)
   if (tid == 0)
      for (int k = 0; k < S && r.t0 + k < r.t1; k++)
         if (bulkOk(r.t0 + k)) fetch(r.t0 + k, k);
   for (int k = 0; k < S && r.t0 + k < r.t1; k++)
      if (bulkOk(r.t0 + k)) pp.pending |= 1u << k;
   // g[c] split into hi/lo, stored at slot c + kBfPadLeft; zero elsewhere.
   for (int sl = tid; sl < slots; sl += kBfWorkers) {
      const int c = sl - kBfPadLeft;
      uint16_t hi = 0, lo = 0;
      if (c >= 0 && c < T_) splitBf16(r.reverse ? r.h[T_ - 1 - c] : r.h[c], hi, lo);
      L.gHi[sl] = hi;
      L.gLo[sl] = lo;
   }
   tc::namedSync(kBfBar, kBfWorkers);
   // Taps band, K-major no swizzle: 16-byte chunk (q, n) at q*2048 + (n/8)*128 + (n%8)*16 holds
   // B[8q .. 8q+7][n]; rows n < 64: g_hi[m - n], rows n >= 64: g_lo[m - (n - 64)].
   // Each chunk is 8 consecutive split taps from an arbitrary element offset o: the two
   // aligned 16-byte vectors around it, shifted into place (funnel shifts by 16 bits for
   // odd offsets), instead of 8 scalar reads.
   for (int cidx = tid; cidx < (Kt / 8) * 128; cidx += kBfWorkers) {
      const int q = cidx >> 7, n = cidx & 127;
      const int o = kBfPadLeft + 8 * q - (n & 63);
      const uint4 *base = (const uint4 *) (n < 64 ? L.gHi : L.gLo) + (o >> 3);
      const uint4 lo4 = base[0], hi4 = base[1];
      const int rr = o & 7, h = rr >> 1;
      // words h .. h + 4 of the 8 (selects, not an indexed array: it stays in registers)
      const uint32_t w0 = h == 0 ? lo4.x : h == 1 ? lo4.y : h == 2 ? lo4.z : lo4.w;
      const uint32_t w1 = h == 0 ? lo4.y : h == 1 ? lo4.z : h == 2 ? lo4.w : hi4.x;
      const uint32_t w2 = h == 0 ? lo4.z : h == 1 ? lo4.w : h == 2 ? hi4.x : hi4.y;
      const uint32_t w3 = h == 0 ? lo4.w : h == 1 ? hi4.x : h == 2 ? hi4.y : hi4.z;
      const uint32_t w4 = h == 0 ? hi4.x : h == 1 ? hi4.y : h == 2 ? hi4.z : hi4.w;
      uint4 v;
      if (rr & 1) {
         v.x = __funnelshift_r(w0, w1, 16);
         v.y = __funnelshift_r(w1, w2, 16);
         v.z = __funnelshift_r(w2, w3, 16);
         v.w = __funnelshift_r(w3, w4, 16);
      }
      else {
         v.x = w0;
         v.y = w1;
         v.z = w2;
         v.w = w3;
      }
      *(uint4 *) (L.Bt + q * 2048 + (n >> 3) * 128 + (n & 7) * 16) = v;
   }
   for (int t = r.t0; t <= r.t1; t++) {
      const int cur = (int) (pp.tiles & 1), prev = cur ^ 1;
      if (t < r.t1) {
         // plane set and accumulator cur are free: tile t - 2 was drained
         const int k = S > 0 ? (t - r.t0) % S : 0;
         bool ok = true;
         const bool viaBulk = bulkOk(t);
         if (viaBulk) {
            ok = tid == 0 ? tc::mbarWait(L.full + k, (pp.par >> k) & 1) : true; // the barrier below releases the rest
            pp.par ^= 1u << k;
            pp.pending &= ~(1u << k);
         }
         if (!ok && tid == 0) raiseError(r.err);
         if (viaBulk) fixEdges(t, k);
         if (tc::namedSyncOr(kBfBar, kBfWorkers, !ok)) return false; // the raw tile landed (and the band is built)
         if (viaBulk) bfSplit(L.slot(k), misOf(t), blocksOf(t), L.hi(cur), L.lo(cur), tid);
         else bfStage(r.x, q0(t), r.inLen, blocksOf(t), L.hi(cur), L.lo(cur), tid); // straight from global memory
         tc::fenceProxyAsync();
         tc::fenceBeforeSync();
         tc::namedSync(kBfBar, kBfWorkers); // planes (and band) written; the raw stage is free again
         if (tid == 0) tc::mbarArrive(L.planesFull + cur);
         if (t + S < r.t1 && bulkOk(t + S)) {
            if (tid == 0) fetch(t + S, k);
            pp.pending |= 1u << k;
         }
         pp.tiles++;
      }
      if (t > r.t0) {
         // tile t - 1 (accumulator and plane set prev) while tile t's MMAs run
         if (!bfWaitMma(L, pp, prev, r.err, tid)) return false;
         bfDrain(r, L, tmem, prev, t - 1, tid);
      }
   }
   return true;
}

// MMA thread: for each tile of run r, once its plane set is full, the Toeplitz
// contraction into the tile's accumulator and a commit to its mmaDone barrier.
__device__ __forceinline__ bool bfIssue(const BfRun &r, const BfSmem &L, uint32_t tmem, BfIssuer &mi)
{
   const int Kt = bfK(r.T);
   const uint32_t bt = tc::smemAddr(L.Bt);
   const uint32_t id128 = tc::idesc(1, 1, 1, kRows, 128);
   for (int t = r.t0; t < r.t1; t++) {
      const int b = (int) (mi.tiles & 1);
      if (!tc::mbarWait(L.planesFull + b, (mi.pfPar >> b) & 1)) {
         raiseError(r.err);
         return false;
      }
      mi.pfPar ^= 1u << b;
      tc::fenceAfterSync();
      const uint32_t ahi = tc::smemAddr(L.hi(b)), alo = tc::smemAddr(L.lo(b));
      const uint32_t d = tmem + (uint32_t) b * 128;
      for (int k16 = 0; k16 < Kt / 16; k16++) {
         const int blk = k16 >> 2, sub = k16 & 3;
         // The swizzle is applied on absolute shared-memory address bits, so a start
         // that is not atom-aligned (block blk of the plane) keeps base offset 0.
         const uint64_t dHi = tc::descSw128(ahi + blk * 128 + sub * 32, 1024, 0);
         const uint64_t dLo = tc::descSw128(alo + blk * 128 + sub * 32, 1024, 0);
         const uint64_t dB = tc::descNoSwizzle(bt + k16 * 4096, 2048, 128);
         tc::mmaF16(d, dHi, dB, id128, k16 > 0);
         tc::mmaF16(d, dLo, dB, id128, true);
      }
      tc::commit(L.mbar + b);
      if (b) mi.commits1++;
      else mi.commits0++;
      mi.tiles++;
   }
   return true;
}

// Set-up and tear-down shared by the bf16x3 kernels.
__device__ __forceinline__ uint32_t bfBegin(const BfSmem &L, int tid)
{
   if ((tid >> 5) == 0) tc::tmemAlloc(L.tslot, kBfTmemCols);
   if (tid == 0) {
      for (int k = 0; k < 2; k++) tc::mbarInit(L.mbar + k, 1);
      for (int k = 0; k < 2; k++) tc::mbarInit(L.planesFull + k, 1);
      for (int k = 0; k < 2; k++) tc::mbarInit(L.full + k, 1);
      tc::fenceMbarInit();
   }
   tc::fenceBeforeSync();
   __syncthreads();
   tc::fenceAfterSync();
   return *L.tslot;
}

// After the roles' loops (also after a failure): the MMA thread waits (bounded) for its
// last commit on each accumulator, worker 0 for the bulk copies still in flight; then
// the accumulators are released.
__device__ __forceinline__ void bfEnd(const BfSmem &L, const BfPipe &pp, const BfIssuer &mi, uint32_t tmem, int tid)
{
   if (tid == kBfWorkers) {
      if (mi.commits0) (void) tc::mbarWait(L.mbar, (mi.commits0 - 1) & 1);
      if (mi.commits1) (void) tc::mbarWait(L.mbar + 1, (mi.commits1 - 1) & 1);
   }
   if (tid == 0)
      for (int k = 0; k < 2; k++)
         if ((pp.pending >> k) & 1) (void) tc::mbarWait(L.full + k, (pp.par >> k) & 1);
   tc::fenceBeforeSync();
   __syncthreads();
   tc::fenceAfterSync();
   if ((tid >> 5) == 0) tc::tmemFree(tmem, kBfTmemCols);
}

__global__ void __launch_bounds__(kBfBlock, 1) fir_bf16x3_tc_kernel(FirLaunch a, int tilesPerCta)
{
   extern __shared__ __align__(16) unsigned char smraw[];
   const BfSmem L = bfSmemLayout(smraw, a.T);
   const int tid = threadIdx.x;
   const uint32_t tmem = bfBegin(L, tid);
   const int nt = (a.outSize + kBfTile - 1) / kBfTile;
   BfPipe pp;
   BfIssuer mi;
   if (tid < kBfWorkers || tid == kBfWorkers)
      for (int l = blockIdx.y; l < a.batch; l += gridDim.y) {
         BfRun r;
         r.x = (const float *) a.x + (long long) l * a.inPitch;
         r.h = (const float *) a.h + (long long) l * a.filtPitch;
         r.y = (float *) a.y + (long long) l * a.outPitch;
         r.inShift = 0;
         r.inLen = (long long) a.outSize + a.T - 1;
         r.outLen = a.outSize;
         r.T = a.T;
         r.reverse = 1;
         r.t0 = blockIdx.x * tilesPerCta;
         r.t1 = min(nt, r.t0 + tilesPerCta);
         r.err = a.err;
         if (!(tid < kBfWorkers ? bfWork(r, L, tmem, pp, tid) : bfIssue(r, L, tmem, mi))) break;
      }
   bfEnd(L, pp, mi, tmem, tid);
}

// Work lists of the batched filter bank: runs of up to kFirBfRunTiles tiles of one
// channel, longest first, taken in turn by one persistent CTA per SM.  DX = false:
// forward, y = valid correlation of x with the taps (DSPLIB_fir order); DX = true:
// input gradient, the full convolution of the output gradient with the taps.
__global__ void __launch_bounds__(kBfBlock, 1)
    fir_bf16x3_ragged_kernel(const RaggedChan *chans, const int4 *runs, int nRuns, const float *in,
                             const float *taps, float *out, int dx, int Tmax, int *err)
{
   extern __shared__ __align__(16) unsigned char smraw[];
   // barriers and the TMEM slot sit at fixed offsets; the rest is laid out per run
   const BfSmem L = bfSmemLayout(smraw, Tmax);
   const int tid = threadIdx.x;
   const uint32_t tmem = bfBegin(L, tid);
   BfPipe pp;
   BfIssuer mi;
   if (tid < kBfWorkers || tid == kBfWorkers)
      for (int i = blockIdx.x; i < nRuns; i += gridDim.x) {
         const int4 it = runs[i];
         const RaggedChan c = chans[it.x];
         const BfSmem Lr = bfSmemLayout(smraw, c.T);
         BfRun r;
         r.x = in + c.xOff;
         r.h = taps + c.hOff;
         r.y = out + (dx ? c.xOff : c.pOff); // forward: plane 0 of the work buffer
         r.T = c.T;
         r.inShift = dx ? -(long long) (c.T - 1) : 0;
         r.inLen = dx ? c.L - c.T + 1 : c.L;
         r.outLen = dx ? c.L : c.L - c.T + 1;
         r.reverse = dx ? 0 : 1;
         r.t0 = it.y;
         r.t1 = it.y + it.z;
         r.err = err;
         if (!(tid < kBfWorkers ? bfWork(r, Lr, tmem, pp, tid) : bfIssue(r, Lr, tmem, mi))) break;
      }
   bfEnd(L, pp, mi, tmem, tid);
}


// ------------------------------------------------------------------ taps gradient (split-BF16x3)

// Taps gradient of the filter bank, dh_lag[c] = sum_j gu[j] x[j + c] (c < T), on the
// tensor cores.  With j = 64 r + s (row r, phase s) and t' = c + s:
//     D[t'][s] = sum_r x[64 r + t'] gu[64 r + s],      dh_lag[c] = sum_s D[c + s][s],
// a GEMM whose contraction runs over the rows r (time) and whose operands are both
// the signal planes as staged for the forward kernels, read MN-major: A = X^T
// (M = 128 positions t', 64 per 128-byte block, block r + t'/64 of the x plane, so the
// second 64-wide atom of a tile starts one block (128 bytes) after the first), B = G
// (N = 64 phases, block r of the gradient plane).  One accumulator tile per 128
// positions (ceil((T + 63) / 128) <= 5 tiles of 64 TMEM columns) collects the three
// split products x_hi g_hi + x_lo g_hi + x_hi g_lo over every row of a run of up to
// four 8192-sample tiles; the diagonal sums are taken once per run, in a fixed order.
// The next tile's planes are staged while the tensor core works on the current one.
constexpr int kDhTile = kBfTile;                  // samples (128 rows) per staged tile
constexpr int kDhMaxMt = (kBfMaxTaps + 63 + 127) / 128;
constexpr int kDhXBlocks = 127 + 2 * kDhMaxMt;    // x blocks a tile's A operands reach
constexpr size_t kDhXPlane = ((kDhXBlocks * 128 + 1023) / 1024) * 1024;
constexpr size_t kDhGPlane = kRows * 128;
constexpr size_t kDhBuf = 2 * kDhXPlane + 2 * kDhGPlane; // x hi, x lo, g hi, g lo
constexpr size_t kDhSmem = 1024 + 2 * kDhBuf + 64;
constexpr int kDhPitch = 65;                      // floats per staged accumulator row
static_assert((size_t) kRows * kDhPitch * 4 <= kDhBuf, "accumulator staging fits one buffer");
static_assert(kDhMaxMt * 64 <= 512, "accumulator tiles fit the TMEM columns");

// MN-major operand with 128-byte swizzle: 64-element atoms (128-byte rows, 8 rows per
// 1024-byte swizzle atom along K), lbo = byte distance between atoms along M/N,
// sbo = byte distance between 8-row groups along K.
__device__ __forceinline__ uint64_t descSw128Mn(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
   uint64_t d = 0;
   d |= (uint64_t) ((saddr >> 4) & 0x3FFF);
   d |= (uint64_t) ((lbo >> 4) & 0x3FFF) << 16;
   d |= (uint64_t) ((sbo >> 4) & 0x3FFF) << 32;
   d |= (uint64_t) 1 << 46;
   d |= (uint64_t) 2 << 61;
   return d;
}

// Warp roles as in the split-BF16x3 FIR: warps 0-15 stage tiles into the two buffers
// (planesFull[b] when buffer b holds tile k) and form the diagonal sums at the end; warp 16
// issues the MMAs (mmaDone[b] when tile k's MMAs, reading buffer b, completed).
__global__ void __launch_bounds__(kBfBlock, 1)
    fir_dh_bf16x3_kernel(const RaggedChan *chans, const int4 *runs, const float *x, const float *gu, float *part,
                         int *err)
{
   extern __shared__ __align__(16) unsigned char smraw[];
   unsigned char *sm = (unsigned char *) (((uintptr_t) smraw + 1023) & ~(uintptr_t) 1023);
   uint64_t *mbar = (uint64_t *) (sm + 2 * kDhBuf); // mmaDone, one per buffer
   uint64_t *full = mbar + 2;                        // planesFull, one per buffer
   uint32_t *tslot = (uint32_t *) (full + 2);
   const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
   const int4 run = runs[blockIdx.x]; // {channel, first tile, tiles, partial slot}
   const RaggedChan c = chans[run.x];
   const int T = c.T;
   const int Mt = (T + 63 + 127) / 128;
   const int nbX = 127 + 2 * Mt;
   const float *xc = x + c.xOff, *gc = gu + c.xOff;
   auto buf = [&](int b) { return sm + (size_t) b * kDhBuf; };
   auto stage = [&](int t, int b) {
      unsigned char *B = buf(b);
      const long long q0 = (long long) t * kDhTile;
      bfStage(xc, q0, c.L, nbX, B, B + kDhXPlane, tid);
      bfStage(gc, q0, c.Lu, kRows, B + 2 * kDhXPlane, B + 2 * kDhXPlane + kDhGPlane, tid);
   };
   if (warp == 0) tc::tmemAlloc(tslot, 512);
   if (tid == 0) {
      for (int k = 0; k < 2; k++) {
         tc::mbarInit(mbar + k, 1);
         tc::mbarInit(full + k, 1);
      }
      tc::fenceMbarInit();
   }
   tc::fenceBeforeSync();
   __syncthreads();
   tc::fenceAfterSync();
   const uint32_t tmem = *tslot;
   bool fail = false;
   if (tid < kBfWorkers) {
      uint32_t par = 0; // mmaDone phase, one bit per buffer
      for (int k = 0; k < run.z; k++) {
         const int b = k & 1;
         if (k >= 2) { // buffer b is free once tile k - 2's MMAs completed
            const bool done = tid == 0 ? tc::mbarWait(mbar + b, (par >> b) & 1) : true;
            par ^= 1u << b;
            if (!done && tid == 0) raiseError(err);
            if (tc::namedSyncOr(kBfBar, kBfWorkers, !done)) {
               fail = true;
               break;
            }
         }
         stage(run.y + k, b);
         tc::fenceProxyAsync();
         tc::namedSync(kBfBar, kBfWorkers);
         if (tid == 0) tc::mbarArrive(full + b);
      }
      // the last two tiles (bounded: after a failure, waits for tiles never issued give up)
      for (int k = run.z >= 2 ? run.z - 2 : 0; !fail && k < run.z; k++) {
         const int b = k & 1;
         const bool done = tid == 0 ? tc::mbarWait(mbar + b, (par >> b) & 1) : true;
         par ^= 1u << b;
         if (!done && tid == 0) {
            raiseError(err);
            fail = true;
         }
      }
   }
   else if (tid == kBfWorkers) {
      const uint32_t id = tc::idesc(1, 1, 1, kRows, 64) | (1u << 15) | (1u << 16); // both operands MN-major
      uint32_t pf = 0;                                                               // planesFull phase per buffer
      int commits = 0;
      for (int k = 0; k < run.z; k++) {
         const int b = k & 1;
         if (!tc::mbarWait(full + b, (pf >> b) & 1)) {
            raiseError(err);
            fail = true;
            break;
         }
         pf ^= 1u << b;
         tc::fenceAfterSync();
         unsigned char *B = buf(b);
         const uint32_t xh = tc::smemAddr(B), xl = tc::smemAddr(B + kDhXPlane);
         const uint32_t gh = tc::smemAddr(B + 2 * kDhXPlane), gl = tc::smemAddr(B + 2 * kDhXPlane + kDhGPlane);
         for (int ks = 0; ks < kRows / 16; ks++) {
            const uint64_t dGh = descSw128Mn(gh + ks * 2048, 128, 1024);
            const uint64_t dGl = descSw128Mn(gl + ks * 2048, 128, 1024);
            for (int m = 0; m < Mt; m++) {
               const uint32_t off = (uint32_t) (ks * 16 + 2 * m) * 128;
               const uint64_t dXh = descSw128Mn(xh + off, 128, 1024);
               const uint64_t dXl = descSw128Mn(xl + off, 128, 1024);
               const uint32_t d = tmem + 64 * m;
               tc::mmaF16(d, dXh, dGh, id, k > 0 || ks > 0);
               tc::mmaF16(d, dXl, dGh, id, true);
               tc::mmaF16(d, dXh, dGl, id, true);
            }
         }
         tc::commit(mbar + b);
         commits++;
      }
      // after a failure: let the MMAs already committed finish before TMEM is released
      // (tile n commits phase n / 2 of barrier n % 2)
      if (fail)
         for (int n = commits >= 2 ? commits - 2 : 0; n < commits; n++) (void) tc::mbarWait(mbar + (n & 1), (n >> 1) & 1);
   }
   if (__syncthreads_or(fail)) {
      tc::fenceAfterSync();
      if (warp == 0) tc::tmemFree(tmem, 512);
      return;
   }
   tc::fenceAfterSync();
   // diagonal sums: lag c (thread c) adds D[c + s][s] over s, accumulator tile by tile
   float acc = 0.0f;
   float *Ds = (float *) buf(0);
   for (int m = 0; m < Mt; m++) {
      if (warp < 16) {
         const int quad = warp & 3, cg = warp >> 2; // TMEM lanes 32 quad.., columns 16 cg..
         uint32_t r[16];
         tc::tmemLoad16(tmem + ((uint32_t) (quad * 32) << 16) + 64 * m + 16 * cg, r);
         tc::tmemWaitLoad();
         float *row = Ds + (quad * 32 + lane) * kDhPitch + 16 * cg;
#pragma unroll
         for (int i = 0; i < 16; i++) row[i] = __uint_as_float(r[i]);
      }
      __syncthreads();
      if (tid < T) {
         const int lo = max(0, 128 * m - tid), hi = min(63, 128 * m + 127 - tid);
         for (int sp = lo; sp <= hi; sp++) acc += Ds[(tid + sp - 128 * m) * kDhPitch + sp];
      }
      __syncthreads();
   }
   if (tid < T) part[(long long) run.w * kBfMaxTaps + tid] = acc;
   tc::fenceBeforeSync();
   __syncthreads();
   if (warp == 0) tc::tmemFree(tmem, 512);
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

bool firBf16x3Supported(const FirLaunch &a) { return a.dtype == DSPLIB_FLOAT32 && a.T >= 1 && a.T <= kBfMaxTaps; }

cudaError_t launchFirBf16x3(const FirLaunch &a, cudaStream_t s)
{
   if (!firBf16x3Supported(a)) return cudaErrorNotSupported;
   const size_t smem = bfSmemBytes(a.T);
   cudaError_t e =
       cudaFuncSetAttribute(fir_bf16x3_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
   if (e != cudaSuccess) return e;
   const int nt = (a.outSize + kBfTile - 1) / kBfTile;
   const int tpc = a.tuneTpc > 0 ? (a.tuneTpc < nt ? a.tuneTpc : nt) : tilesPerCtaFor(nt, a.batch, 1);
   dim3 grid((nt + tpc - 1) / tpc, a.batch < 65535 ? a.batch : 65535);
   fir_bf16x3_tc_kernel<<<grid, kBfBlock, smem, s>>>(a, tpc);
   countLaunch();
   return cudaGetLastError();
}

cudaError_t launchFirBf16x3Ragged(const RaggedChan *chans, const int4 *runs, int nRuns, const float *in,
                                  const float *taps, float *out, bool dx, int Tmax, int *err, cudaStream_t s)
{
   if (Tmax < 1 || Tmax > kBfMaxTaps) return cudaErrorNotSupported;
   if (nRuns <= 0) return cudaSuccess;
   const size_t smem = kBfSmemLimit; // every run's layout (for its own taps) fits
   cudaError_t e =
       cudaFuncSetAttribute(fir_bf16x3_ragged_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) smem);
   if (e != cudaSuccess) return e;
   int sms = 148, dev = 0;
   if (cudaGetDevice(&dev) == cudaSuccess) (void) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
   const int grid = nRuns < sms ? nRuns : sms;
   fir_bf16x3_ragged_kernel<<<grid, kBfBlock, smem, s>>>(chans, runs, nRuns, in, taps, out, dx ? 1 : 0, Tmax, err);
   countLaunch();
   return cudaGetLastError();
}

std::string firTuneKey(const FirLaunch &a, FirKernelKind kind)
{
   char buf[160];
   if (kind == FIR_F32_BF16X3 && firBf16x3Supported(a)) {
      const int nt = (a.outSize + kBfTile - 1) / kBfTile;
      snprintf(buf, sizeof(buf), "fir_bf16x3|T=%d|tiles=2^%d|batch=2^%d|nch=%d|sms=%d", a.T, tuneClass(nt),
               tuneClass(a.batch), a.filtPitch ? 1 : 0, deviceSms());
      return buf;
   }
   if ((kind == FIR_INT_WRAP_TC || kind == FIR_INT_Q_TC) && firIntTcSupported(a)) {
      const int nt = (a.outSize + kTile - 1) / kTile;
      snprintf(buf, sizeof(buf), "fir_int|dtype=%d|q=%d|T=%d|tiles=2^%d|batch=2^%d|sms=%d", a.dtype,
               kind == FIR_INT_Q_TC ? 1 : 0, a.T, tuneClass(nt), tuneClass(a.batch), deviceSms());
      return buf;
   }
   return std::string();
}

// bf16x3: the choice is the tiles per CTA; int: tiles per CTA * 16 + CTAs per SM.
std::vector<int> firTuneCandidates(const FirLaunch &a, FirKernelKind kind)
{
   std::vector<int> c;
   if (firTuneKey(a, kind).empty()) return c;
   // tiles per CTA: powers of two up to a whole channel, and the built-in rule's value
   auto tileCounts = [](int nt, int rule) {
      std::vector<int> t;
      for (int v = 1; v < nt && v <= 64; v *= 2) t.push_back(v);
      t.push_back(nt < 64 ? nt : 64);
      t.push_back(rule);
      return t;
   };
   if (kind == FIR_F32_BF16X3) {
      const int nt = (a.outSize + kBfTile - 1) / kBfTile;
      c = tileCounts(nt, tilesPerCtaFor(nt, a.batch, 1));
   }
   else {
      const int nt = (a.outSize + kTile - 1) / kTile;
      const int bound = a.dtype == DSPLIB_INT16 ? intLaunchBound<int16_t>() : intLaunchBound<int8_t>();
      for (int t : tileCounts(nt, tilesPerCtaFor(nt, a.batch, 8)))
         for (int per = 4; per <= bound; per += 2) c.push_back(t * 16 + per);
   }
   std::sort(c.begin(), c.end());
   c.erase(std::unique(c.begin(), c.end()), c.end());
   return c;
}

void firApplyChoice(FirLaunch &a, FirKernelKind kind, int choice)
{
   if (choice <= 0) return;
   if (kind == FIR_F32_BF16X3) a.tuneTpc = choice;
   else if (kind == FIR_INT_WRAP_TC || kind == FIR_INT_Q_TC) {
      a.tuneTpc = choice / 16;
      a.tunePerSm = choice % 16;
   }
}

cudaError_t launchFirDhBf16x3Ragged(const RaggedChan *chans, const int4 *runs, int nRuns, const float *x,
                                    const float *gu, float *part, int *err, cudaStream_t s)
{
   if (nRuns <= 0) return cudaSuccess;
   cudaError_t e =
       cudaFuncSetAttribute(fir_dh_bf16x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int) kDhSmem);
   if (e != cudaSuccess) return e;
   fir_dh_bf16x3_kernel<<<nRuns, kBfBlock, kDhSmem, s>>>(chans, runs, x, gu, part, err);
   countLaunch();
   return cudaGetLastError();
}


} // namespace dsplib
