// Internal declarations of the B200 DSPLIB library: handle layouts, the
// device-buffer staging helpers and the kernel launchers that the C-ABI entry
// points (fir_api.cpp, biquad_api.cpp) call.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <functional>
#include <string>
#include <vector>

#include "dsplib.h"

namespace dsplib {

constexpr uint32_t kMagicFir = 0xF1A0B200u;
constexpr uint32_t kMagicBiquad = 0xB1A0B200u;
constexpr uint32_t kMagicFltoq15 = 0xF15AB200u;
constexpr uint32_t kMagicQ15tofl = 0x15F0B200u;
constexpr uint32_t kMagicInterleave = 0x1E7EB200u;
constexpr uint32_t kMagicDeinterleave = 0xDE1EB200u;
constexpr uint32_t kMagicAddNCh = 0xADDCB200u;

// First member of every handle: GPU settings that survive re-init
// (the reference test drivers re-run init on the same handle to switch
// NATC <-> OPTIMIZED, test/DSPLIB_fir/DSPLIB_fir_d.c:291-297).
struct HandleCommon {
   uint32_t magic;
   int32_t async;
   cudaStream_t stream;
   int32_t firPrecision;
   int32_t firQMode;
   char err[200];
   int32_t errSlot;  // 1 + this handle's slot in the error-word pool (0: none yet)
   int32_t injectAt; // testing: the n-th CUDA operation of the next exec reports failure (0: off)
};

struct FirPriv {
   HandleCommon common;
   DSPLIB_fir_InitArgs initArgs;
   int32_t dtype;
   int32_t elt;
   int32_t inPitch;     // elements, bufParamsIn->stride_y / elt (DSPLIB_fir.cpp:153)
   int32_t outPitch;    // elements (DSPLIB_fir.cpp:154)
   int32_t filterPitch; // elements (DSPLIB_fir.cpp:156)
   int32_t outputSize;  // bufParamsOut->dim_x (DSPLIB_fir.cpp:155)
   int32_t initialized;
   uint32_t tuneGen;    // autotuner generation the cached choice was resolved at (0: none)
   int32_t tuneKind;    // kernel kind it was resolved for
   int32_t tuneChoice;  // the choice (-1: the built-in rule)
};

struct BiquadPriv {
   HandleCommon common;
   DSPLIB_cascadeBiquad_InitArgs initArgs;
   int32_t inPitch;   // elements (DSPLIB_cascadeBiquad.cpp:450)
   int32_t outPitch;  // elements (:451)
   int32_t varPitch;  // elements (:452)
   int32_t coefPitch; // elements between channel-interleaved coefficient rows (OPT, per-channel)
   int32_t coefRows;  // rows of the coefficient buffer passed to init
   int32_t coefCols;  // elements per coefficient row
   int32_t initialized;
   uint32_t tuneGen;   // autotuner generation the cached choice was resolved at (0: none)
   int32_t tuneChoice; // the scan's choice (-1: the built-in rule)
};

// DSPLIB_fltoq15 / DSPLIB_q15tofl handle (DSPLIB_fltoq15_priv.h / DSPLIB_q15tofl_priv.h
// of the reference keep blockSize = dataSize and the type-specific exec).
struct Q15Priv {
   HandleCommon common;
   int32_t funcStyle;
   uint32_t dataSize; // elements per exec
   int32_t isDouble;  // float side is FLOAT64
   int32_t initialized;
};

// DSPLIB_interleave / DSPLIB_deinterleave handle: the fields the reference keeps in
// DSPLIB_matTrans_PrivArgs (widthIn, heightIn, strideIn, strideOut) plus the type.
struct LayoutPriv {
   HandleCommon common;
   uint32_t widthIn, heightIn;
   int32_t strideIn, strideOut; // bytes
   int32_t dataType;
   int32_t initialized;
};

// DSPLIB_addNCh handle: the fields of DSPLIB_addNCh_PrivArgs.
struct AddNChPriv {
   HandleCommon common;
   uint32_t inputs, samples, channels;
   int32_t strideInElementsY, strideInElementsZ, strideOutElements;
   int32_t dataType;
   int32_t initialized;
};

// ---------------------------------------------------------------- autotuner (autotune.cpp)

// Current mode (DSPLIB_GPU_TUNE_*), and a counter that changes whenever an entry or
// the mode does (handles re-resolve their choice when it moved).
int tuneMode();
unsigned tuneGeneration();
// The cached choice for key (false when absent or the tuner is off).
bool tuneLookup(const std::string &key, int *choice);
void tuneStore(const std::string &key, int choice, bool save);
// Power-of-two class of v (smallest c with 2^c >= v), and the current device's SM count.
int tuneClass(long long v);
int deviceSms();
// Median of `reps` event-timed launches after one warm-up (ms; negative on failure), the
// L2 cache flushed through `flush` (256 MiB, or null) before each.
float tuneTime(const std::function<cudaError_t(cudaStream_t)> &launch, cudaStream_t s, int reps, void *flush);
// Fill scratch with a hashed pattern (tune_fill.cu): floats in [-0.5, 0.5) or raw bits.
cudaError_t launchTuneFill(void *p, size_t bytes, bool asFloat, cudaStream_t s);
// The same on a private stream, waited for.
bool tuneFill(void *p, size_t bytes, bool asFloat);
// Time every candidate on a private stream, store the fastest under key (and rewrite the
// cache file); returns it, or -1 when nothing could be timed.
int tunePick(const std::string &key, const std::vector<int> &cands,
             const std::function<cudaError_t(int, cudaStream_t)> &launch);

// Autotuner entry points of the handle families (fir_api.cpp, biquad_api.cpp): the
// tuning key of an initialised handle's configuration with its candidates ("" when its
// kernel has no shapes to choose), and a measurement of them stored in the table.
std::string firHandleTuneKey(DSPLIB_kernelHandle h, std::vector<int> *cands);
DSPLIB_STATUS firHandleTune(DSPLIB_kernelHandle h);
std::string biquadHandleTuneKey(DSPLIB_kernelHandle h, std::vector<int> *cands);
DSPLIB_STATUS biquadHandleTune(DSPLIB_kernelHandle h);

// ---------------------------------------------------------------- runtime

void setError(HandleCommon *h, const char *fmt, ...);

// Error words written by kernels when a bounded wait gives up: one per handle, in
// mapped page-locked host memory (kernels store to it, the host reads it after the
// stream has synchronized; no copy).  errorWord never returns null.
int *errorWord(HandleCommon *h);
void releaseErrorWord(HandleCommon *h);
// The word's value, cleared when set.
int takeErrorWord(HandleCommon *h);
// Process-wide words for callers without a handle (filter-bank plans).
int *allocErrorWord();
void freeErrorWord(int *w);

// Fault injection for tests (DSPLIB_gpu_injectFault): armed from the handle at the start
// of an exec on this thread; injectCheck passes e through, except that the armed
// operation (counted over the calls of injectCheck) reports cudaErrorUnknown.
void injectArm(HandleCommon *h);
void injectDisarm();
cudaError_t injectCheck(cudaError_t e);
DSPLIB_STATUS cudaFail(HandleCommon *h, cudaError_t e, const char *what);
void countLaunch(int n = 1);

// True when p is device-accessible global memory (device or managed allocation).
bool isDevicePtr(const void *p);

// Per-device, per-thread growable scratch used to stage host buffers, from the
// device's stream-ordered pool (a buffer that grows is replaced in the order of s).
// Returns nullptr on allocation failure.
void *stagingBuffer(int slot, size_t bytes, cudaStream_t s);

// A strided 2-D region of a caller buffer: rows of width bytes, pitch bytes apart.
struct Region {
   void *host;        // caller pointer
   void *dev;         // device pointer the kernel uses
   size_t width;      // bytes per row that the kernel touches
   size_t height;     // rows
   size_t pitch;      // bytes between rows
   bool staged;       // host buffer copied through a staging buffer
   bool zeroCopy;     // the kernel touches each element about once: a small pinned buffer may be used in place
   bool streamed = false; // ... and in whole coalesced rows: a pinned buffer of any size may be used in place
   bool onHost = false;   // set by regionIn: the caller's buffer is host memory (staged or mapped)
   size_t bytes() const { return height ? (height - 1) * pitch + width : 0; }
};

// Whether exec must synchronize its stream before returning: always in the synchronous
// mode; whenever the per-thread staging buffers hold part of the call (the next call may
// reuse them); and for host buffers used in place unless the caller asked for asynchronous
// completion of those too (async level 2).
inline bool mustSync(const HandleCommon *hc, bool staged, bool onHost)
{
   return !hc->async || staged || (onHost && hc->async < 2);
}

// Prepare a region: device pointers, and (zeroCopy regions) pinned host buffers
// of at most kZeroCopyMaxBytes (of any size for streamed regions), are used in
// place through their mapped addresses; other host pointers are
// staged (copied in when copyIn).  Returns cudaSuccess or the failure.
constexpr size_t kZeroCopyMaxBytes = 64 * 1024;
cudaError_t regionIn(Region &r, int slot, bool copyIn, cudaStream_t s);
// Copy a staged region back to the caller's host buffer (row by row, leaving
// the bytes between rows untouched).
cudaError_t regionOut(const Region &r, cudaStream_t s);

// Device pointer through which kernels reach a page-locked host buffer (nullptr
// when p is not page-locked host memory).
void *mappedHostPtr(const void *p);

// Copy `rows` rows of `width` bytes, `pitch` bytes apart, in one call.
cudaError_t copyRows(void *dst, const void *src, size_t width, size_t rows, size_t pitch, cudaMemcpyKind kind,
                     cudaStream_t s);

// Streams and events of the host-buffer pipeline (per host thread and device):
// block b is copied in on `in`, computed on `comp`, copied out on `out`, so
// the copies of neighbouring blocks overlap the kernels (and each other: the
// two directions use separate copy engines).
constexpr int kPipeMaxBlocks = 8;
constexpr size_t kFirPipeMinBytes = 8u << 20;    // host in + out bytes from which FIR exec pipelines
constexpr size_t kFirPipeBlockBytes = 16u << 20; // in + out bytes per block (2 .. kPipeMaxBlocks blocks)
constexpr size_t kBqPipeMinBytes = 4u << 20;      // page-locked input bytes from which cascade-biquad exec pipelines
constexpr size_t kBqPipeBlockBytes = 2u << 20;    // input bytes per time block (2 .. kPipeMaxBlocks blocks)
struct PipeContext {
   bool ready = false;
   cudaStream_t in = nullptr, comp = nullptr, out = nullptr;
   cudaEvent_t start = nullptr, done = nullptr;
   cudaEvent_t copied[kPipeMaxBlocks] = {}, computed[kPipeMaxBlocks] = {};
};
PipeContext *pipeContext();
// A failure inside a pipeline: let the copies and kernels already queued on its streams
// finish (they read and write the caller's host buffers) before reporting it.
DSPLIB_STATUS pipeFail(HandleCommon *h, PipeContext *pc, cudaError_t e, const char *what);

// ---------------------------------------------------------------- kernels

struct FirLaunch {
   const void *x;
   const void *h; // first tap row (already offset past any MMA padding)
   void *y;
   int dtype;
   int batch;
   int T;
   int outSize;
   long long inPitch;   // elements
   long long outPitch;  // elements
   long long filtPitch; // elements between tap rows, 0 = shared
   int shift;
   int *err = nullptr; // tensor-core kernels: error word for an expired bounded wait
   int tuneTpc = 0;    // tensor-core kernels: output tiles per CTA (0: the built-in rule)
   int tunePerSm = 0;  // int8/int16 tensor-core kernel: resident CTAs per SM (0: the built-in rule)
};

enum FirKernelKind {
   FIR_NATC = 0,       // bit-exact natural-C semantics (wrap / sequential float), CUDA cores
   FIR_QMODE = 1,      // exact accumulator, round/shift/saturate, CUDA cores
   FIR_F32_SIMT = 2,   // FP32 FMA register-tiled CUDA-core kernel
   FIR_F32_BF16X3 = 3, // tcgen05 split-BF16x3 tensor-core kernel
   FIR_INT_WRAP_TC = 4, // tcgen05 kind::i8 kernel, int8/int16, natural-C wrap output
   FIR_INT_Q_TC = 5,    // tcgen05 kind::i8 kernel, int8/int16, Q-mode output
   FIR_F32_Q = 6        // FLOAT32 in float Q mode (InitArgs.enableQ): int32 quantisation, exact sums
};

// Largest InitArgs.shift the Q-mode output stages accept.
constexpr int kFirMaxQShift = 62;
// Largest InitArgs.Q of the float Q mode (the reference scales by 1U << Q).
constexpr int kFirMaxFloatQ = 31;

cudaError_t launchFir(const FirLaunch &a, FirKernelKind kind, cudaStream_t s);

// Q.15 conversions over n elements (any alignment; 16-byte aligned pointers take the
// vector kernels).  natc: the natural-C rounding steps, else round-half-to-even.
cudaError_t launchFltoq15(const void *in, int16_t *out, long long n, bool isDouble, bool natc, cudaStream_t s);
cudaError_t launchQ15tofl(const int16_t *in, void *out, long long n, bool isDouble, cudaStream_t s);

// Strided transpose of DSPLIB_interleave / DSPLIB_deinterleave:
// out[(i * sOutB) / elt + j] = in[i + sInE * j], i < W, j < H.
struct TransposeLaunch {
   const void *in;
   void *out;
   long long W, H;
   long long sInE; // input row stride, elements
   long long sOutB; // output row stride, bytes
   int elt;         // 1, 2, 4 or 8
};
cudaError_t launchTranspose(const TransposeLaunch &a, cudaStream_t s);

// DSPLIB_addNCh: out[row * sO + col] = sum over l of in[row * sY + col + l * sZ] (element strides).
struct AddNChLaunch {
   const void *in;
   void *out;
   long long samples, channels;
   int inputs;
   long long sY, sZ, sO;
   bool isDouble;
};
cudaError_t launchAddNCh(const AddNChLaunch &a, cudaStream_t s);
bool firIntTcSupported(const FirLaunch &a);
bool firBf16x3Supported(const FirLaunch &a);
cudaError_t launchFirIntTc(const FirLaunch &a, bool qmode, cudaStream_t s);
// Autotuner entries of the tensor-core FIR kernels (kind FIR_F32_BF16X3, FIR_INT_WRAP_TC,
// FIR_INT_Q_TC): the key of a launch's problem class ("" for kernels without shapes to
// choose), its candidate choices, and a choice applied to a launch.
std::string firTuneKey(const FirLaunch &a, FirKernelKind kind);
std::vector<int> firTuneCandidates(const FirLaunch &a, FirKernelKind kind);
void firApplyChoice(FirLaunch &a, FirKernelKind kind, int choice);

// One channel of the batched filter bank: samples at xOff (length L; the FIR
// output and the biquad signals use the first Lu = L - T + 1), T taps at hOff,
// S biquad stages (5 coefficients each) at cOff; its slice of every work plane
// (FIR output, stage outputs) at pOff, a multiple of 16 floats, round16(Lu) long.
struct RaggedChan {
   long long xOff, hOff, cOff, pOff;
   int L, T, S, Lu;
   long long ckOff;  // first unit state (float2) of the channel: one per 512-sample unit and stage
   long long phiOff; // first double of the channel's unit transitions
   long long grpOff; // first float of the channel's chain group states (2S per 32 units)
};
// Split-BF16x3 tensor-core FIR over a list of runs {channel, first tile, tiles, 0}
// of kFirBfTile outputs: forward (valid correlation of the channel's x with its
// taps) or dx (full convolution of the output gradient with the taps).
constexpr int kFirBfTile = 8192;
constexpr int kFirBfRunTiles = 4;
constexpr int kFirBfMaxTaps = 512;
// Device the plan was built on (-1 for a null plan).
int raggedPlanDevice(DSPLIB_gpu_raggedPlan plan);
// Taps gradient of the filter bank on the tensor cores over runs {channel, first tile,
// tiles, partial slot} of 8192 samples of the gradient at the FIR output:
// part[slot * 512 + c] = sum over the run of gu[j] x[j + c], c < T.
cudaError_t launchFirDhBf16x3Ragged(const RaggedChan *chans, const int4 *runs, int nRuns, const float *x,
                                    const float *gu, float *part, int *err, cudaStream_t s);
cudaError_t launchFirBf16x3Ragged(const RaggedChan *chans, const int4 *runs, int nRuns, const float *in,
                                  const float *taps, float *out, bool dx, int Tmax, int *err, cudaStream_t s);

// Cascade of the filter bank split along time (bank_scan.cu): units of kBankSpan
// samples (one warp each), chained per channel through the 2S-dimensional cascade
// state; per stage a table of kBankTabFloats floats (coefficients, transition
// powers, free-response rows), per channel the unit transitions of both directions.
constexpr int kBankSpan = 512;
constexpr int kBankTabFloats = 80;

struct BankLaunch {
   const RaggedChan *chans;
   int C;
   const int2 *units; // (channel, unit index within the channel)
   int nUnits;
   int Smax;
   const float *tables;
   const double *phi;
   const float *u;    // FIR output plane
   float *y;          // forward output
   const float *gy;   // adjoint: output gradient
   float *g;          // adjoint: gradient w.r.t. the FIR output
   float2 *aggF, *ckptF, *aggA, *ckptA;
   float *groupF, *groupA; // chain group states of channels beyond 64 groups of 32 units
   const int *chainOrder;  // channel of each chain CTA (most units first)
   float *part;       // adjoint: 5 coefficient-gradient sums per unit and stage
   float *gcoefs;
   // forward with the loss fused (target != nullptr): gyOut = scale (y - target), unit
   // sums of squares in lossPart, the adjoint's unit aggregates in aggA
   const float *target;
   float *gyOut;
   double *lossPart;
   float scale;
   bool aggReady; // adjoint: aggA already computed by the fused forward
   // the unit list is ordered by stage count, deepest first: bucket k holds the units of
   // the channels of bucketS[k] stages, from bucketStart[k] (host arrays)
   const int *bucketS, *bucketStart;
   int nBuckets;
   // streams the adjoint's buckets fan out to (forked from and joined back into the
   // caller's stream with events; capturable), or nAux = 0
   const cudaStream_t *aux;
   int nAux;
   cudaEvent_t fork;
   const cudaEvent_t *join;
};
// Doubles of both unit transitions of a channel of S stages.
long long bankTransitionDoubles(int S);
cudaError_t launchBankTables(const RaggedChan *chans, int C, const float *coefs, int totalStages, int Smax,
                             float *tables, double *phi, cudaStream_t s);
cudaError_t launchBankForward(const BankLaunch &b, cudaStream_t s);
cudaError_t launchBankBackward(const BankLaunch &b, cudaStream_t s);

struct BiquadLaunch {
   const float *x;
   float *y;
   float *state;
   const float *coef;
   int form;     // DSPLIB_biquadForm (TIF only with optLayout)
   int nch;      // per-channel coefficients
   int optLayout; // 1: coefficients in the get_coefficients layout
   int N, C, S;
   long long inPitch, outPitch, varPitch, coefPitch; // elements
   int prefetch = 0; // x is device memory: the scan kernel may fetch the next window early (cp.async)
   int tuneChoice = -1; // scan shape from the autotuner: 100 * warps per CTA + CTAs per cluster, or 1 for
                        // the per-channel kernel (-1: the rule)
};

// Autotuner entries of the cascade-biquad scan (OPTIMIZED style): the key of a launch's
// problem class ("" when the per-channel kernel or the sequential one runs) and its
// candidate shapes (100 * warps per CTA + CTAs per cluster; 1: one CTA per channel).
std::string biquadTuneKey(const BiquadLaunch &a);
std::vector<int> biquadTuneCandidates(const BiquadLaunch &a);

// DSPLIB_cascadeBiquad_get_coefficients for device buffers (coef_kernels.cu): TIF transform
// (tif != 0) or the per-channel coefficient-major reorder of the DF forms; pitch in floats
// between the rows of per-channel layouts.
cudaError_t launchBiquadCoefTransform(int tif, int nch, const float *nat, float *opt, int S, int C, long long pitch,
                                      cudaStream_t s);

// NATC: sequential recursion per channel, bit-exact to the reference _cn kernels.
cudaError_t launchBiquadSequential(const BiquadLaunch &a, cudaStream_t s);
// OPTIMIZED: chunked parallel-in-time scan.
// Stages up to which launchBiquadScan runs the scan kernels (beyond: the sequential kernel).
int biquadScanMaxStages();
cudaError_t launchBiquadScan(const BiquadLaunch &a, cudaStream_t s);

} // namespace dsplib
