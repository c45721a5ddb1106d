/*
 * GPU extensions of the DSPLIB API.  None of these has a counterpart in the
 * reference (which runs on a single C7x core); they expose the GPU plumbing:
 * the CUDA stream a handle launches on, whether exec waits for completion,
 * kernel-variant selection, and error text.  All take a handle that
 * DSPLIB_fir_init or DSPLIB_cascadeBiquad_init has initialised; settings
 * survive later init calls on the same handle.
 */
#ifndef DSPLIB_GPU_H_
#define DSPLIB_GPU_H_

#include "DSPLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Launch this handle's kernels (and staging copies) on the given cudaStream_t
 *  (NULL = the legacy default stream, the default).  This and DSPLIB_gpu_setAsync apply to
 *  an initialised handle (DSPLIB_ERR_NULL_POINTER before its first init) and persist across
 *  later inits of the same handle. */
DSPLIB_STATUS DSPLIB_gpu_setStream(DSPLIB_kernelHandle handle, void *cudaStream);

/** async = 0 (default): exec returns after the results are written.
 *  async = 1: exec returns once the work is queued on the handle's stream when every
 *  buffer is device memory; calls with host buffers complete before returning.
 *  async = 2: as 1, and also when host buffers are page-locked and read or written in
 *  place by the kernels (no staging copy): exec returns once queued and the caller
 *  synchronizes the handle's stream before touching those buffers.  Independent calls
 *  on several handles and streams then overlap their PCIe reads, kernels and writes.
 *  Calls that stage host data through the library's per-thread buffers (pageable
 *  memory, pipelined copies) still complete before returning. */
DSPLIB_STATUS DSPLIB_gpu_setAsync(DSPLIB_kernelHandle handle, int32_t async);

/** Text of the last failure recorded on this handle ("" when none). */
const char *DSPLIB_gpu_lastError(DSPLIB_kernelHandle handle);

/** Float FIR precision forms for DSPLIB_FUNCTION_OPTIMIZED:
 *  SIMT  = FP32 fused multiply-add on CUDA cores (the plain kernel, default),
 *  BF16X3 = each FP32 operand split into BF16 hi + lo parts, the products
 *           hi*hi + hi*lo + lo*hi (and lo*lo, which costs nothing extra here and keeps the
 *           error within 1e-5 of the peak output) accumulated in FP32 on tcgen05 tensor
 *           cores. */
typedef enum {
   DSPLIB_GPU_FIR_SIMT = 0,
   DSPLIB_GPU_FIR_BF16X3 = 1,
} DSPLIB_gpu_firPrecision;
DSPLIB_STATUS DSPLIB_gpu_firSetPrecision(DSPLIB_kernelHandle handle, int32_t precision);

/** Integer FIR output stage for DSPLIB_FUNCTION_OPTIMIZED:
 *  0 (default) = wrap modulo 2^bits, identical to the natural-C kernel;
 *  1 = Q mode: y = saturate((acc + 2^(shift-1)) >> shift) with the exact
 *      accumulator and InitArgs.shift (shift = 0: saturate(acc)). */
DSPLIB_STATUS DSPLIB_gpu_firSetQMode(DSPLIB_kernelHandle handle, int32_t enable);

/** After asynchronous calls on this handle (DSPLIB_gpu_setAsync) and a synchronisation of
 *  its stream: DSPLIB_ERR_FAILURE (reason in DSPLIB_gpu_lastError) if a bounded wait of a
 *  tensor-core kernel expired in any of them since the last check, else DSPLIB_SUCCESS.
 *  Synchronous calls check this themselves.  Each handle has its own error word (in
 *  page-locked host memory shared by the library's handles; DSPLIB_gpu_releaseHandle
 *  returns it). */
DSPLIB_STATUS DSPLIB_gpu_status(DSPLIB_kernelHandle handle);

/** Testing hook: the n-th CUDA operation (staging copy, kernel launch or pipeline block
 *  copy) that the next exec on this handle queues reports a failure after it was queued,
 *  so the call takes its error path (DSPLIB_ERR_FAILURE, reason in DSPLIB_gpu_lastError,
 *  work already queued drained before returning).  Applies to one exec; 0 disables. */
DSPLIB_STATUS DSPLIB_gpu_injectFault(DSPLIB_kernelHandle handle, int32_t operation);

/** Number of CUDA kernels this library has launched in this process. */
int64_t DSPLIB_gpu_kernelLaunchCount(void);

/* ---------------------------------------------------------------------------
 * Autotuner of launch shapes.  The reference picks its kernel variants by fixed
 * size classes in init (src/DSPLIB_fir/DSPLIB_fir_ci.cpp:350-405,
 * src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad.cpp:480-615); this library keeps a
 * measured choice per problem class and GPU instead, where a kernel has shapes to
 * choose from:
 *   fir_bf16x3  output tiles per CTA of the split-BF16x3 FIR;
 *   fir_int     output tiles per CTA and resident CTAs per SM of the int8/int16 FIR;
 *   bq_scan     warps per CTA (the 32-sample chunks of one window: its length) and
 *               CTAs per cluster of the cascade-biquad scan;
 *   bank_runs   output tiles per run of the batched filter bank's FIR work lists.
 * Keys are text: "<op>|<parameter>=<value>|...|sms=<SM count>"; lengths, batch sizes
 * and channel counts enter as power-of-two classes ("2^k"), taps, stages, form and
 * data type exactly.  A choice is one integer (see DSPLIB_gpu_autotuneHandleKey).
 * Entries are process-wide, read from and written to a JSON cache file:
 *   {"format": "dsplib_b200 autotune 1", "entries": {"<key>": <choice>, ...}}
 * The environment variables DSPLIB_GPU_TUNE_CACHE (the file) and DSPLIB_GPU_AUTOTUNE
 * (the mode) give the initial settings.  Choices never change results beyond the
 * floating-point summation order of the cascade scan's cluster carry.
 * ------------------------------------------------------------------------- */
typedef enum {
   DSPLIB_GPU_TUNE_OFF = 0,     /* built-in rules only */
   DSPLIB_GPU_TUNE_CACHED = 1,  /* default: a cached choice where one exists, else the rule */
   DSPLIB_GPU_TUNE_MEASURE = 2, /* as CACHED; a class without an entry is timed (every
                                   candidate on scratch buffers of the problem's shape) when a
                                   handle is initialised or a plan is built, the fastest kept
                                   and the cache file rewritten */
} DSPLIB_gpu_tuneMode;

DSPLIB_STATUS DSPLIB_gpu_autotuneSetMode(int32_t mode);
int32_t DSPLIB_gpu_autotuneGetMode(void);
/** Cache file (NULL or "": none); entries it holds are merged into the table. */
DSPLIB_STATUS DSPLIB_gpu_autotuneSetCachePath(const char *path);
/** Write the table to the cache file (DSPLIB_ERR_INVALID_VALUE when none is set). */
DSPLIB_STATUS DSPLIB_gpu_autotuneSave(void);
/** Forget every entry (the file is left as it is). */
DSPLIB_STATUS DSPLIB_gpu_autotuneClear(void);
/** The entry for key, or -1. */
int32_t DSPLIB_gpu_autotuneLookup(const char *key);
/** Set an entry (pins a choice; not written to the file until DSPLIB_gpu_autotuneSave). */
DSPLIB_STATUS DSPLIB_gpu_autotuneStore(const char *key, int32_t choice);
/** Number of entries. */
int32_t DSPLIB_gpu_autotuneCount(void);
/** Time the candidates of an initialised FIR or cascade-biquad handle's configuration now
 *  (as MEASURE mode does in init) and store the fastest; DSPLIB_ERR_NOT_IMPLEMENTED when
 *  its kernel has no shapes to choose from. */
DSPLIB_STATUS DSPLIB_gpu_autotune(DSPLIB_kernelHandle handle);
/** The tuning key of an initialised handle's configuration (copied into buf, at most len
 *  bytes with the terminator) and the number of candidate choices (0: nothing to tune). */
int32_t DSPLIB_gpu_autotuneHandleKey(DSPLIB_kernelHandle handle, char *buf, int32_t len);
/** Candidate i (0 <= i < the count above) of that key, or -1. */
int32_t DSPLIB_gpu_autotuneHandleCandidate(DSPLIB_kernelHandle handle, int32_t i);

/** End of a handle's life (the reference API has no destructor: callers free
 *  the handle memory themselves).  Waits for work an asynchronous exec queued
 *  on the handle's stream, then marks the handle uninitialised so later calls
 *  on it fail with DSPLIB_ERR_NULL_POINTER; the caller may then free it.
 *  Handles own no device memory, so skipping this call leaks nothing. */
DSPLIB_STATUS DSPLIB_gpu_releaseHandle(DSPLIB_kernelHandle handle);

/* ---------------------------------------------------------------------------
 * Streaming (overlap-save) FIR.  DSPLIB_fir computes "valid" outputs: N input
 * samples give N - T + 1 outputs, and a caller filtering a continuous signal in
 * blocks must carry each channel's last T - 1 input samples into the next call
 * (the reference leaves this to the caller, test/DSPLIB_fir/DSPLIB_fir_d.c).  A
 * stream keeps that history on the device: every call takes dataSize new samples
 * per channel and returns dataSize outputs per channel, as if the whole signal,
 * preceded by T - 1 zeros, had been filtered in one call.  No counterpart in the
 * reference.
 * ------------------------------------------------------------------------- */
typedef struct DSPLIB_gpu_firStream_s *DSPLIB_gpu_firStream;

/** args, bufParamsFilter as for DSPLIB_fir_init, with args->dataSize = new samples
 *  per channel and block; bufParamsIn / bufParamsOut describe one block of input /
 *  output (dim_x = dataSize, dim_y = channels, stride_y = row pitch in bytes).
 *  Allocates the device history and window buffers (DSPLIB_gpu_firStreamDestroy
 *  frees them); the history starts at zero. */
DSPLIB_STATUS DSPLIB_gpu_firStreamCreate(DSPLIB_gpu_firStream *stream, const DSPLIB_fir_InitArgs *args,
                                         const DSPLIB_bufParams2D_t *bufParamsIn,
                                         const DSPLIB_bufParams2D_t *bufParamsFilter,
                                         const DSPLIB_bufParams2D_t *bufParamsOut);
/** The stream's internal DSPLIB_fir handle: DSPLIB_gpu_setStream / setAsync /
 *  firSetPrecision / firSetQMode / lastError apply to the stream through it. */
DSPLIB_kernelHandle DSPLIB_gpu_firStreamHandle(DSPLIB_gpu_firStream stream);
/** Filter the next block (host or device buffers, as DSPLIB_fir_exec). */
DSPLIB_STATUS DSPLIB_gpu_firStreamExec(DSPLIB_gpu_firStream stream, const void *pIn, void *pFilter, void *pOut);
/** Zero the history (start a new signal). */
DSPLIB_STATUS DSPLIB_gpu_firStreamReset(DSPLIB_gpu_firStream stream);
DSPLIB_STATUS DSPLIB_gpu_firStreamDestroy(DSPLIB_gpu_firStream stream);

/* ---------------------------------------------------------------------------
 * Batched filter bank over channels of uneven length, forward and adjoint.
 * Per channel c (length L_c, T_c taps, S_c second-order stages):
 *     u_c = DSPLIB_fir valid correlation of x_c with h_c      (L_c - T_c + 1 samples)
 *     y_c = S_c cascaded direct-form-II biquads applied to u_c from a zero state
 * Every buffer is FP32 in device memory, channels packed back to back:
 *     x, y, gx, gy: channel c at sample offset sum_{k<c} L_k (y and gy use the
 *                   first L_c - T_c + 1 samples; the remaining T_c - 1 of y are
 *                   written as zero and those of gy are ignored);
 *     taps, gtaps:  channel c at offset sum_{k<c} T_k, same tap order as DSPLIB_fir;
 *     coefs, gcoefs: channel c at offset 5 * sum_{k<c} S_k, rows [b0 b1 b2 a1 a2]
 *                   (a0 = 1; y[t] = b0 w[t] + b1 w[t-1] + b2 w[t-2],
 *                    w[t] = u[t] - a1 w[t-1] - a2 w[t-2]).
 * The reference has no counterpart: it filters one channel layout at a time and
 * has no gradients; these entry points serve a training loop over many filters
 * (the fused form of DSPLIB_fir followed by DSPLIB_cascadeBiquad).
 * ------------------------------------------------------------------------- */
typedef struct DSPLIB_gpu_raggedPlan_s *DSPLIB_gpu_raggedPlan;

typedef enum {
   DSPLIB_GPU_RAGGED_SAMPLES = 0, /* floats in x / gx (sum L_c) */
   DSPLIB_GPU_RAGGED_TAPS = 1,    /* floats in taps / gtaps (sum T_c) */
   DSPLIB_GPU_RAGGED_COEFS = 2,   /* floats in coefs / gcoefs (5 sum S_c) */
   DSPLIB_GPU_RAGGED_WORK = 3,    /* floats the forward leaves for the adjoint: the FIR output
                                     (sum_c round16(L_c - T_c + 1) floats), one 2-float state per
                                     512 samples and stage (the cascade's checkpoints) and the
                                     unit aggregates, per-stage tables and per-channel unit
                                     transitions: about 4 bytes per sample plus 0.03 per sample
                                     and stage; no stage output is kept */
   DSPLIB_GPU_RAGGED_SCRATCH = 4, /* floats of adjoint scratch (about 4 bytes per sample plus
                                     0.07 per sample and stage) */
   DSPLIB_GPU_RAGGED_OUTPUTS = 5, /* valid output samples (sum L_c - T_c + 1) */
} DSPLIB_gpu_raggedSize;

/** Build a plan (per-channel offsets and work lists, uploaded to the current
 *  device).  1 <= T_c <= 512, T_c <= L_c, 0 <= S_c <= 64, else
 *  DSPLIB_ERR_INVALID_DIMENSION.  The plan may be used from any stream of that device. */
DSPLIB_STATUS DSPLIB_gpu_raggedPlanCreate(DSPLIB_gpu_raggedPlan *plan, int32_t numChannels, const int32_t *length,
                                          const int32_t *taps, const int32_t *stages);
/** Buffer sizes in floats (DSPLIB_gpu_raggedSize); -1 for an unknown query. */
int64_t DSPLIB_gpu_raggedPlanSize(DSPLIB_gpu_raggedPlan plan, int32_t what);
DSPLIB_STATUS DSPLIB_gpu_raggedPlanDestroy(DSPLIB_gpu_raggedPlan plan);

/** Forward: y from x, taps and coefs.  work (16-byte aligned) receives the FIR
 *  output and the cascade's checkpoint states (what the adjoint needs; it
 *  recomputes the stage outputs from them).  Queued on `stream`; no allocation,
 *  no host synchronisation. */
DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_fwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, float *y, float *work, void *stream);
/** Adjoint: given gy = dLoss/dy and the forward's work buffer, writes
 *  gx = dLoss/dx, gtaps = dLoss/dtaps and gcoefs = dLoss/dcoefs.  scratch holds
 *  DSPLIB_GPU_RAGGED_SCRATCH floats (no initial contents needed).  Reductions
 *  run in a fixed order: results are bitwise repeatable. */
DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_bwd(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                              const float *coefs, const float *work, const float *gy, float *gx,
                                              float *gtaps, float *gcoefs, float *scratch, void *stream);
/** Mean squared error over the valid output samples and its gradient:
 *  loss[0] = sum (y - target)^2 / n (n = DSPLIB_GPU_RAGGED_OUTPUTS, FP64 sums in
 *  a fixed order), gy = 2 (y - target) / n, zero on the tail samples.  scratch
 *  is a DSPLIB_GPU_RAGGED_SCRATCH buffer (the same one the adjoint takes). */
DSPLIB_STATUS DSPLIB_gpu_raggedMseGrad(DSPLIB_gpu_raggedPlan plan, const float *y, const float *target, float *gy,
                                       float *loss, float *scratch, void *stream);

/** One training step: the forward, the mean squared error against target (as
 *  DSPLIB_gpu_raggedMseGrad: loss[0], gy) and the adjoint (as
 *  DSPLIB_gpu_firBiquadBatched_bwd with that gy) in one call, sharing passes: the
 *  cascade's output pass also forms gy and runs the adjoint's first pass over it.
 *  Results equal those of the three separate calls; y and gy are outputs too.
 *  work and scratch as for the separate calls.  No counterpart in the reference. */
DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_stepMse(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                                  const float *coefs, const float *target, float *y, float *gy,
                                                  float *loss, float *gx, float *gtaps, float *gcoefs, float *work,
                                                  float *scratch, void *stream);

/** The training step of DSPLIB_gpu_firBiquadBatched_stepMse on buffers in host memory
 *  (device pointers are accepted too, per array, and used in place): x, taps, coefs and
 *  target are read, y, gy, loss, gx, gtaps and gcoefs written (gy may be NULL when the
 *  caller does not want it).  No work or scratch argument: the plan stages through
 *  device buffers of its own (allocated by the first call, about 20 bytes per sample,
 *  released by DSPLIB_gpu_raggedPlanDestroy).
 *  The channels are split into up to 8 contiguous segments of about equal samples, each
 *  with a plan of its own (built by the first call on the plan); segment k is copied in
 *  while segment k - 1 is filtered and segment k - 2's results are copied out, on three
 *  streams, so that both transfer directions and the kernels overlap.  With page-locked
 *  buffers the copies run at the link's rate; pageable ones are copied by the driver
 *  through its own bounce buffers and overlap less.  Synchronous by default: returns once
 *  every result is in the caller's memory (after the work queued on `stream` before it);
 *  after DSPLIB_gpu_raggedPlanSetAsync(plan, 1) it returns once the work is queued, so
 *  calls on different plans overlap one call's copies out with the next call's copies in;
 *  the caller synchronises `stream` before touching the buffers, then checks
 *  DSPLIB_gpu_raggedPlanStatus.
 *  y, gy, gx, gtaps and gcoefs equal the device call's bit for bit; loss is the same sum
 *  of squares added per segment, then over the segments in order.  DSPLIB_ERR_FAILURE if
 *  a copy or launch fails or a bounded tensor-core wait expired.  No counterpart in the
 *  reference. */
DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_stepMseHost(DSPLIB_gpu_raggedPlan plan, const float *x, const float *taps,
                                                      const float *coefs, const float *target, float *y, float *gy,
                                                      float *loss, float *gx, float *gtaps, float *gcoefs,
                                                      void *stream);

/** 1: DSPLIB_gpu_firBiquadBatched_stepMseHost on this plan returns once queued (page-locked
 *  buffers; the caller synchronises the stream); 0 (default): it returns complete. */
DSPLIB_STATUS DSPLIB_gpu_raggedPlanSetAsync(DSPLIB_gpu_raggedPlan plan, int32_t async);

/** After the calls queued on this plan were synchronised: DSPLIB_ERR_FAILURE if a bounded
 *  wait of one of its tensor-core kernels expired since the last check (the outputs of
 *  that call are incomplete), else DSPLIB_SUCCESS; the check clears the plan's word. */
DSPLIB_STATUS DSPLIB_gpu_raggedPlanStatus(DSPLIB_gpu_raggedPlan plan);

/** Size, in floats, of the scratch array built into the library for
 *  DSPLIB_gpu_firBiquadBatched_bwdStaticScratch (16 MiB per device). */
#define DSPLIB_GPU_STATIC_SCRATCH_FLOATS (4u << 20)

/** The adjoint of DSPLIB_gpu_firBiquadBatched_bwd without a scratch argument
 *  and without allocating: its scratch is a fixed array inside the library, one
 *  per device.  No counterpart in the reference (which has no adjoint); it is
 *  for callers that cannot allocate device memory while they run (deadline-bound
 *  processing threads, memory reserved up front, buffers owned by an allocator
 *  they do not control).
 *  - Plans needing more than DSPLIB_GPU_STATIC_SCRATCH_FLOATS floats of scratch
 *    (DSPLIB_GPU_RAGGED_SCRATCH) return DSPLIB_ERR_BUFFER_TOO_SMALL, nothing queued.
 *  - All calls on a device share the array: calls that overlap in time race and
 *    corrupt each other's results; order them (same stream or events).
 *  - No part of the array needs to start at zero.
 *  - The array's device address is looked up, with the plan's device current, on
 *    every call made outside stream capture (so it survives cudaDeviceReset); a call
 *    made while its stream is being captured reuses the last address found, so make
 *    the first call on a device before any stream capture begins.
 *  Results are those of DSPLIB_gpu_firBiquadBatched_bwd with the same inputs. */
DSPLIB_STATUS DSPLIB_gpu_firBiquadBatched_bwdStaticScratch(DSPLIB_gpu_raggedPlan plan, const float *x,
                                                           const float *taps, const float *coefs, const float *work,
                                                           const float *gy, float *gx, float *gtaps, float *gcoefs,
                                                           void *stream);

#ifdef __cplusplus
}
#endif

#endif
