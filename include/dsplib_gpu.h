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
 *  (NULL = the legacy default stream, the default). */
DSPLIB_STATUS DSPLIB_gpu_setStream(DSPLIB_kernelHandle handle, void *cudaStream);

/** async = 1: exec returns once the work is queued on the handle's stream
 *  (device buffers only; host buffers always complete before return).
 *  async = 0 (default): exec returns after the results are written. */
DSPLIB_STATUS DSPLIB_gpu_setAsync(DSPLIB_kernelHandle handle, int32_t async);

/** Text of the last failure recorded on this handle ("" when none). */
const char *DSPLIB_gpu_lastError(DSPLIB_kernelHandle handle);

/** Float FIR precision forms for DSPLIB_FUNCTION_OPTIMIZED:
 *  SIMT  = FP32 fused multiply-add on CUDA cores (the plain kernel, default),
 *  BF16X3 = each FP32 operand split into BF16 hi + lo parts, hi*hi + hi*lo + lo*hi
 *           accumulated in FP32 on tcgen05 tensor cores. */
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

/** Number of CUDA kernels this library has launched in this process. */
int64_t DSPLIB_gpu_kernelLaunchCount(void);

#ifdef __cplusplus
}
#endif

#endif
