/*
 * DSPLIB_fir: multichannel FIR filter ("valid" convolution) on a B200.
 *
 * Drop-in for src/DSPLIB_fir/DSPLIB_fir.h of the reference.  Every entry point
 * keeps the reference signature, argument meaning and status codes; each
 * declaration cites the reference interface it replaces.  Computation runs on
 * the GPU (sm_100a CUDA kernels); there is no CPU fallback.
 *
 * Semantics (reference src/DSPLIB_fir/DSPLIB_fir_cn.cpp:19-87):
 *   y[l][j] = sum_{c=0}^{T-1} x[l][j+c] * h[l'][T-1-c],   j = 0 .. dataSize-T
 * with l' = l when enableNchCoefs = 1 and 0 otherwise.  Buffers are
 * channel-major with byte pitches taken from the descriptors passed to init.
 *
 * funcStyle selects the arithmetic contract:
 *   DSPLIB_FUNCTION_NATC       results identical to the reference natural-C
 *                              kernel: integers wrap modulo 2^bits, floats are
 *                              summed in tap order with separately rounded
 *                              multiply and add (bit-exact to _cn).
 *   DSPLIB_FUNCTION_OPTIMIZED  fast kernels.  Integer types give the same
 *                              wrapped result as NATC unless Q mode is enabled
 *                              (DSPLIB_gpu_firSetQMode, dsplib_gpu.h): then the
 *                              output is round-half-up(acc >> shift) saturated,
 *                              the C7x MMA output-stage convention.  Float
 *                              results use fused multiply-add (plain CUDA-core
 *                              kernel) or split-BF16x3 tensor-core products,
 *                              see DSPLIB_gpu_firSetPrecision.
 *
 * Buffers may live in device memory (fast path; the kernel reads them in
 * place) or in host memory (staged through device buffers inside exec).
 * exec returns after the output is complete unless DSPLIB_gpu_setAsync(h, 1)
 * was called.
 */
#ifndef DSPLIB_FIR_H_
#define DSPLIB_FIR_H_

#include "DSPLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Same fields, order and meaning as DSPLIB_fir.h:30-77 of the reference. */
typedef struct {
   int8_t funcStyle;        /**< DSPLIB_FUNCTION_STYLE */
   int32_t dataSize;        /**< input samples per channel (N) */
   int32_t batchSize;       /**< channels */
   int32_t filterSize;      /**< taps (T) */
   uint32_t shift;          /**< Q-mode right shift of the exact accumulator */
   uint32_t enableNchCoefs; /**< 0: one tap row for all channels, 1: one per channel */
   uint32_t enableMMA;      /**< 1: filter rows use the padded MMA layout (2*MMA_SIZE leading zeros) */
   int32_t MMA_SIZE;        /**< panel width used by the padded layout */
   uint32_t enableQ;        /**< float-in Q-format quantisation flag (accepted, see DSPLIB_gpu_firSetPrecision) */
   uint32_t Q;              /**< Q value for enableQ */
} DSPLIB_fir_InitArgs;

/** Replaces DSPLIB_fir_getHandleSize (reference DSPLIB_fir.h:87, DSPLIB_fir.cpp:7-11). */
int32_t DSPLIB_fir_getHandleSize(DSPLIB_fir_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_fir_getSizes (DSPLIB_fir.h:109-112; DSPLIB_fir.cpp:71-98 -> DSPLIB_fir_ci.cpp:63-103):
 *  out.dim_x = dataSize - filterSize + 1; filter.dim_y = 1 or batchSize; with enableMMA the
 *  filter row is 2*MMA_SIZE + filterSize + MMA_SIZE - 1 elements. */
DSPLIB_STATUS DSPLIB_fir_getSizes(const DSPLIB_fir_InitArgs *pKerInitArgs,
                                  DSPLIB_bufParams2D_t *bufParamsIn,
                                  DSPLIB_bufParams2D_t *bufParamsFilter,
                                  DSPLIB_bufParams2D_t *bufParamsOut);

/** Replaces DSPLIB_fir_init (DSPLIB_fir.h:137-141; DSPLIB_fir.cpp:120-199). */
DSPLIB_STATUS DSPLIB_fir_init(DSPLIB_kernelHandle handle,
                              DSPLIB_bufParams2D_t *bufParamsIn,
                              DSPLIB_bufParams2D_t *bufParamsFilter,
                              DSPLIB_bufParams2D_t *bufParamsOut,
                              DSPLIB_fir_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_fir_init_checkParams (DSPLIB_fir.h:166-171; DSPLIB_fir.cpp:13-69).
 *  Keeps the reference quirk: only FLOAT32 passes this check, although init/exec accept
 *  INT8/INT16/INT32 (reference coverage case DSPLIB_fir_d.c:562-575). */
DSPLIB_STATUS DSPLIB_fir_init_checkParams(DSPLIB_kernelHandle handle,
                                          const DSPLIB_bufParams2D_t *bufParamsIn,
                                          const DSPLIB_bufParams2D_t *bufParamsFilter,
                                          const DSPLIB_bufParams2D_t *bufParamsOut,
                                          const DSPLIB_fir_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_fir_exec (DSPLIB_fir.h:201-202; DSPLIB_fir.cpp:201-215). */
DSPLIB_STATUS DSPLIB_fir_exec(DSPLIB_kernelHandle handle, void *pIn, void *pFilter, void *pOut);

/** Replaces DSPLIB_fir_exec_checkParams (DSPLIB_fir.h:222-225; DSPLIB_fir.cpp:100-118). */
DSPLIB_STATUS DSPLIB_fir_exec_checkParams(DSPLIB_kernelHandle handle,
                                          const void *pIn,
                                          const void *pFilter,
                                          const void *pOut);

/** Replaces DSPLIB_fir_perfEst (DSPLIB_fir.h:244-249; an empty stub in the reference,
 *  DSPLIB_fir_ci.cpp:53-61).  Here: roofline estimate of the exec time in nanoseconds
 *  (archCycles = compute/HBM bound, estCycles = that plus launch overhead). */
void DSPLIB_fir_perfEst(DSPLIB_kernelHandle handle,
                        const DSPLIB_bufParams2D_t *bufParamsIn,
                        const DSPLIB_bufParams2D_t *bufParamsFilter,
                        const DSPLIB_bufParams2D_t *bufParamsOut,
                        uint64_t *archCycles,
                        uint64_t *estCycles);

#ifdef __cplusplus
}
#endif

#endif /* DSPLIB_FIR_H_ */
