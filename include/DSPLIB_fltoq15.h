/*
 * DSPLIB_fltoq15: IEEE float (FLOAT32 or FLOAT64) to Q.15 (int16) conversion on a B200.
 *
 * Drop-in for src/DSPLIB_fltoq15/DSPLIB_fltoq15.h of the reference: same entry
 * points, InitArgs layout, argument meaning and status codes.  The conversion
 * runs in a CUDA kernel; there is no CPU fallback.
 *
 * out[i] = saturate_int16(round(in[i] * 32768)), i = 0 .. dataSize-1, where
 * round is round-half-to-even and saturation maps to [-32768, 32767]
 * (reference DSPLIB_fltoq15.h:18-26).
 *   DSPLIB_FUNCTION_NATC       the natural-C arithmetic of DSPLIB_fltoq15_cn.cpp:35-62,
 *                              restated step by step: truncate, test for an exact
 *                              half with an even integer part, otherwise add or
 *                              subtract 0.5 in the input precision and truncate.
 *                              That add can round: for the single input magnitude
 *                              (0.5 - 2^-25) / 32768 (FLOAT32; (0.5 - 2^-54) / 32768
 *                              for FLOAT64) the result is +-1 instead of 0, as in
 *                              the reference natural-C code.
 *   DSPLIB_FUNCTION_OPTIMIZED  one hardware round-to-nearest-even conversion with
 *                              saturation, as the reference C7x kernel
 *                              (DSPLIB_fltoq15_ci.cpp, __float_to_int / __double_to_int
 *                              then __int_to_short_sat).
 *   Both styles: values whose scaled magnitude reaches 2^31 saturate by sign
 *   (the reference C code converts them to int32 with undefined behaviour);
 *   NaN gives 0.
 *
 * Buffers may be host or device pointers (device: read in place; host: staged).
 */
#ifndef DSPLIB_FLTOQ15_H_
#define DSPLIB_FLTOQ15_H_

#include "DSPLIB_types.h"
#include "DSPLIB_bufParams.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Same fields and order as DSPLIB_fltoq15.h:34-39 of the reference. */
typedef struct {
   int8_t funcStyle;  /**< DSPLIB_FUNCTION_STYLE */
   uint32_t dataSize; /**< elements converted by each exec */
} DSPLIB_fltoq15_InitArgs;

/** Replaces DSPLIB_fltoq15_getHandleSize (DSPLIB_fltoq15.h:49, DSPLIB_fltoq15.cpp:7-14). */
int32_t DSPLIB_fltoq15_getHandleSize(DSPLIB_fltoq15_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_fltoq15_init_checkParams (DSPLIB_fltoq15.h:72-76, DSPLIB_fltoq15.cpp:16-44):
 *  NULL handle -> DSPLIB_ERR_NULL_POINTER; input not FLOAT32/FLOAT64 or output not
 *  INT16 -> DSPLIB_ERR_INVALID_TYPE. */
DSPLIB_STATUS DSPLIB_fltoq15_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams1D_t *bufParamsIn,
                                              const DSPLIB_bufParams1D_t *bufParamsOut,
                                              const DSPLIB_fltoq15_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_fltoq15_init (DSPLIB_fltoq15.h:99-102, DSPLIB_fltoq15.cpp:64-108): records
 *  dataSize and the input type; DSPLIB_ERR_INVALID_TYPE for an input type other than
 *  FLOAT32/FLOAT64 (the output type is checked only by init_checkParams, as in the reference). */
DSPLIB_STATUS DSPLIB_fltoq15_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams1D_t *bufParamsIn,
                                  DSPLIB_bufParams1D_t *bufParamsOut, const DSPLIB_fltoq15_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_fltoq15_exec_checkParams (DSPLIB_fltoq15.h:121-122, DSPLIB_fltoq15.cpp:46-62). */
DSPLIB_STATUS DSPLIB_fltoq15_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut);

/** Replaces DSPLIB_fltoq15_exec (DSPLIB_fltoq15.h:152, DSPLIB_fltoq15.cpp:110-125). */
DSPLIB_STATUS DSPLIB_fltoq15_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut);

#ifdef __cplusplus
}
#endif

#endif
