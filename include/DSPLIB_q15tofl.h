/*
 * DSPLIB_q15tofl: Q.15 (int16) to IEEE float (FLOAT32 or FLOAT64) conversion on a B200.
 *
 * Drop-in for src/DSPLIB_q15tofl/DSPLIB_q15tofl.h of the reference: same entry
 * points, InitArgs layout, argument meaning and status codes.  The conversion
 * runs in a CUDA kernel; there is no CPU fallback.
 *
 * out[i] = in[i] / 32768, i = 0 .. dataSize-1 (DSPLIB_q15tofl_cn.cpp:33-37).  The
 * quotient is exact in both output types, so both function styles give the
 * reference's results bit for bit.
 *
 * Buffers may be host or device pointers (device: read in place; host: staged).
 */
#ifndef DSPLIB_Q15TOFL_H_
#define DSPLIB_Q15TOFL_H_

#include "DSPLIB_types.h"
#include "DSPLIB_bufParams.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Same fields and order as DSPLIB_q15tofl.h:29-34 of the reference. */
typedef struct {
   int8_t funcStyle;  /**< DSPLIB_FUNCTION_STYLE */
   uint32_t dataSize; /**< elements converted by each exec */
} DSPLIB_q15tofl_InitArgs;

/** Replaces DSPLIB_q15tofl_getHandleSize (DSPLIB_q15tofl.h:44, DSPLIB_q15tofl.cpp:7-14). */
int32_t DSPLIB_q15tofl_getHandleSize(DSPLIB_q15tofl_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_q15tofl_init (DSPLIB_q15tofl.h:67-70, DSPLIB_q15tofl.cpp:64-109): records
 *  dataSize and the output type; DSPLIB_ERR_INVALID_TYPE for an output type other than
 *  FLOAT32/FLOAT64. */
DSPLIB_STATUS DSPLIB_q15tofl_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams1D_t *bufParamsIn,
                                  DSPLIB_bufParams1D_t *bufParamsOut, const DSPLIB_q15tofl_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_q15tofl_init_checkParams (DSPLIB_q15tofl.h:93-97, DSPLIB_q15tofl.cpp:16-44):
 *  NULL handle -> DSPLIB_ERR_NULL_POINTER; input not INT16 or output not FLOAT32/FLOAT64
 *  -> DSPLIB_ERR_INVALID_TYPE. */
DSPLIB_STATUS DSPLIB_q15tofl_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams1D_t *bufParamsIn,
                                              const DSPLIB_bufParams1D_t *bufParamsOut,
                                              const DSPLIB_q15tofl_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_q15tofl_exec_checkParams (DSPLIB_q15tofl.h:116-117, DSPLIB_q15tofl.cpp:46-62). */
DSPLIB_STATUS DSPLIB_q15tofl_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut);

/** Replaces DSPLIB_q15tofl_exec (DSPLIB_q15tofl.h:147, DSPLIB_q15tofl.cpp:111-126). */
DSPLIB_STATUS DSPLIB_q15tofl_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut);

#ifdef __cplusplus
}
#endif

#endif
