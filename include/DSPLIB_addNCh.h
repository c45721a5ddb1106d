/*
 * DSPLIB_addNCh: element-wise sum of several stacked multichannel inputs on a B200.
 *
 * Drop-in for src/DSPLIB_addNCh/DSPLIB_addNCh.h of the reference: same entry
 * points, InitArgs layout, argument meaning and status codes.
 *
 * Semantics (src/DSPLIB_addNCh/DSPLIB_addNCh_cn.cpp:30-39), FLOAT32 or FLOAT64, with
 * samples = in.dim_x, channels = in.dim_y, inputs = in.dim_z and element strides
 * sY = in.stride_y / size, sZ = in.stride_z / size, sO = out.stride_y / size:
 *   out[row * sO + col] = ((0 + in[row*sY + col]) + in[row*sY + col + sZ]) + ...
 * summed in input order from zero in the data type, so both function styles are
 * bit-exact to the reference natural-C kernel.
 * Buffers may be host or device pointers.
 */
#ifndef DSPLIB_ADDNCH_H_
#define DSPLIB_ADDNCH_H_

#include "DSPLIB_types.h"
#include "DSPLIB_bufParams.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Same fields as DSPLIB_addNCh.h:70-74 of the reference. */
typedef struct {
   int8_t funcStyle; /**< DSPLIB_FUNCTION_STYLE */
} DSPLIB_addNCh_InitArgs;

/** Replaces DSPLIB_addNCh_getHandleSize (DSPLIB_addNCh.h:84, DSPLIB_addNCh.cpp:7-11). */
int32_t DSPLIB_addNCh_getHandleSize(DSPLIB_addNCh_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_addNCh_init (DSPLIB_addNCh.h:107-110, DSPLIB_addNCh.cpp:60-133):
 *  DSPLIB_ERR_INVALID_TYPE unless the input is FLOAT32 or FLOAT64. */
DSPLIB_STATUS DSPLIB_addNCh_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams3D_t *bufParamsIn,
                                 DSPLIB_bufParams2D_t *bufParamsOut, const DSPLIB_addNCh_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_addNCh_init_checkParams (DSPLIB_addNCh.h:133-137, DSPLIB_addNCh.cpp:13-41):
 *  NULL handle -> NULL_POINTER; input not FLOAT32/FLOAT64, or output type different -> INVALID_TYPE. */
DSPLIB_STATUS DSPLIB_addNCh_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams3D_t *bufParamsIn,
                                             const DSPLIB_bufParams2D_t *bufParamsOut,
                                             const DSPLIB_addNCh_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_addNCh_exec_checkParams (DSPLIB_addNCh.h:156-157, DSPLIB_addNCh.cpp:43-58). */
DSPLIB_STATUS DSPLIB_addNCh_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut);

/** Replaces DSPLIB_addNCh_exec (DSPLIB_addNCh.h:187-188, DSPLIB_addNCh.cpp:135-146). */
DSPLIB_STATUS DSPLIB_addNCh_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut);

/** Replaces DSPLIB_addNCh_perfEst (DSPLIB_addNCh.h:202): B200 roofline estimate in nanoseconds. */
void DSPLIB_addNCh_perfEst(DSPLIB_kernelHandle handle, uint64_t *archCycles, uint64_t *estCycles, uint32_t dataType);

#ifdef __cplusplus
}
#endif

#endif
