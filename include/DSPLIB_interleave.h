/*
 * DSPLIB_interleave: interleave the rows of a matrix (channel rows -> one sample
 * row per time step) on a B200.
 *
 * Drop-in for src/DSPLIB_interleave/DSPLIB_interleave.h of the reference: same
 * entry points, InitArgs layout, argument meaning and status codes.
 *
 * Semantics (the reference runs the matrix-transpose kernel for every shape,
 * src/DSPLIB_interleave/DSPLIB_interleave.cpp:89-253 -> src/DSPLIB_matTrans/
 * DSPLIB_matTrans_cn.cpp:41-45), with W = in.dim_x, H = in.dim_y and byte strides:
 *   out[(i * out.stride_y) / size + j] = in[i + (in.stride_y / size) * j],  i < W, j < H
 * for 1-, 2-, 4- and 8-byte element types (INT8..UINT64, FLOAT32, FLOAT64).  Pure
 * data movement: both function styles give identical, bit-exact results.
 * Buffers may be host or device pointers.
 */
#ifndef DSPLIB_INTERLEAVE_H_
#define DSPLIB_INTERLEAVE_H_

#include "DSPLIB_types.h"
#include "DSPLIB_bufParams.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Same fields as DSPLIB_interleave.h:40-43 of the reference. */
typedef struct {
   int8_t funcStyle; /**< DSPLIB_FUNCTION_STYLE */
} DSPLIB_interleaveInitArgs;

/** Replaces DSPLIB_interleave_getHandleSize (DSPLIB_interleave.h:53, DSPLIB_interleave.cpp:9-16). */
int32_t DSPLIB_interleave_getHandleSize(DSPLIB_interleaveInitArgs *pKerInitArgs);

/** Replaces DSPLIB_interleave_init (DSPLIB_interleave.h:74-77, DSPLIB_interleave.cpp:89-253):
 *  DSPLIB_ERR_INVALID_TYPE for an input type outside the ten supported ones. */
DSPLIB_STATUS DSPLIB_interleave_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams2D_t *bufParamsIn,
                                     DSPLIB_bufParams2D_t *bufParamsOut, const DSPLIB_interleaveInitArgs *pKerInitArgs);

/** Replaces DSPLIB_interleave_init_checkParams (DSPLIB_interleave.h:98-101, DSPLIB_interleave.cpp:18-69),
 *  with its order of checks: for in.dim_y of 1 or 2 with a packed output row only the type list
 *  applies; otherwise in/out types must match and 16-bit (8-bit) rows need dim_x % 2 (% 4) == 0
 *  (DSPLIB_ERR_INVALID_VALUE), and that branch's verdict replaces the type-list one. */
DSPLIB_STATUS DSPLIB_interleave_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams2D_t *bufParamsIn,
                                                 const DSPLIB_bufParams2D_t *bufParamsOut,
                                                 const DSPLIB_interleaveInitArgs *pKerInitArgs);

/** Replaces DSPLIB_interleave_exec_checkParams (DSPLIB_interleave.h:119-120, DSPLIB_interleave.cpp:71-87). */
DSPLIB_STATUS DSPLIB_interleave_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut);

/** Replaces DSPLIB_interleave_exec (DSPLIB_interleave.h:149, DSPLIB_interleave.cpp:255-268). */
DSPLIB_STATUS DSPLIB_interleave_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut);

/** Replaces DSPLIB_interleave_perfEst (DSPLIB_interleave.h:161): B200 roofline estimate in
 *  nanoseconds (bytes moved / HBM bandwidth; estCycles adds launch and synchronisation). */
void DSPLIB_interleave_perfEst(DSPLIB_kernelHandle handle, uint64_t *archCycles, uint64_t *estCycles);

#ifdef __cplusplus
}
#endif

#endif
