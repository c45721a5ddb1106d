/*
 * DSPLIB_deinterleave: split interleaved samples back into channel rows on a B200.
 *
 * Drop-in for src/DSPLIB_deinterleave/DSPLIB_deinterleave.h of the reference: same
 * entry points, InitArgs layout, argument meaning and status codes.
 *
 * Semantics (matrix transpose, src/DSPLIB_deinterleave/DSPLIB_deinterleave.cpp:89-251
 * -> src/DSPLIB_matTrans/DSPLIB_matTrans_cn.cpp:41-45), with W = in.dim_x (channels),
 * H = in.dim_y (samples) and byte strides:
 *   out[(i * out.stride_y) / size + j] = in[i + (in.stride_y / size) * j],  i < W, j < H
 * for 1-, 2-, 4- and 8-byte element types.  Bit-exact in both function styles.
 * Buffers may be host or device pointers.
 */
#ifndef DSPLIB_DEINTERLEAVE_H_
#define DSPLIB_DEINTERLEAVE_H_

#include "DSPLIB_types.h"
#include "DSPLIB_bufParams.h"

#ifdef __cplusplus
extern "C" {
#endif

/** Same fields as DSPLIB_deinterleave.h:40-43 of the reference. */
typedef struct {
   int8_t funcStyle; /**< DSPLIB_FUNCTION_STYLE */
} DSPLIB_deinterleaveInitArgs;

/** Replaces DSPLIB_deinterleave_getHandleSize (DSPLIB_deinterleave.h:53, DSPLIB_deinterleave.cpp:9-16). */
int32_t DSPLIB_deinterleave_getHandleSize(DSPLIB_deinterleaveInitArgs *pKerInitArgs);

/** Replaces DSPLIB_deinterleave_init (DSPLIB_deinterleave.h:74-77, DSPLIB_deinterleave.cpp:89-251). */
DSPLIB_STATUS DSPLIB_deinterleave_init(DSPLIB_kernelHandle handle, DSPLIB_bufParams2D_t *bufParamsIn,
                                       DSPLIB_bufParams2D_t *bufParamsOut,
                                       const DSPLIB_deinterleaveInitArgs *pKerInitArgs);

/** Replaces DSPLIB_deinterleave_init_checkParams (DSPLIB_deinterleave.h:98-101,
 *  DSPLIB_deinterleave.cpp:18-69): one channel, or two packed channels, pass; otherwise the
 *  type list, equal in/out types and the 16-bit (8-bit) dim_x % 2 (% 4) rule apply. */
DSPLIB_STATUS DSPLIB_deinterleave_init_checkParams(DSPLIB_kernelHandle handle, const DSPLIB_bufParams2D_t *bufParamsIn,
                                                   const DSPLIB_bufParams2D_t *bufParamsOut,
                                                   const DSPLIB_deinterleaveInitArgs *pKerInitArgs);

/** Replaces DSPLIB_deinterleave_exec_checkParams (DSPLIB_deinterleave.h:119-120, DSPLIB_deinterleave.cpp:71-87). */
DSPLIB_STATUS DSPLIB_deinterleave_exec_checkParams(DSPLIB_kernelHandle handle, const void *pIn, const void *pOut);

/** Replaces DSPLIB_deinterleave_exec (DSPLIB_deinterleave.h:150, DSPLIB_deinterleave.cpp:253-266). */
DSPLIB_STATUS DSPLIB_deinterleave_exec(DSPLIB_kernelHandle handle, void *pIn, void *pOut);

/** Replaces DSPLIB_deinterleave_perfEst (DSPLIB_deinterleave.h:163-166): B200 roofline estimate
 *  in nanoseconds. */
void DSPLIB_deinterleave_perfEst(DSPLIB_kernelHandle handle, uint64_t *archCycles, uint64_t *estCycles,
                                 uint64_t dataType);

#ifdef __cplusplus
}
#endif

#endif
