/*
 * DSPLIB_cascadeBiquad: multichannel cascade of second-order IIR sections on a B200.
 *
 * Drop-in for src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad.h of the reference.
 * Every entry point keeps the reference signature, argument meaning and status
 * codes; each declaration cites the interface it replaces.
 *
 * Layouts (reference DSPLIB_cascadeBiquad_cn.cpp:46-150):
 *   in/out   time-major: x[t*pitch + ch], pitch = stride_y / 4 (in and out pitch must match)
 *   state    [(stage*nv + v)*varPitch + ch], nv = 4 (DF1) or 2 (DF2, TDF2, TIF);
 *            read at the start of exec and written back at the end, so
 *            consecutive exec calls continue the stream.
 *   coefficients, NATC: natural [ch][stage][b0 b1 b2 a1 a2] (one row when shared),
 *            H(z) = (b0 + b1 z^-1 + b2 z^-2) / (1 + a1 z^-1 + a2 z^-2).
 *   coefficients, OPTIMIZED: the layout produced by DSPLIB_cascadeBiquad_get_coefficients
 *            (TIF transform with per-7-stage-group gains; channel-interleaved
 *            rows for per-channel coefficients); DF1/DF2/TDF2 with shared
 *            coefficients use the natural layout.
 *
 * funcStyle:
 *   NATC       one sequential recursion per channel in the reference operation
 *              order with separately rounded float operations: bit-exact to the
 *              reference _cn kernels (TIF runs DF2 on natural coefficients, as
 *              the reference NATC path does).
 *   OPTIMIZED  chunked parallel-in-time scan: each chunk runs the form's own
 *              recursion; chunk-boundary states are propagated with the
 *              stage's state-transition matrix raised to the chunk length,
 *              computed in FP64.
 */
#ifndef DSPLIB_CASCADEBIQUAD_H_
#define DSPLIB_CASCADEBIQUAD_H_

#include "DSPLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

#define DSPLIB_NUM_BIQUAD_COEFS (5)
#define DSPLIB_NUM_STATE_VARS_DF1 (4)
#define DSPLIB_NUM_STATE_VARS_DF2 (2)

/** Same values as DSPLIB_cascadeBiquad.h:80-90 of the reference. */
typedef enum {
   DSPLIB_BIQUAD_TIF = 0,
   DSPLIB_BIQUAD_DF1 = 1,
   DSPLIB_BIQUAD_DF2 = 2,
   DSPLIB_BIQUAD_TDF2 = 3,
} DSPLIB_biquadForm;

/** Same fields, order and meaning as DSPLIB_cascadeBiquad.h:95-111 of the reference. */
typedef struct {
   int8_t funcStyle;
   uint32_t dataSize;
   uint32_t numStages;
   uint32_t numChannels;
   uint32_t enableNChCoeffs;
   uint32_t biquadForm;
} DSPLIB_cascadeBiquad_InitArgs;

/** Replaces DSPLIB_cascadeBiquad_getHandleSize (DSPLIB_cascadeBiquad.h:121; .cpp:329-333). */
int32_t DSPLIB_cascadeBiquad_getHandleSize(DSPLIB_cascadeBiquad_InitArgs *pKerInitArgs);

/** Replaces ..._get_coefficientsBufferDesc (DSPLIB_cascadeBiquad.h:147-152; utils.cpp:44-159). */
DSPLIB_STATUS DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(uint32_t dataType,
                                                              uint32_t numStages,
                                                              uint32_t numChannels,
                                                              uint32_t biquadForm,
                                                              uint32_t enableNChCoeffs,
                                                              DSPLIB_bufParams2D_t *pBufParamsFilterCoeffOpt);

/** Replaces ..._get_coefficients (DSPLIB_cascadeBiquad.h:169-174; utils.cpp:652-709).
 *  Host or device buffers.  DF1/DF2/TDF2 with shared coefficients return
 *  DSPLIB_ERR_INVALID_VALUE, as the reference does (utils.cpp:691-694). */
DSPLIB_STATUS DSPLIB_cascadeBiquad_get_coefficients(uint32_t biquadForm,
                                                    uint32_t enableNChCoeffs,
                                                    DSPLIB_bufParams2D_t *pBufParamsFilterCoeff,
                                                    DSPLIB_bufParams2D_t *pBufParamsFilterCoeffOpt,
                                                    const void *pFilterCoeff,
                                                    const void *pFilterCoeffOpt);

/** Replaces DSPLIB_cascadeBiquad_init (DSPLIB_cascadeBiquad.h:198-203; .cpp:419-620). */
DSPLIB_STATUS DSPLIB_cascadeBiquad_init(DSPLIB_kernelHandle handle,
                                        DSPLIB_bufParams2D_t *bufParamsIn,
                                        DSPLIB_bufParams2D_t *bufParamsFilterCoeff,
                                        DSPLIB_bufParams2D_t *bufParamsFilterVar,
                                        DSPLIB_bufParams2D_t *bufParamsOut,
                                        DSPLIB_cascadeBiquad_InitArgs *pKerInitArgs);

/** Replaces ..._init_checkParams (DSPLIB_cascadeBiquad.h:228-233; .cpp:335-399). */
DSPLIB_STATUS DSPLIB_cascadeBiquad_init_checkParams(DSPLIB_kernelHandle handle,
                                                    const DSPLIB_bufParams2D_t *bufParamsIn,
                                                    const DSPLIB_bufParams2D_t *bufParamsFilterCoeff,
                                                    const DSPLIB_bufParams2D_t *bufParamsFilterVar,
                                                    const DSPLIB_bufParams2D_t *bufParamsOut,
                                                    const DSPLIB_cascadeBiquad_InitArgs *pKerInitArgs);

/** Replaces DSPLIB_cascadeBiquad_exec (DSPLIB_cascadeBiquad.h:263-267; .cpp:622-635). */
DSPLIB_STATUS DSPLIB_cascadeBiquad_exec(DSPLIB_kernelHandle handle,
                                        void *pIn,
                                        void *pFilterCoeff,
                                        void *pFilterVar,
                                        void *pOut);

/** Replaces ..._exec_checkParams (DSPLIB_cascadeBiquad.h:287-291; .cpp:401-417). */
DSPLIB_STATUS DSPLIB_cascadeBiquad_exec_checkParams(DSPLIB_kernelHandle handle,
                                                    const void *pIn,
                                                    const void *pFilterCoeff,
                                                    const void *pFilterVar,
                                                    const void *pOut);

/** Replaces DSPLIB_cascadeBiquad_perfEst (DSPLIB_cascadeBiquad.h:312-318; a C7x cycle
 *  model in the reference, .cpp:7-327).  Here: roofline estimate in nanoseconds. */
void DSPLIB_cascadeBiquad_perfEst(DSPLIB_kernelHandle handle,
                                  const DSPLIB_bufParams2D_t *bufParamsIn,
                                  const DSPLIB_bufParams2D_t *bufParamsFilterCoeff,
                                  const DSPLIB_bufParams2D_t *bufParamsFilterVar,
                                  const DSPLIB_bufParams2D_t *bufParamsOut,
                                  uint64_t *archCycles,
                                  uint64_t *estCycles);

#ifdef __cplusplus
}
#endif

#endif /* DSPLIB_CASCADEBIQUAD_H_ */
