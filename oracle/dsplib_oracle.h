/*
 * CPU restatement of the DSPLIB filtering path (DSPLIB_fir, DSPLIB_cascadeBiquad).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never linked
 * into it.  Every function cites the reference file:line it restates (paths
 * relative to the reference project root).  Parity of this restatement is
 * pinned by tests/test_oracle.py against (a) the reference's own _cn kernels
 * compiled unmodified into oracle/_ref/ and (b) golden vectors produced by the
 * reference's Python test models (tests/golden/).
 *
 * Buffers follow the reference layouts exactly:
 *   FIR:    channel-major, x[ch*inPitch + t], y[ch*outPitch + j] (pitches in elements)
 *   biquad: time-major,    x[t*inPitch + ch], state[(s*nv + v)*varPitch + ch]
 */
#ifndef DSPLIB_ORACLE_H_
#define DSPLIB_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* dtype codes are DSPLIB_data_type_e values: INT8=0, INT16=1, INT32=2, FLOAT32=12 */

/* Natural-C FIR, reference semantics (src/DSPLIB_fir/DSPLIB_fir_cn.cpp:19-87):
 *   y[l][j] = sum_{c=0}^{T-1} x[l][j+c] * h[f(l) + T-1-c]
 * accumulated in the data type itself (integers wrap modulo 2^bits, floats are
 * summed sequentially in c order with a separately rounded multiply and add).
 * filtPitch is the distance between per-channel tap rows (0 = shared taps). */
void oracle_fir_cn(int dtype, const void *x, const void *h, void *y, int batch, int T, int outSize,
                   int inPitch, int outPitch, int filtPitch);

/* Fixed-point output stage of the C7x MMA FIR path (Q mode):
 *   acc = exact sum;  y = sat_T((acc + 2^(s-1)) >> s)  (s > 0),  y = sat_T(acc)  (s == 0)
 * Rounding/saturation follow src/common/c7504/DSPLIB_configurations.cpp:94-160
 * (X_RE = 1: add half an LSB; X_SAT = 1: saturate to the output type). */
void oracle_fir_floatq(const float *x, const float *h, float *y, int batch, int T, int outSize, int inPitch,
                       int outPitch, int filtPitch, int Q);
void oracle_fir_q(int dtype, const void *x, const void *h, void *y, int batch, int T, int outSize,
                  int inPitch, int outPitch, int filtPitch, int shift);

/* FP64 FIR on float inputs: y64 = sum x*h in double (ground truth). */
void oracle_fir_f64(const float *x, const float *h, double *y, int batch, int T, int outSize, int inPitch,
                    int outPitch, int filtPitch);

/* Direct-form cascade biquads, float32, operation order of
 * src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_cn.cpp (DF2 :84-85, DF1 :230, TDF2 :386-388).
 * form: 1 = DF1, 2 = DF2, 3 = TDF2.  coef: natural [ch][stage][b0 b1 b2 a1 a2]
 * (one row shared when enableNch == 0).  state is read then written back. */
void oracle_biquad_df(int form, const float *x, const float *coef, float *state, float *y, int N, int S, int C,
                      int enableNch, int inPitch, int outPitch, int varPitch);

/* Same recursions evaluated in double (inputs/coefficients widened, state kept in double). */
void oracle_biquad_df_f64(int form, const float *x, const float *coef, double *state, double *y, int N, int S,
                          int C, int enableNch, int inPitch, int outPitch, int varPitch);

/* TI biquad form (TIF).  Per stage, operation order of
 * src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_tif_lStage_ci.cpp:204-214:
 *   out = x + d0;  d0' = (a11*d0) + ((c0*x) + d1);  d1' = (c1*x) + (a12*d0)
 * with c0 = b1/b0 - a1, c1 = b2/b0 - a2, a12 = -a2, a11 = -a1 and the group gain
 * (product of b0 over each 7-stage group) applied after the group's last stage.
 * tifCoef: [ch][stage][4] in storage order {c0, c1, a12, a11}; gains: [ch][group].
 * state: 2 per stage (d0, d1). */
void oracle_biquad_tif(const float *x, const float *tifCoef, const float *gains, float *state, float *y, int N,
                       int S, int C, int enableNch, int inPitch, int outPitch, int varPitch);

/* Number of TIF stage groups: one group up to 7 stages, else ceil(S/7)
 * (src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_utils.cpp:81-93). */
int oracle_tif_num_groups(int S);

/* TIF coefficient transform for one channel (utils.cpp:161-265): from natural
 * [S][5] to tifCoef [S][4] {b1/b0-a1, b2/b0-a2, -a2, -a1} and gains [groups].
 * The reciprocal is the correctly rounded 1/b0. */
void oracle_tif_coefficients(const float *natural, int S, float *tifCoef, float *gains);

/* ------------------------------------------------------------ Q.15 conversions */

/* Float to Q.15, natural-C arithmetic of src/DSPLIB_fltoq15/DSPLIB_fltoq15_cn.cpp:35-62
 * (style 0) or one round-half-to-even conversion with saturation, the reference
 * C7x kernel's __float_to_int / __double_to_int + __int_to_short_sat
 * (DSPLIB_fltoq15_ci.cpp; style 1).  dtype 12 = float input, 13 = double input.
 * Where the reference C code converts a value outside the int32 range (undefined
 * behaviour) this restatement saturates by sign and maps NaN to 0. */
void oracle_fltoq15(int dtype, int style, const void *in, int16_t *out, long long n);

/* Q.15 to float: out = in / 32768 (src/DSPLIB_q15tofl/DSPLIB_q15tofl_cn.cpp:33-37);
 * dtype 12 = float output, 13 = double output. */
void oracle_q15tofl(int dtype, const int16_t *in, void *out, long long n);

/* ------------------------------------------------------------ layout kernels */

/* Strided matrix transpose of DSPLIB_interleave / DSPLIB_deinterleave
 * (src/DSPLIB_matTrans/DSPLIB_matTrans_cn.cpp:41-45): for i < W, j < H
 *   out[(i * strideOut) / elt + j] = in[i + (strideIn / elt) * j]   (strides in bytes). */
void oracle_transpose(int elt, const void *in, void *out, long long W, long long H, long long strideIn,
                      long long strideOut);

/* DSPLIB_addNCh (src/DSPLIB_addNCh/DSPLIB_addNCh_cn.cpp:30-39): out[row*sO + col] is the sum over
 * the inputs in order, starting from zero, in the data type (dtype 12 float, 13 double);
 * strides in elements. */
void oracle_addnch(int dtype, const void *in, void *out, long long samples, long long channels, long long inputs,
                   long long sY, long long sZ, long long sO);

#ifdef __cplusplus
}
#endif

#endif
