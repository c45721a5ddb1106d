/* A C caller of the library, compiled with gcc against include/ only and linked to
 * libdsplib_b200.so: it replays the call sequences of the reference's test drivers
 * (test/DSPLIB_fir/DSPLIB_fir_d.c:101-305, test/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_d.c:123-343)
 * on host buffers, the way an application that links the reference library calls it:
 *   getHandleSize -> malloc(handle) -> [getSizes | get_coefficientsBufferDesc,
 *   get_coefficients] -> init_checkParams -> init -> exec_checkParams -> exec (xN).
 * Inputs are seeded here; every input and output is written to <outdir>/<name>.bin
 * (raw little-endian arrays) for tests/test_c_caller.py to check against the
 * reference's natural-C kernels.  Test infrastructure, not part of the library.
 *
 *   dsplib_caller <outdir>     exit status 0 when every call returned as expected */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "dsplib.h"

static int failures = 0;
static const char *outdir = ".";

#define EXPECT(call, want)                                                                                    \
   do {                                                                                                       \
      DSPLIB_STATUS st_ = (call);                                                                             \
      if (st_ != (want)) {                                                                                    \
         fprintf(stderr, "%s:%d: %s returned %d, expected %d\n", __FILE__, __LINE__, #call, (int) st_, (int) (want)); \
         failures++;                                                                                          \
      }                                                                                                       \
   } while (0)

static uint32_t lcg = 12345u;
static float frand(void) /* uniform in [-1, 1) */
{
   lcg = lcg * 1664525u + 1013904223u;
   return (float) ((lcg >> 8) & 0xFFFFFF) / 8388608.0f - 1.0f;
}

static void dump(const char *name, const void *p, size_t bytes)
{
   char path[512];
   snprintf(path, sizeof(path), "%s/%s.bin", outdir, name);
   FILE *f = fopen(path, "wb");
   if (!f || fwrite(p, 1, bytes, f) != bytes) {
      fprintf(stderr, "cannot write %s\n", path);
      failures++;
   }
   if (f) fclose(f);
}

/* FLOAT32 FIR, per-channel taps: natural C, then optimized on the same handle (the
 * reference driver re-runs init to switch styles, DSPLIB_fir_d.c:291-297). */
static void fir_float(void)
{
   const int B = 3, N = 1000, T = 37;
   DSPLIB_fir_InitArgs a;
   memset(&a, 0, sizeof(a));
   a.dataSize = N;
   a.batchSize = B;
   a.filterSize = T;
   a.enableNchCoefs = 1;
   a.MMA_SIZE = DSPLIB_MMA_SIZE_32_BIT;
   DSPLIB_bufParams2D_t pin = {DSPLIB_FLOAT32, (uint32_t) N, (uint32_t) B, (int32_t) (N * 4)};
   DSPLIB_bufParams2D_t pout = {DSPLIB_FLOAT32, (uint32_t) (N - T + 1), (uint32_t) B, (int32_t) ((N - T + 1) * 4)};
   DSPLIB_bufParams2D_t pfilt = {DSPLIB_FLOAT32, (uint32_t) T, (uint32_t) B, (int32_t) (T * 4)};
   EXPECT(DSPLIB_fir_getSizes(&a, &pin, &pfilt, &pout), DSPLIB_SUCCESS);
   DSPLIB_kernelHandle h = malloc((size_t) DSPLIB_fir_getHandleSize(&a));
   float *x = malloc((size_t) pin.stride_y * B), *f = malloc((size_t) pfilt.stride_y * B);
   float *y0 = malloc((size_t) pout.stride_y * B), *y1 = malloc((size_t) pout.stride_y * B);
   for (int i = 0; i < B * N; i++) x[i] = frand();
   for (int i = 0; i < B * T; i++) f[i] = frand() / 8.0f;
   a.funcStyle = DSPLIB_FUNCTION_NATC;
   EXPECT(DSPLIB_fir_init_checkParams(h, &pin, &pfilt, &pout, &a), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_fir_init(h, &pin, &pfilt, &pout, &a), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_fir_exec_checkParams(h, x, f, y0), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_fir_exec(h, x, f, y0), DSPLIB_SUCCESS);
   a.funcStyle = DSPLIB_FUNCTION_OPTIMIZED;
   EXPECT(DSPLIB_fir_init(h, &pin, &pfilt, &pout, &a), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_fir_exec(h, x, f, y1), DSPLIB_SUCCESS);
   dump("fir_f32_x", x, (size_t) B * N * 4);
   dump("fir_f32_h", f, (size_t) B * T * 4);
   dump("fir_f32_natc", y0, (size_t) B * (N - T + 1) * 4);
   dump("fir_f32_opt", y1, (size_t) B * (N - T + 1) * 4);
   EXPECT(DSPLIB_fir_exec_checkParams(h, NULL, f, y1), DSPLIB_ERR_NULL_POINTER);
   EXPECT(DSPLIB_gpu_releaseHandle(h), DSPLIB_SUCCESS);
   free(h), free(x), free(f), free(y0), free(y1);
}

/* FLOAT32 FIR with the MMA filter layout (enableMMA = 1): getSizes pads each tap row,
 * the driver writes the taps 2 * MMA_SIZE elements in (DSPLIB_fir_d.c:195-208). */
static void fir_float_mma(void)
{
   const int B = 2, N = 700, T = 20;
   DSPLIB_fir_InitArgs a;
   memset(&a, 0, sizeof(a));
   a.funcStyle = DSPLIB_FUNCTION_OPTIMIZED;
   a.dataSize = N;
   a.batchSize = B;
   a.filterSize = T;
   a.enableNchCoefs = 1;
   a.enableMMA = 1;
   a.MMA_SIZE = DSPLIB_MMA_SIZE_32_BIT;
   DSPLIB_bufParams2D_t pin = {DSPLIB_FLOAT32, (uint32_t) N, (uint32_t) B, (int32_t) (N * 4)};
   DSPLIB_bufParams2D_t pout = {DSPLIB_FLOAT32, (uint32_t) (N - T + 1), (uint32_t) B, (int32_t) ((N - T + 1) * 4)};
   DSPLIB_bufParams2D_t pfilt = {DSPLIB_FLOAT32, (uint32_t) T, (uint32_t) B, (int32_t) (T * 4)};
   EXPECT(DSPLIB_fir_getSizes(&a, &pin, &pfilt, &pout), DSPLIB_SUCCESS);
   const int pitch = pfilt.stride_y / 4, lead = 2 * a.MMA_SIZE;
   DSPLIB_kernelHandle h = malloc((size_t) DSPLIB_fir_getHandleSize(&a));
   float *x = malloc((size_t) pin.stride_y * B), *f = calloc((size_t) pitch * B, 4);
   float *taps = malloc((size_t) B * T * 4), *y = malloc((size_t) pout.stride_y * B);
   for (int i = 0; i < B * N; i++) x[i] = frand();
   for (int i = 0; i < B * T; i++) taps[i] = frand() / 4.0f;
   for (int l = 0; l < B; l++) memcpy(f + (size_t) l * pitch + lead, taps + (size_t) l * T, (size_t) T * 4);
   EXPECT(DSPLIB_fir_init(h, &pin, &pfilt, &pout, &a), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_fir_exec(h, x, f, y), DSPLIB_SUCCESS);
   dump("fir_mma_x", x, (size_t) B * N * 4);
   dump("fir_mma_h", taps, (size_t) B * T * 4);
   dump("fir_mma_opt", y, (size_t) B * (N - T + 1) * 4);
   free(h), free(x), free(f), free(taps), free(y);
}

/* INT16 FIR: init_checkParams rejects non-float types (DSPLIB_fir.cpp:54-66, coverage
 * case 1010), init accepts them; natural C wraps modulo 2^16. */
static void fir_int16(void)
{
   const int B = 4, N = 512, T = 64;
   DSPLIB_fir_InitArgs a;
   memset(&a, 0, sizeof(a));
   a.funcStyle = DSPLIB_FUNCTION_NATC;
   a.dataSize = N;
   a.batchSize = B;
   a.filterSize = T;
   a.MMA_SIZE = DSPLIB_MMA_SIZE_16_BIT;
   DSPLIB_bufParams2D_t pin = {DSPLIB_INT16, (uint32_t) N, (uint32_t) B, (int32_t) (N * 2)};
   DSPLIB_bufParams2D_t pout = {DSPLIB_INT16, (uint32_t) (N - T + 1), (uint32_t) B, (int32_t) ((N - T + 1) * 2)};
   DSPLIB_bufParams2D_t pfilt = {DSPLIB_INT16, (uint32_t) T, 1, (int32_t) (T * 2)};
   EXPECT(DSPLIB_fir_getSizes(&a, &pin, &pfilt, &pout), DSPLIB_SUCCESS);
   DSPLIB_kernelHandle h = malloc((size_t) DSPLIB_fir_getHandleSize(&a));
   int16_t *x = malloc((size_t) B * N * 2), *f = malloc((size_t) T * 2), *y = malloc((size_t) B * (N - T + 1) * 2);
   for (int i = 0; i < B * N; i++) x[i] = (int16_t) (frand() * 32767.0f);
   for (int i = 0; i < T; i++) f[i] = (int16_t) (frand() * 32767.0f);
   EXPECT(DSPLIB_fir_init_checkParams(h, &pin, &pfilt, &pout, &a), DSPLIB_ERR_INVALID_TYPE);
   EXPECT(DSPLIB_fir_init(h, &pin, &pfilt, &pout, &a), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_fir_exec(h, x, f, y), DSPLIB_SUCCESS);
   dump("fir_i16_x", x, (size_t) B * N * 2);
   dump("fir_i16_h", f, (size_t) T * 2);
   dump("fir_i16_natc", y, (size_t) B * (N - T + 1) * 2);
   free(h), free(x), free(f), free(y);
}

/* Stable sections with natural coefficients [b0 b1 b2 a1 a2]: poles at radius r, angle th. */
static void sections(float *c, int S)
{
   for (int s = 0; s < S; s++) {
      const float r = 0.6f + 0.3f * (frand() * 0.5f + 0.5f), cs = frand();
      c[5 * s + 0] = 0.3f + 0.2f * frand();
      c[5 * s + 1] = 0.2f * frand();
      c[5 * s + 2] = 0.1f * frand();
      c[5 * s + 3] = -2.0f * r * cs;
      c[5 * s + 4] = r * r;
   }
}

/* Cascade biquad over numBlocks consecutive blocks of one signal, the state buffer
 * carrying the history (DSPLIB_cascadeBiquad_d.c:260-273).  OPTIMIZED calls take the
 * buffer get_coefficients makes (DSPLIB_cascadeBiquad_d.c:198-224). */
static void biquad(const char *tag, uint32_t form, int style, int nch, int C, int N, int S, int blocks)
{
   const int nv = form == DSPLIB_BIQUAD_DF1 ? 4 : 2;
   DSPLIB_cascadeBiquad_InitArgs a;
   memset(&a, 0, sizeof(a));
   a.funcStyle = (int8_t) style;
   a.dataSize = (uint32_t) N;
   a.numStages = (uint32_t) S;
   a.numChannels = (uint32_t) C;
   a.enableNChCoeffs = (uint32_t) nch;
   a.biquadForm = form;
   const int rows = nch ? C : 1;
   DSPLIB_bufParams2D_t pin = {DSPLIB_FLOAT32, (uint32_t) C, (uint32_t) N, (int32_t) (C * 4)};
   DSPLIB_bufParams2D_t pout = pin;
   DSPLIB_bufParams2D_t pvar = {DSPLIB_FLOAT32, (uint32_t) C, (uint32_t) (S * nv), (int32_t) (C * 4)};
   DSPLIB_bufParams2D_t pnat = {DSPLIB_FLOAT32, (uint32_t) (5 * S), (uint32_t) rows, (int32_t) (5 * S * 4)};
   DSPLIB_bufParams2D_t popt;
   float *nat = malloc((size_t) rows * 5 * S * 4), *coef = nat;
   for (int r = 0; r < rows; r++) sections(nat + (size_t) r * 5 * S, S);
   DSPLIB_bufParams2D_t *pcoef = &pnat;
   if (style == DSPLIB_FUNCTION_OPTIMIZED && (form == DSPLIB_BIQUAD_TIF || nch)) {
      EXPECT(DSPLIB_cascadeBiquad_get_coefficientsBufferDesc(DSPLIB_FLOAT32, (uint32_t) S, (uint32_t) C, form,
                                                             (uint32_t) nch, &popt),
             DSPLIB_SUCCESS);
      coef = calloc((size_t) popt.dim_y * (size_t) popt.stride_y, 1);
      EXPECT(DSPLIB_cascadeBiquad_get_coefficients(form, (uint32_t) nch, &pnat, &popt, nat, coef), DSPLIB_SUCCESS);
      pcoef = &popt;
   }
   DSPLIB_kernelHandle h = malloc((size_t) DSPLIB_cascadeBiquad_getHandleSize(&a));
   float *x = malloc((size_t) blocks * N * C * 4), *y = malloc((size_t) blocks * N * C * 4);
   float *var = calloc((size_t) S * nv * C, 4);
   for (int i = 0; i < blocks * N * C; i++) x[i] = frand();
   EXPECT(DSPLIB_cascadeBiquad_init_checkParams(h, &pin, pcoef, &pvar, &pout, &a), DSPLIB_SUCCESS);
   EXPECT(DSPLIB_cascadeBiquad_init(h, &pin, pcoef, &pvar, &pout, &a), DSPLIB_SUCCESS);
   for (int b = 0; b < blocks; b++) {
      float *xb = x + (size_t) b * N * C, *yb = y + (size_t) b * N * C;
      EXPECT(DSPLIB_cascadeBiquad_exec_checkParams(h, xb, coef, var, yb), DSPLIB_SUCCESS);
      EXPECT(DSPLIB_cascadeBiquad_exec(h, xb, coef, var, yb), DSPLIB_SUCCESS);
   }
   char name[64];
   snprintf(name, sizeof(name), "bq_%s_x", tag);
   dump(name, x, (size_t) blocks * N * C * 4);
   snprintf(name, sizeof(name), "bq_%s_nat", tag);
   dump(name, nat, (size_t) rows * 5 * S * 4);
   snprintf(name, sizeof(name), "bq_%s_y", tag);
   dump(name, y, (size_t) blocks * N * C * 4);
   snprintf(name, sizeof(name), "bq_%s_var", tag);
   dump(name, var, (size_t) S * nv * C * 4);
   EXPECT(DSPLIB_gpu_releaseHandle(h), DSPLIB_SUCCESS);
   if (coef != nat) free(coef);
   free(nat), free(h), free(x), free(y), free(var);
}

int main(int argc, char **argv)
{
   if (argc > 1) outdir = argv[1];
   fir_float();
   fir_float_mma();
   fir_int16();
   /* tag, form, style, per-channel coefficients, channels, samples per block, stages, blocks */
   biquad("df2_natc", DSPLIB_BIQUAD_DF2, DSPLIB_FUNCTION_NATC, 0, 8, 500, 3, 2);
   biquad("df1_natc_nch", DSPLIB_BIQUAD_DF1, DSPLIB_FUNCTION_NATC, 1, 5, 300, 2, 1);
   biquad("df2_opt_nch", DSPLIB_BIQUAD_DF2, DSPLIB_FUNCTION_OPTIMIZED, 1, 40, 4000, 4, 2);
   biquad("tdf2_opt_nch", DSPLIB_BIQUAD_TDF2, DSPLIB_FUNCTION_OPTIMIZED, 1, 17, 600, 3, 1);
   biquad("tif_opt", DSPLIB_BIQUAD_TIF, DSPLIB_FUNCTION_OPTIMIZED, 0, 33, 2000, 9, 2);
   printf("%d failed calls\n", failures);
   return failures == 0 ? 0 : 1;
}
