/*
 * CPU restatement of the DSPLIB filtering path.  TEST INFRASTRUCTURE ONLY
 * (see dsplib_oracle.h); built with -ffp-contract=off so that float
 * multiply-adds round exactly like the reference's host build (x86-64 SSE,
 * no FMA contraction).
 */
#include "dsplib_oracle.h"

#include <math.h>
#include <string.h>

enum { DT_INT8 = 0, DT_INT16 = 1, DT_INT32 = 2, DT_FLOAT32 = 12 };

/* ---------------------------------------------------------------- FIR */

/* src/DSPLIB_fir/DSPLIB_fir_cn.cpp:54-83.  The reference multiplies and adds
 * in the data type itself; for integers that is the exact sum reduced modulo
 * 2^bits, which is what the wide accumulation below followed by the
 * truncating store computes (two's complement wrap). */
void oracle_fir_cn(int dtype, const void *x, const void *h, void *y, int batch, int T, int outSize,
                   int inPitch, int outPitch, int filtPitch)
{
   for (int l = 0; l < batch; l++) {
      for (int j = 0; j < outSize; j++) {
         size_t xo = (size_t) l * inPitch + j;
         size_t ho = (size_t) l * filtPitch;
         size_t yo = (size_t) l * outPitch + j;
         if (dtype == DT_FLOAT32) {
            const float *xf = (const float *) x, *hf = (const float *) h;
            float acc = 0.0f;
            for (int c = 0; c < T; c++) {
               float p = xf[xo + c] * hf[ho + T - 1 - c];
               acc = acc + p;
            }
            ((float *) y)[yo] = acc;
         }
         else {
            uint64_t acc = 0; /* modular arithmetic: exact mod 2^64, truncated below */
            for (int c = 0; c < T; c++) {
               int64_t xv, hv;
               if (dtype == DT_INT8) {
                  xv = ((const int8_t *) x)[xo + c];
                  hv = ((const int8_t *) h)[ho + T - 1 - c];
               }
               else if (dtype == DT_INT16) {
                  xv = ((const int16_t *) x)[xo + c];
                  hv = ((const int16_t *) h)[ho + T - 1 - c];
               }
               else {
                  xv = ((const int32_t *) x)[xo + c];
                  hv = ((const int32_t *) h)[ho + T - 1 - c];
               }
               acc += (uint64_t) xv * (uint64_t) hv;
            }
            if (dtype == DT_INT8) ((int8_t *) y)[yo] = (int8_t) (uint8_t) acc;
            else if (dtype == DT_INT16) ((int16_t *) y)[yo] = (int16_t) (uint16_t) acc;
            else ((int32_t *) y)[yo] = (int32_t) (uint32_t) acc;
         }
      }
   }
}

/* Q-mode output stage: round half up (add 2^(s-1)), arithmetic shift right,
 * saturate (src/common/c7504/DSPLIB_configurations.cpp:94-160, fields
 * X_RE/X_SAT/X_SHIFT at :141-147).  Exact accumulation in 128 bits. */
void oracle_fir_q(int dtype, const void *x, const void *h, void *y, int batch, int T, int outSize,
                  int inPitch, int outPitch, int filtPitch, int shift)
{
   __int128 lo, hi;
   if (dtype == DT_INT8) { lo = INT8_MIN; hi = INT8_MAX; }
   else if (dtype == DT_INT16) { lo = INT16_MIN; hi = INT16_MAX; }
   else { lo = INT32_MIN; hi = INT32_MAX; }
   for (int l = 0; l < batch; l++) {
      for (int j = 0; j < outSize; j++) {
         size_t xo = (size_t) l * inPitch + j;
         size_t ho = (size_t) l * filtPitch;
         size_t yo = (size_t) l * outPitch + j;
         __int128 acc = 0;
         for (int c = 0; c < T; c++) {
            int64_t xv, hv;
            if (dtype == DT_INT8) {
               xv = ((const int8_t *) x)[xo + c];
               hv = ((const int8_t *) h)[ho + T - 1 - c];
            }
            else if (dtype == DT_INT16) {
               xv = ((const int16_t *) x)[xo + c];
               hv = ((const int16_t *) h)[ho + T - 1 - c];
            }
            else {
               xv = ((const int32_t *) x)[xo + c];
               hv = ((const int32_t *) h)[ho + T - 1 - c];
            }
            acc += (__int128) xv * (__int128) hv;
         }
         if (shift > 0) acc = (acc + ((__int128) 1 << (shift - 1))) >> shift;
         if (acc < lo) acc = lo;
         if (acc > hi) acc = hi;
         if (dtype == DT_INT8) ((int8_t *) y)[yo] = (int8_t) acc;
         else if (dtype == DT_INT16) ((int16_t *) y)[yo] = (int16_t) acc;
         else ((int32_t *) y)[yo] = (int32_t) acc;
      }
   }
}

/* FLOAT32 FIR in float Q mode (src/DSPLIB_fir/DSPLIB_fir_ci.cpp:1559-1625 with the
 * helpers src/common/c71/DSPLIB_UTIL_Q_*.h): signal and taps times 2^Q converted to
 * int32 (__float_to_int: round to nearest even, saturating; NaN taken as 0), an exact
 * integer sum, the MMA output stage with X_SHIFT = Q (round half up, arithmetic shift,
 * saturate to int32, src/DSPLIB_fir/DSPLIB_fir_ci.cpp:229-233), then int to float and
 * times 2^-Q (the reciprocal of the scale, exact). */
static int32_t quant_q(float v, float scale)
{
   float p = v * scale; /* one rounding, as the vector multiply */
   if (p != p) return 0;
   double r = nearbyint((double) p); /* the default rounding mode: nearest even */
   if (r >= 2147483647.0) return INT32_MAX;
   if (r <= -2147483648.0) return INT32_MIN;
   return (int32_t) r;
}

void oracle_fir_floatq(const float *x, const float *h, float *y, int batch, int T, int outSize, int inPitch,
                       int outPitch, int filtPitch, int Q)
{
   const float scale = ldexpf(1.0f, Q), unscale = ldexpf(1.0f, -Q);
   for (int l = 0; l < batch; l++) {
      for (int j = 0; j < outSize; j++) {
         size_t xo = (size_t) l * inPitch + j;
         size_t ho = (size_t) l * filtPitch;
         __int128 acc = 0;
         for (int c = 0; c < T; c++)
            acc += (__int128) ((int64_t) quant_q(x[xo + c], scale) * (int64_t) quant_q(h[ho + T - 1 - c], scale));
         if (Q > 0) acc = (acc + ((__int128) 1 << (Q - 1))) >> Q;
         if (acc < INT32_MIN) acc = INT32_MIN;
         if (acc > INT32_MAX) acc = INT32_MAX;
         y[(size_t) l * outPitch + j] = (float) (int32_t) acc * unscale;
      }
   }
}

void oracle_fir_f64(const float *x, const float *h, double *y, int batch, int T, int outSize, int inPitch,
                    int outPitch, int filtPitch)
{
   for (int l = 0; l < batch; l++) {
      for (int j = 0; j < outSize; j++) {
         double acc = 0.0;
         for (int c = 0; c < T; c++)
            acc += (double) x[(size_t) l * inPitch + j + c] * (double) h[(size_t) l * filtPitch + T - 1 - c];
         y[(size_t) l * outPitch + j] = acc;
      }
   }
}

/* ------------------------------------------------------------- biquad */

static int state_vars(int form) { return form == 1 ? 4 : 2; }

/* src/DSPLIB_cascadeBiquad/DSPLIB_cascadeBiquad_cn.cpp:46-150 (DF2),
 * :190-308 (DF1), :348-450 (TDF2).  Stage 0 reads x with inPitch; later
 * stages run in place on y with outPitch. */
void oracle_biquad_df(int form, const float *x, const float *coef, float *state, float *y, int N, int S, int C,
                      int enableNch, int inPitch, int outPitch, int varPitch)
{
   int nv = state_vars(form);
   for (int ch = 0; ch < C; ch++) {
      const float *cf = enableNch ? coef + (size_t) ch * S * 5 : coef;
      for (int s = 0; s < S; s++) {
         float b0 = cf[s * 5 + 0], b1 = cf[s * 5 + 1], b2 = cf[s * 5 + 2], a1 = cf[s * 5 + 3],
               a2 = cf[s * 5 + 4];
         float *st = state + (size_t) (s * nv) * varPitch + ch;
         const float *in = (s == 0) ? x + ch : y + ch;
         int ip = (s == 0) ? inPitch : outPitch;
         float *out = y + ch;
         if (form == 2) {
            float w1 = st[0], w2 = st[varPitch];
            for (int t = 0; t < N; t++) {
               float v = in[(size_t) t * ip];
               float w0 = v - a1 * w1 - a2 * w2;
               float o = b0 * w0 + b1 * w1 + b2 * w2;
               w2 = w1;
               w1 = w0;
               out[(size_t) t * outPitch] = o;
            }
            st[0] = w1;
            st[varPitch] = w2;
         }
         else if (form == 1) {
            float xd1 = st[0], xd2 = st[varPitch], yd1 = st[2 * varPitch], yd2 = st[3 * varPitch];
            for (int t = 0; t < N; t++) {
               float v = in[(size_t) t * ip];
               float o = b0 * v + b1 * xd1 + b2 * xd2 - a1 * yd1 - a2 * yd2;
               xd2 = xd1;
               xd1 = v;
               yd2 = yd1;
               yd1 = o;
               out[(size_t) t * outPitch] = o;
            }
            st[0] = xd1;
            st[varPitch] = xd2;
            st[2 * varPitch] = yd1;
            st[3 * varPitch] = yd2;
         }
         else {
            float w1 = st[0], w2 = st[varPitch];
            for (int t = 0; t < N; t++) {
               float v = in[(size_t) t * ip];
               float o = w1 + v * b0;
               w1 = w2 + v * b1 - a1 * o;
               w2 = v * b2 - a2 * o;
               out[(size_t) t * outPitch] = o;
            }
            st[0] = w1;
            st[varPitch] = w2;
         }
      }
   }
}

void oracle_biquad_df_f64(int form, const float *x, const float *coef, double *state, double *y, int N, int S,
                          int C, int enableNch, int inPitch, int outPitch, int varPitch)
{
   int nv = state_vars(form);
   for (int ch = 0; ch < C; ch++) {
      const float *cf = enableNch ? coef + (size_t) ch * S * 5 : coef;
      for (int s = 0; s < S; s++) {
         double b0 = cf[s * 5 + 0], b1 = cf[s * 5 + 1], b2 = cf[s * 5 + 2], a1 = cf[s * 5 + 3],
                a2 = cf[s * 5 + 4];
         double *st = state + (size_t) (s * nv) * varPitch + ch;
         double *out = y + ch;
         for (int t = 0; t < N; t++) {
            double v = (s == 0) ? (double) x[(size_t) t * inPitch + ch] : out[(size_t) t * outPitch];
            double o;
            if (form == 2) {
               double w0 = v - a1 * st[0] - a2 * st[varPitch];
               o = b0 * w0 + b1 * st[0] + b2 * st[varPitch];
               st[varPitch] = st[0];
               st[0] = w0;
            }
            else if (form == 1) {
               o = b0 * v + b1 * st[0] + b2 * st[varPitch] - a1 * st[2 * varPitch] - a2 * st[3 * varPitch];
               st[varPitch] = st[0];
               st[0] = v;
               st[3 * varPitch] = st[2 * varPitch];
               st[2 * varPitch] = o;
            }
            else {
               o = st[0] + v * b0;
               st[0] = st[varPitch] + v * b1 - a1 * o;
               st[varPitch] = v * b2 - a2 * o;
            }
            out[(size_t) t * outPitch] = o;
         }
      }
   }
}

int oracle_tif_num_groups(int S) { return S <= 7 ? 1 : (S + 6) / 7; }

void oracle_biquad_tif(const float *x, const float *tifCoef, const float *gains, float *state, float *y, int N,
                       int S, int C, int enableNch, int inPitch, int outPitch, int varPitch)
{
   int G = oracle_tif_num_groups(S);
   int per = S <= 7 ? S : 7;
   for (int ch = 0; ch < C; ch++) {
      const float *cf = enableNch ? tifCoef + (size_t) ch * S * 4 : tifCoef;
      const float *gn = enableNch ? gains + (size_t) ch * G : gains;
      for (int t = 0; t < N; t++) {
         float v = (float) x[(size_t) t * inPitch + ch];
         for (int g = 0; g < G; g++) {
            int s0 = g * per, s1 = (g + 1) * per < S ? (g + 1) * per : S;
            for (int s = s0; s < s1; s++) {
               float c0 = cf[s * 4 + 0], c1 = cf[s * 4 + 1], a12 = cf[s * 4 + 2], a11 = cf[s * 4 + 3];
               float *d0p = state + (size_t) (2 * s) * varPitch + ch;
               float *d1p = d0p + varPitch;
               float d0 = *d0p, d1 = *d1p;
               float o = v + d0;
               float t1 = v * c0;
               float t1a = t1 + d1;
               float t0 = a12 * d0;
               float dt = a11 * d0;
               *d0p = dt + t1a;
               float dm = c1 * v;
               *d1p = dm + t0;
               v = o;
            }
            v = v * gn[g];
         }
         y[(size_t) t * outPitch + ch] = v;
      }
   }
}

void oracle_tif_coefficients(const float *natural, int S, float *tifCoef, float *gains)
{
   int G = oracle_tif_num_groups(S);
   int per = S <= 7 ? S : 7;
   for (int g = 0; g < G; g++) {
      float gain = 1.0f;
      int s1 = (g + 1) * per < S ? (g + 1) * per : S;
      for (int s = g * per; s < s1; s++) {
         float b0 = natural[s * 5 + 0];
         float r = 1.0f / b0;
         float b1 = natural[s * 5 + 1] * r;
         float b2 = natural[s * 5 + 2] * r;
         float a1 = -natural[s * 5 + 3];
         float a2 = -natural[s * 5 + 4];
         gain = gain * b0;
         tifCoef[s * 4 + 0] = b1 + a1;
         tifCoef[s * 4 + 1] = b2 + a2;
         tifCoef[s * 4 + 2] = a2;
         tifCoef[s * 4 + 3] = a1;
      }
      gains[g] = gain;
   }
}

/* ---------------------------------------------------------------- Q.15 conversions */

/* float/double -> int32 truncation toward zero; saturating by sign outside the
 * int32 range and 0 for NaN (where the reference's C cast is undefined). */
static int32_t trunc_sat(double v)
{
   if (v != v) return 0;
   if (v >= 2147483647.0) return INT32_MAX;
   if (v <= -2147483648.0) return INT32_MIN;
   return (int32_t) v;
}

static int16_t sat16(int32_t v) { return (int16_t) (v > 32767 ? 32767 : (v < -32768 ? -32768 : v)); }

/* DSPLIB_fltoq15_cn.cpp:36-60, float arithmetic kept in float. */
static int16_t q15_natc_f(float a)
{
   const float m = a * 32768.0f;
   const int32_t ip = trunc_sat(m);
   const float fp = m - (float) ip;
   int32_t r;
   if (ip % 2 == 0 && fabsf(fp) == 0.5f) r = ip;
   else if (a < 0) r = trunc_sat((float) (m - 0.5f));
   else r = trunc_sat((float) (m + 0.5f));
   return sat16(r);
}

/* The same steps for double input (the 0.5f constant widens to 0.5). */
static int16_t q15_natc_d(double a)
{
   const double m = a * 32768.0;
   const int32_t ip = trunc_sat(m);
   const double fp = m - (double) ip;
   int32_t r;
   if (ip % 2 == 0 && fabs(fp) == 0.5) r = ip;
   else if (a < 0) r = trunc_sat(m - 0.5);
   else r = trunc_sat(m + 0.5);
   return sat16(r);
}

/* Round half to even with saturation (the C7x conversion instructions). */
static int16_t q15_rne(double m)
{
   if (m != m) return 0;
   if (m >= 32767.0) return 32767;
   if (m <= -32768.0) return -32768;
   double f = floor(m);
   const double d = m - f;
   if (d > 0.5 || (d == 0.5 && fmod(f, 2.0) != 0.0)) f += 1.0;
   return (int16_t) f;
}

void oracle_fltoq15(int dtype, int style, const void *in, int16_t *out, long long n)
{
   for (long long i = 0; i < n; i++) {
      if (dtype == DT_FLOAT32) {
         const float a = ((const float *) in)[i];
         out[i] = style ? q15_rne((double) (a * 32768.0f)) : q15_natc_f(a);
      }
      else {
         const double a = ((const double *) in)[i];
         out[i] = style ? q15_rne(a * 32768.0) : q15_natc_d(a);
      }
   }
}

void oracle_q15tofl(int dtype, const int16_t *in, void *out, long long n)
{
   for (long long i = 0; i < n; i++) {
      if (dtype == DT_FLOAT32) ((float *) out)[i] = (float) in[i] / 32768.0f;
      else ((double *) out)[i] = (double) in[i] / 32768.0;
   }
}

/* ---------------------------------------------------------------- layout kernels */

void oracle_transpose(int elt, const void *in, void *out, long long W, long long H, long long strideIn,
                      long long strideOut)
{
   const unsigned char *src = (const unsigned char *) in;
   unsigned char *dst = (unsigned char *) out;
   const long long sInE = strideIn / elt;
   for (long long i = 0; i < W; i++)
      for (long long j = 0; j < H; j++)
         memcpy(dst + ((i * strideOut) / elt + j) * elt, src + (i + sInE * j) * elt, (size_t) elt);
}

void oracle_addnch(int dtype, const void *in, void *out, long long samples, long long channels, long long inputs,
                   long long sY, long long sZ, long long sO)
{
   for (long long row = 0; row < channels; row++)
      for (long long col = 0; col < samples; col++) {
         if (dtype == DT_FLOAT32) {
            const float *x = (const float *) in;
            float acc = 0.0f;
            for (long long l = 0; l < inputs; l++) acc = acc + x[row * sY + col + sZ * l];
            ((float *) out)[row * sO + col] = acc;
         }
         else {
            const double *x = (const double *) in;
            double acc = 0.0;
            for (long long l = 0; l < inputs; l++) acc = acc + x[row * sY + col + sZ * l];
            ((double *) out)[row * sO + col] = acc;
         }
      }
}
