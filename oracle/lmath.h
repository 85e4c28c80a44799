/*
 * ORACLE (test infrastructure; never shipped, never measured as the product).
 *
 * Float32 elementary functions written from their mathematics, with every operation spelled out (explicit fmaf,
 * no contraction), so that the CPU restatement and the CUDA engine evaluate them to the same bits. The reference
 * evaluates exp / log / sin / cos / arccos / cbrt / erf_inv through XLA (src/lumen/transport/step.py:338,
 * src/lumen/media/phase.py:43-57, src/lumen/sources/_base.py:318); these are accurate to a few float32 ulps.
 *
 *  - exp: Cody-Waite reduction by ln 2 (a two-part split of ln 2), degree-7 Taylor polynomial on |r| <= ln2 / 2.
 *  - log: x = 2^e m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m - 1) / (m + 1), odd series to s^11.
 *  - sin / cos: reduction by pi/2 (a three-part Cody-Waite split), Taylor polynomials on |r| <= pi/4.
 *  - sin / cos of 2 pi u: exact quarter-turn reduction of 4u, then the same polynomials.
 *  - asin / acos: asin x = x + x^3 P(x^2) on |x| <= 1/2 (P a least-squares fit on Chebyshev nodes, float64, to
 *    (asin x - x) / x^3), acos by the half-angle identities beyond.
 *  - cbrt: exp(log|x| / 3) and one Newton step; in float64 that root and two Newton steps in float64.
 *  - erfinv: M. Giles, "Approximating the erfinv function" (GPU Computing Gems Jade, 2011), single precision.
 */
#ifndef LUMEN_ORACLE_LMATH_H
#define LUMEN_ORACLE_LMATH_H

#include <math.h>
#include <stdint.h>
#include <string.h>

static inline float o_bits_f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t o_f_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* 2^k as a float, k in [-126, 127] */
static inline float o_pow2i(int k) { return o_bits_f((uint32_t)(k + 127) << 23); }

static inline float o_exp(float x) {
  if (!(x == x)) return x;
  if (x > 88.72283935546875f) return INFINITY;
  if (x < -103.972084045410f) return 0.0f;
  const float L2E = 1.44269502162933349609f;
  const float LN2_HI = 0.693145751953125f;        /* ln 2 rounded to 16 significant bits: k * LN2_HI exact */
  const float LN2_LO = 1.42860682030941723212e-6f; /* ln 2 - LN2_HI */
  float kf = floorf(x * L2E + 0.5f);
  float r = x - kf * LN2_HI;
  r = r - kf * LN2_LO;
  float p = 1.98412698412698412526e-4f;            /* 1/7! */
  p = fmaf(p, r, 1.38888888888888894189e-3f);     /* 1/6! */
  p = fmaf(p, r, 8.33333333333333321769e-3f);     /* 1/5! */
  p = fmaf(p, r, 4.16666666666666643537e-2f);     /* 1/4! */
  p = fmaf(p, r, 1.66666666666666657415e-1f);     /* 1/3! */
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  int k = (int)kf;
  if (k > 127) return (p * o_pow2i(127)) * o_pow2i(k - 127);
  if (k < -126) return (p * o_pow2i(k + 100)) * o_pow2i(-100);
  return p * o_pow2i(k);
}

static inline float o_log(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? -INFINITY : NAN;
  if (x == INFINITY) return x;
  int adj = 0;
  if (x < 1.17549435e-38f) { x = x * 8388608.0f; adj = -23; }
  uint32_t u = o_f_bits(x);
  int e = (int)((u >> 23) & 0xff) - 127 + adj;
  float m = o_bits_f((u & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984f) { m = m * 0.5f; e = e + 1; }
  float f = m - 1.0f;
  float s = f / (2.0f + f);
  float z = s * s;
  float p = 0.181818181818181823f;                 /* 2/11 */
  p = fmaf(p, z, 0.222222222222222210f);          /* 2/9 */
  p = fmaf(p, z, 0.285714285714285698f);          /* 2/7 */
  p = fmaf(p, z, 0.400000000000000022f);          /* 2/5 */
  p = fmaf(p, z, 0.666666666666666630f);          /* 2/3 */
  float lm = fmaf(s * z, p, 2.0f * s);
  const float LN2_HI = 0.693145751953125f;
  const float LN2_LO = 1.42860682030941723212e-6f;
  float ef = (float)e;
  return fmaf(ef, LN2_HI, fmaf(ef, LN2_LO, lm));
}

/* sin and cos of r, |r| <= pi/4 (Taylor) */
static inline void o_sincos_poly(float r, float* s, float* c) {
  float z = r * r;
  float ps = 2.75573192239858906526e-6f;           /* 1/9! */
  ps = fmaf(ps, z, -1.98412698412698412526e-4f);  /* -1/7! */
  ps = fmaf(ps, z, 8.33333333333333321769e-3f);   /* 1/5! */
  ps = fmaf(ps, z, -1.66666666666666657415e-1f);  /* -1/3! */
  *s = fmaf(r * z, ps, r);
  float pc = -2.75573192239858906526e-7f;          /* -1/10! */
  pc = fmaf(pc, z, 2.48015873015873015658e-5f);   /* 1/8! */
  pc = fmaf(pc, z, -1.38888888888888894189e-3f);  /* -1/6! */
  pc = fmaf(pc, z, 4.16666666666666643537e-2f);   /* 1/4! */
  pc = fmaf(pc, z, -0.5f);
  *c = fmaf(z, pc, 1.0f);
}

static inline void o_quadrant(int q, float s, float c, float* so, float* co) {
  switch (q & 3) {
    case 0: *so = s; *co = c; break;
    case 1: *so = c; *co = -s; break;
    case 2: *so = -s; *co = -c; break;
    default: *so = -c; *co = s; break;
  }
}

/* sin and cos of 2 pi u (u a float in [0, 1]: the reduction 4u - round(4u) is exact) */
static inline void o_sincos2pi(float u, float* s, float* c) {
  float v = 4.0f * u;
  float q = floorf(v + 0.5f);
  float f = v - q;
  float r = f * 1.57079632679489661923f;
  float ss, cc;
  o_sincos_poly(r, &ss, &cc);
  o_quadrant((int)q, ss, cc, s, c);
}

/* sin and cos of a moderate angle (|x| < 1e4) */
static inline void o_sincos(float x, float* s, float* c) {
  const float TWO_OVER_PI = 0.636619772367581343076f;
  const float P1 = 1.5703125f;                     /* pi/2 split in three parts (8 + 16 + rest bits) */
  const float P2 = 4.83512878417968750000e-4f;
  const float P3 = 3.13855707717955556e-7f;
  float q = floorf(x * TWO_OVER_PI + 0.5f);
  float r = x - q * P1;
  r = r - q * P2;
  r = r - q * P3;
  float ss, cc;
  o_sincos_poly(r, &ss, &cc);
  o_quadrant((int)q, ss, cc, s, c);
}

/* asin x for |x| <= 1/2: x + x^3 P(x^2) */
static inline float o_asin_small(float x) {
  float z = x * x;
  float p = 3.38055603e-02f;
  p = fmaf(p, z, 1.70779899e-02f);
  p = fmaf(p, z, 3.11161242e-02f);
  p = fmaf(p, z, 4.45980355e-02f);
  p = fmaf(p, z, 7.50009865e-02f);
  p = fmaf(p, z, 1.66666657e-01f);
  return fmaf(x * z, p, x);
}

static inline float o_acos(float x) {
  const float PI = 3.14159265358979323846f;
  const float PIO2 = 1.57079632679489661923f;
  if (x > 1.0f) x = 1.0f;
  if (x < -1.0f) x = -1.0f;
  if (x <= 0.5f && x >= -0.5f) return PIO2 - o_asin_small(x);
  if (x > 0.5f) return 2.0f * o_asin_small(sqrtf((1.0f - x) * 0.5f));
  return PI - 2.0f * o_asin_small(sqrtf((1.0f + x) * 0.5f));
}

static inline float o_asin(float v) {
  const float PIO2 = 1.57079632679489661923f;
  float a = fabsf(v);
  if (a > 1.0f) a = 1.0f;
  float r = a <= 0.5f ? o_asin_small(a) : PIO2 - 2.0f * o_asin_small(sqrtf((1.0f - a) * 0.5f));
  return v < 0.0f ? -r : r;
}

/* atan2 from asin / acos on the octant where each is well conditioned */
static inline float o_atan2(float y, float x) {
  const float PI = 3.14159265358979323846f;
  float r = sqrtf(x * x + y * y);
  if (r == 0.0f) return 0.0f;
  float a;
  if (fabsf(y) <= fabsf(x)) {
    a = o_asin(fabsf(y) / r);
    if (x < 0.0f) a = PI - a;
  } else {
    a = o_acos(x / r);
  }
  return y < 0.0f ? -a : a;
}

static inline float o_cbrt(float x) {
  if (x == 0.0f) return 0.0f;
  float a = x < 0.0f ? -x : x;
  float y = o_exp(o_log(a) * 0.333333343267440796f);
  y = y - (y * y * y - a) / (3.0f * y * y);
  return x < 0.0f ? -y : y;
}

/* the cube root in float64 (the float64 navigator's torus): the float32 cube root of |x| (brought into float32's
   normal range by powers of 2^96) as the start, then two Newton steps on y^3 = |x| */
static inline double o_cbrt64(double x) {
  if (x == 0.0) return 0.0;
  double a = x < 0.0 ? -x : x;
  int k = 0;
  for (int i = 0; i < 12 && a < 1e-30; ++i) { a = a * 79228162514264337593543950336.0; --k; }
  for (int i = 0; i < 12 && a > 1e30; ++i) { a = a * 1.26217744835361888865876570445245796747713029617443680e-29; ++k; }
  double y = (double)o_cbrt((float)a);
  y = y - (y * y * y - a) / (3.0 * y * y);
  y = y - (y * y * y - a) / (3.0 * y * y);
  for (; k < 0; ++k) y = y * 2.3283064365386962890625e-10;
  for (; k > 0; --k) y = y * 4294967296.0;
  return x < 0.0 ? -y : y;
}

/* M. Giles' single-precision erfinv (published coefficients), x in (-1, 1) */
static inline float o_erfinv(float x) {
  float w = -o_log((1.0f - x) * (1.0f + x));
  float p;
  if (w < 5.0f) {
    w = w - 2.5f;
    p = 2.81022636e-08f;
    p = fmaf(p, w, 3.43273939e-07f);
    p = fmaf(p, w, -3.5233877e-06f);
    p = fmaf(p, w, -4.39150654e-06f);
    p = fmaf(p, w, 0.00021858087f);
    p = fmaf(p, w, -0.00125372503f);
    p = fmaf(p, w, -0.00417768164f);
    p = fmaf(p, w, 0.246640727f);
    p = fmaf(p, w, 1.50140941f);
  } else {
    w = sqrtf(w) - 3.0f;
    p = -0.000200214257f;
    p = fmaf(p, w, 0.000100950558f);
    p = fmaf(p, w, 0.00134934322f);
    p = fmaf(p, w, -0.00367342844f);
    p = fmaf(p, w, 0.00573950773f);
    p = fmaf(p, w, -0.0076224613f);
    p = fmaf(p, w, 0.00943887047f);
    p = fmaf(p, w, 1.00167406f);
    p = fmaf(p, w, 2.83297682f);
  }
  return p * x;
}

/* log(1 + x) and exp(y) - 1 by Kahan's corrections (D. Goldberg, "What every computer scientist should know about
   floating-point arithmetic", 1991, Theorem 4): exact where the plain forms cancel */
static inline float o_log1p(float x) {
  float u = 1.0f + x;
  if (u == 1.0f) return x;
  return o_log(u) * x / (u - 1.0f);
}
static inline float o_expm1(float y) {
  float u = o_exp(y);
  if (u == 1.0f) return y;
  float um = u - 1.0f;
  if (um == -1.0f) return -1.0f;
  return um * y / o_log(u);
}

#endif
