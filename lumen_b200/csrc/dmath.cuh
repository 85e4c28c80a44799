// Float32 elementary functions and the counter-based RNG on the device.
//
// Every function spells out its operations (explicit fmaf; the engine is compiled with -fmad=false) so that it
// evaluates to the same bits as the CPU checker. Methods (each from its mathematics):
//  - exp: Cody-Waite reduction by a two-part ln 2, degree-7 Taylor polynomial on |r| <= ln2 / 2.
//  - log: x = 2^e m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s), s = (m - 1) / (m + 1), odd series to s^11.
//  - sin / cos: reduction by a three-part pi/2 (or exact quarter turns of 2 pi u), Taylor on |r| <= pi/4.
//  - acos: asin x = x + x^3 P(x^2) on |x| <= 1/2 (P a float64 least-squares fit on Chebyshev nodes), half-angle
//    identities beyond.
//  - erfinv: M. Giles, "Approximating the erfinv function" (GPU Computing Gems Jade, 2011), single precision.
//  - threefry2x32-20 (Salmon et al., SC'11) with JAX's fold_in / partitionable bits composition, the reference's
//    random numbers (src/lumen/_core/rng.py:71-97).
#pragma once
#include <stdint.h>

#define L_DEV __device__ __forceinline__
// one copy shared by every call site: the threefry block (called for every draw) and the torus's root finders (their
// 40-step bisections, in the extended geometry only). Every other device function is inlined: measured on B200, the
// inlined step is 11 % faster on the tank's plain forward and 26 % faster on its wavefront with tangents than with the
// surface kernel, the media and the navigator's helpers called (their frames and argument copies were local memory)
#define L_CALL static __device__ __noinline__

namespace lb {

L_DEV float bits_f(uint32_t u) { return __uint_as_float(u); }
L_DEV uint32_t f_bits(float f) { return __float_as_uint(f); }
L_DEV float pow2i(int k) { return bits_f((uint32_t)(k + 127) << 23); }

L_DEV float l_exp(float x) {
  if (!(x == x)) return x;
  if (x > 88.72283935546875f) return __int_as_float(0x7f800000);
  if (x < -103.972084045410f) return 0.0f;
  const float L2E = 1.44269502162933349609f;
  const float LN2_HI = 0.693145751953125f;
  const float LN2_LO = 1.42860682030941723212e-6f;
  float kf = floorf(__fadd_rn(__fmul_rn(x, L2E), 0.5f));
  float r = __fsub_rn(x, __fmul_rn(kf, LN2_HI));
  r = __fsub_rn(r, __fmul_rn(kf, LN2_LO));
  float p = 1.98412698412698412526e-4f;
  p = fmaf(p, r, 1.38888888888888894189e-3f);
  p = fmaf(p, r, 8.33333333333333321769e-3f);
  p = fmaf(p, r, 4.16666666666666643537e-2f);
  p = fmaf(p, r, 1.66666666666666657415e-1f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  int k = (int)kf;
  if (k > 127) return (p * pow2i(127)) * pow2i(k - 127);
  if (k < -126) return (p * pow2i(k + 100)) * pow2i(-100);
  return p * pow2i(k);
}

L_DEV float l_log(float x) {
  if (!(x > 0.0f)) return x == 0.0f ? __int_as_float(0xff800000) : __int_as_float(0x7fc00000);
  if (x == __int_as_float(0x7f800000)) return x;
  int adj = 0;
  if (x < 1.17549435e-38f) { x = x * 8388608.0f; adj = -23; }
  uint32_t u = f_bits(x);
  int e = (int)((u >> 23) & 0xff) - 127 + adj;
  float m = bits_f((u & 0x7fffffu) | 0x3f800000u);
  if (m > 1.41421353816986083984f) { m = m * 0.5f; e = e + 1; }
  float f = m - 1.0f;
  float s = f / (2.0f + f);
  float z = s * s;
  float p = 0.181818181818181823f;
  p = fmaf(p, z, 0.222222222222222210f);
  p = fmaf(p, z, 0.285714285714285698f);
  p = fmaf(p, z, 0.400000000000000022f);
  p = fmaf(p, z, 0.666666666666666630f);
  float lm = fmaf(s * z, p, 2.0f * s);
  const float LN2_HI = 0.693145751953125f;
  const float LN2_LO = 1.42860682030941723212e-6f;
  float ef = (float)e;
  return fmaf(ef, LN2_HI, fmaf(ef, LN2_LO, lm));
}

L_DEV void l_sincos_poly(float r, float* s, float* c) {
  float z = r * r;
  float ps = 2.75573192239858906526e-6f;
  ps = fmaf(ps, z, -1.98412698412698412526e-4f);
  ps = fmaf(ps, z, 8.33333333333333321769e-3f);
  ps = fmaf(ps, z, -1.66666666666666657415e-1f);
  *s = fmaf(r * z, ps, r);
  float pc = -2.75573192239858906526e-7f;
  pc = fmaf(pc, z, 2.48015873015873015658e-5f);
  pc = fmaf(pc, z, -1.38888888888888894189e-3f);
  pc = fmaf(pc, z, 4.16666666666666643537e-2f);
  pc = fmaf(pc, z, -0.5f);
  *c = fmaf(z, pc, 1.0f);
}

L_DEV void l_quadrant(int q, float s, float c, float* so, float* co) {
  switch (q & 3) {
    case 0: *so = s; *co = c; break;
    case 1: *so = c; *co = -s; break;
    case 2: *so = -s; *co = -c; break;
    default: *so = -c; *co = s; break;
  }
}

L_DEV void l_sincos2pi(float u, float* s, float* c) {
  float v = 4.0f * u;
  float q = floorf(v + 0.5f);
  float f = v - q;
  float r = f * 1.57079632679489661923f;
  float ss, cc;
  l_sincos_poly(r, &ss, &cc);
  l_quadrant((int)q, ss, cc, s, c);
}

L_DEV void l_sincos(float x, float* s, float* c) {
  const float TWO_OVER_PI = 0.636619772367581343076f;
  const float P1 = 1.5703125f;
  const float P2 = 4.83512878417968750000e-4f;
  const float P3 = 3.13855707717955556e-7f;
  float q = floorf(x * TWO_OVER_PI + 0.5f);
  float r = x - q * P1;
  r = r - q * P2;
  r = r - q * P3;
  float ss, cc;
  l_sincos_poly(r, &ss, &cc);
  l_quadrant((int)q, ss, cc, s, c);
}

L_DEV float l_asin_small(float x) {
  float z = x * x;
  float p = 3.38055603e-02f;
  p = fmaf(p, z, 1.70779899e-02f);
  p = fmaf(p, z, 3.11161242e-02f);
  p = fmaf(p, z, 4.45980355e-02f);
  p = fmaf(p, z, 7.50009865e-02f);
  p = fmaf(p, z, 1.66666657e-01f);
  return fmaf(x * z, p, x);
}

L_DEV float l_acos(float x) {
  const float PI = 3.14159265358979323846f;
  const float PIO2 = 1.57079632679489661923f;
  if (x > 1.0f) x = 1.0f;
  if (x < -1.0f) x = -1.0f;
  if (x <= 0.5f && x >= -0.5f) return PIO2 - l_asin_small(x);
  if (x > 0.5f) return 2.0f * l_asin_small(sqrtf((1.0f - x) * 0.5f));
  return PI - 2.0f * l_asin_small(sqrtf((1.0f + x) * 0.5f));
}

L_DEV float l_asin(float v) {
  const float PIO2 = 1.57079632679489661923f;
  float a = fabsf(v);
  if (a > 1.0f) a = 1.0f;
  float r = a <= 0.5f ? l_asin_small(a) : PIO2 - 2.0f * l_asin_small(sqrtf((1.0f - a) * 0.5f));
  return v < 0.0f ? -r : r;
}

// atan2 from asin / acos on the octant where each is well conditioned
L_DEV float l_atan2(float y, float x) {
  const float PI = 3.14159265358979323846f;
  float r = sqrtf(x * x + y * y);
  if (r == 0.0f) return 0.0f;
  float a;
  if (fabsf(y) <= fabsf(x)) {
    a = l_asin(fabsf(y) / r);
    if (x < 0.0f) a = PI - a;
  } else {
    a = l_acos(x / r);
  }
  return y < 0.0f ? -a : a;
}

// the cube root: exp(log|x| / 3) and one Newton step on y^3 = |x|
L_DEV float l_cbrt(float x) {
  if (x == 0.0f) return 0.0f;
  float a = x < 0.0f ? -x : x;
  float y = l_exp(l_log(a) * 0.333333343267440796f);
  y = y - (y * y * y - a) / (3.0f * y * y);
  return x < 0.0f ? -y : y;
}

// the cube root in float64 (the float64 navigator's torus): the float32 cube root of |x| (brought into float32's
// normal range by powers of 2^96) as the start, then two Newton steps on y^3 = |x|, each squaring the relative error
// (about 2^-22 -> 2^-44 -> below an ulp)
L_DEV double l_cbrt64(double x) {
  if (x == 0.0) return 0.0;
  double a = x < 0.0 ? -x : x;
  int k = 0;
  for (int i = 0; i < 12 && a < 1e-30; ++i) { a = a * 79228162514264337593543950336.0; --k; }
  for (int i = 0; i < 12 && a > 1e30; ++i) { a = a * 1.26217744835361888865876570445245796747713029617443680e-29; ++k; }
  double y = (double)l_cbrt((float)a);
  y = y - (y * y * y - a) / (3.0 * y * y);
  y = y - (y * y * y - a) / (3.0 * y * y);
  for (; k < 0; ++k) y = y * 2.3283064365386962890625e-10;
  for (; k > 0; --k) y = y * 4294967296.0;
  return x < 0.0 ? -y : y;
}

L_DEV float l_erfinv(float x) {
  float w = -l_log((1.0f - x) * (1.0f + x));
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

// ------------------------------------------------------------------------------------------------- threefry
struct Key { uint32_t k0, k1; };

L_DEV uint32_t rotl(uint32_t x, int r) { return __funnelshift_l(x, x, r); }

L_CALL void threefry(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1, uint32_t* y0, uint32_t* y1) {
  const uint32_t k2 = k0 ^ k1 ^ 0x1BD11BDAu;
  x0 += k0; x1 += k1;
#define TF_R(r) x0 += x1; x1 = rotl(x1, r); x1 ^= x0;
  TF_R(13) TF_R(15) TF_R(26) TF_R(6) x0 += k1; x1 += k2 + 1u;
  TF_R(17) TF_R(29) TF_R(16) TF_R(24) x0 += k2; x1 += k0 + 2u;
  TF_R(13) TF_R(15) TF_R(26) TF_R(6) x0 += k0; x1 += k1 + 3u;
  TF_R(17) TF_R(29) TF_R(16) TF_R(24) x0 += k1; x1 += k2 + 4u;
  TF_R(13) TF_R(15) TF_R(26) TF_R(6) x0 += k2; x1 += k0 + 5u;
#undef TF_R
  *y0 = x0; *y1 = x1;
}

L_DEV Key fold_in(Key k, uint32_t d) {
  Key r;
  threefry(k.k0, k.k1, 0u, d, &r.k0, &r.k1);
  return r;
}

L_DEV float uniform(Key k, uint32_t i) {
  uint32_t y0, y1;
  threefry(k.k0, k.k1, 0u, i, &y0, &y1);
  uint32_t b = (y0 ^ y1) >> 9;
  return ((float)b + 0.5f) * 1.1920928955078125e-7f;
}

}  // namespace lb
