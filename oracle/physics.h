/*
 * ORACLE (test infrastructure): the reference's optics at a crossing and in the bulk, restated in float32.
 *
 * Tables: src/lumen/media/laws.py:86 (_table: linear in photon energy, held beyond), :97 group_index.
 * Media: src/lumen/media/bulk.py:76 rate, :88 evaluate; src/lumen/transport/medium.py:27 medium_at.
 * Surfaces: src/lumen/surfaces/types.py:211 chained_cuts, :243-275 the three Fresnel branches, :277 Geant4's chain,
 * :352 kernel; fresnel.py:25-75 amplitudes; polar.py (fill, project, mirror, s_axis, components, recombine,
 * fractions); outcomes.py:36 refract; lobes.py:55 Lambert; media/phase.py:43-57 Rayleigh (polarised dipole draw).
 * Frames: src/lumen/_core/frames.py (Duff et al. 2017 basis).
 */
#ifndef LUMEN_ORACLE_PHYSICS_H
#define LUMEN_ORACLE_PHYSICS_H

#include "geom.h"

#define O_HC 1239.84198433200208f   /* h c in eV nm (src/lumen/units.py:20) */
#define O_C_VACUUM 0.299792458f     /* m / ns */
#define O_FLOOR32 1e-30f
#define O_FLT_TINY 1.17549435e-38f
#define O_FRESNEL_SMALL 1e-12f
#define O_NORMAL_INCIDENCE 1.42108547152020037e-14f /* eps32^2 */
#define O_ZERO_STATE 0.5f
#define O_TWO_PI 6.28318530717958647692f
#define O_PI 3.14159265358979323846f
#define O_LOG_2_3 (-0.405465108108164381978f) /* log(2/3) */

enum { O_STRAIGHT = 0, O_REFRACT, O_SPECULAR, O_BACKSCATTER, O_GLOSSY, O_DIFFUSE, O_N_OUT };

/* ------------------------------------------------------------------------------------------------- tables */
typedef struct OPools { const float* live; const float* ref; } OPools;

/* value of table t at photon energy E (jnp.interp: held at the ends) and its slope in E there */
static inline float o_tab(const LumenSceneDesc* D, const float* pool, int t, float E, float* slope) {
  int off = D->tab[2 * t], k = D->tab[2 * t + 1];
  const float* xe = pool + off;
  const float* fv = pool + off + k;
  if (slope) *slope = 0.0f;
  if (k == 1 || E <= xe[0]) return fv[0];
  if (E >= xe[k - 1]) return fv[k - 1];
  int i = 1;
  while (i < k - 1 && xe[i] <= E) ++i;
  float dx = xe[i] - xe[i - 1];
  float df = fv[i] - fv[i - 1];
  float sl = df / dx;
  if (slope) *slope = sl;
  return fv[i - 1] + (E - xe[i - 1]) / dx * df;
}

/* rate 1 / L of a length (bulk.py:76) */
static inline float o_rate(float L) { return L >= O_FLT_TINY ? 1.0f / L : 1.0f / O_FLT_TINY; }

/* Geant4's GROUPVEL group index c / v_g at photon energy E of an index table (laws.py:156 _group_index_knot,
   :170 geant4_group_index): knot values at the first knot, the segments' midpoints and the last knot, n + dn / d log E
   (not below n), 1 / n_g linear in energy between them and held beyond. A one-knot (constant) table: n. */
static inline float o_g4_group_knot(const float* e, const float* n, int k, int j) {
  int s = j - 1 < 0 ? 0 : (j - 1 > k - 1 ? k - 1 : j - 1);
  float slope = (n[s + 1] - n[s]) / o_log(e[s + 1] / e[s]);
  float base = (j == 0 || j == k) ? n[j] : 0.5f * (n[s] + n[s + 1]);
  float g = base + slope;
  return g > base ? g : base;
}
static inline float o_group_index(const LumenSceneDesc* D, const float* pool, int t, float E) {
  int off = D->tab[2 * t], kk = D->tab[2 * t + 1];
  const float* e = pool + off;
  const float* n = pool + off + kk;
  if (kk == 1) return n[0];
  int k = kk - 1;
  /* eg: e0, the midpoints of segments 0 .. k-2, e_k */
  float eg_[LUMEN_MAX_KNOTS + 1];
  eg_[0] = e[0];
  for (int i = 0; i + 1 < k; ++i) eg_[1 + i] = 0.5f * (e[i] + e[i + 1]);
  eg_[k] = e[k];
  int p = 0;
  while (p < k + 1 && eg_[p] <= E) ++p; /* searchsorted, side right */
  p = p < 1 ? 1 : (p > k ? k : p);
  float x0 = eg_[p - 1], x1 = eg_[p];
  float f0 = 1.0f / o_g4_group_knot(e, n, k, p - 1), f1 = 1.0f / o_g4_group_knot(e, n, k, p);
  float f;
  if (E < x0) f = f0;
  else if (E > x1) f = f1;
  else {
    float dx = x1 - x0;
    f = fabsf(dx) <= 1.4e-45f ? f0 : f0 + (E - x0) / dx * (f1 - f0);
  }
  return 1.0f / f;
}

typedef struct OMed { float n, ng, mu_abs, mu_c, ch[LUMEN_N_CHANNEL]; } OMed;

/* the length table of channel c (Rayleigh, Mie, WLS: bulk.py:21 CHANNEL_ORDER) of a medium record, -1 if absent */
static inline int o_channel_tab(const int32_t* m, int c) {
  return m[c == 0 ? LUMEN_MI_RAY : (c == 1 ? LUMEN_MI_MIE : LUMEN_MI_WLS)];
}

/* (n, n_g, mu_abs, the channels' rates and their sum) of medium mi at lam (medium.py:27, bulk.py:88 evaluate) */
static inline OMed o_medium_at(const LumenSceneDesc* D, const float* pool, float lam, int mi) {
  const int32_t* m = D->med_i + (size_t)mi * LUMEN_MED_I;
  float E = O_HC / lam;
  OMed r = {1.0f, 1.0f, 0.0f, 0.0f, {0.0f, 0.0f, 0.0f}};
  if (m[LUMEN_MI_INDEX] >= 0) {
    r.n = o_tab(D, pool, m[LUMEN_MI_INDEX], E, 0);
    r.ng = o_group_index(D, pool, m[LUMEN_MI_INDEX], E);
  }
  if (m[LUMEN_MI_ABS] >= 0) r.mu_abs = o_rate(o_tab(D, pool, m[LUMEN_MI_ABS], E, 0));
  for (int c = 0; c < LUMEN_N_CHANNEL; ++c) {
    int t = o_channel_tab(m, c);
    if (t >= 0) r.ch[c] = o_rate(o_tab(D, pool, t, E, 0));
  }
  r.mu_c = (r.ch[0] + r.ch[1]) + r.ch[2];
  return r;
}
static inline float o_index_at(const LumenSceneDesc* D, const float* pool, float lam, int mi) {
  const int32_t* m = D->med_i + (size_t)mi * LUMEN_MED_I;
  if (m[LUMEN_MI_INDEX] < 0) return 1.0f;
  return o_tab(D, pool, m[LUMEN_MI_INDEX], O_HC / lam, 0);
}

/* ---------------------------------------------------------------------------------------------- vectors */
static inline void o_unit(float* v) {
  float s = o_dot(v, v);
  if (s > 0.0f) {
    float r = sqrtf(s);
    v[0] = v[0] / r; v[1] = v[1] / r; v[2] = v[2] / r;
  }
}
static inline void o_cross(const float* a, const float* b, float* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
/* frames.py:14 basis (Duff et al.) */
static inline void o_basis(const float* n, float* t1, float* t2) {
  float sign = n[2] >= 0.0f ? 1.0f : -1.0f;
  float a = -1.0f / (sign + n[2]);
  float b = n[0] * n[1] * a;
  t1[0] = 1.0f + sign * (n[0] * n[0]) * a; t1[1] = sign * b; t1[2] = -sign * n[0];
  t2[0] = b; t2[1] = sign + (n[1] * n[1]) * a; t2[2] = -n[1];
}
static inline void o_to_world(const float* l, const float* n, float* w) {
  float t1[3], t2[3];
  o_basis(n, t1, t2);
  for (int a = 0; a < 3; ++a) w[a] = l[0] * t1[a] + l[1] * t2[a] + l[2] * n[a];
}

/* --------------------------------------------------------------------------------------- complex float32 */
typedef struct Oc { float re, im; } Oc;
static inline Oc oc(float r, float i) { Oc z = {r, i}; return z; }
static inline Oc oc_add(Oc a, Oc b) { return oc(a.re + b.re, a.im + b.im); }
static inline Oc oc_sub(Oc a, Oc b) { return oc(a.re - b.re, a.im - b.im); }
static inline Oc oc_mul(Oc a, Oc b) { return oc(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
static inline Oc oc_div(Oc a, Oc b) {
  float den = b.re * b.re + b.im * b.im;
  return oc((a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den);
}
static inline float oc_abs2(Oc a) { return a.re * a.re + a.im * a.im; }
static inline float oc_abs(Oc a) { return sqrtf(oc_abs2(a)); }
/* principal square root */
static inline Oc oc_sqrt(Oc z) {
  float r = oc_abs(z);
  if (r == 0.0f) return oc(0.0f, 0.0f);
  if (z.re >= 0.0f) {
    float t = sqrtf((r + z.re) * 0.5f);
    return oc(t, z.im / (2.0f * t));
  }
  float t = sqrtf((r - z.re) * 0.5f);
  return oc(fabsf(z.im) / (2.0f * t), z.im < 0.0f ? -t : t);
}
/* sqrt with Im >= 0, and 0 near 0 (fresnel.py:14 decaying_sqrt) */
static inline Oc oc_decaying_sqrt(Oc z) {
  if (oc_abs(z) < O_FRESNEL_SMALL) return oc(0.0f, 0.0f);
  Oc q = oc_sqrt(z);
  if (q.im < 0.0f) q = oc(-q.re, -q.im);
  return q;
}

/* (r_s, r_p, t_s, t_p) from n1 into n2 at incidence cos_i (fresnel.py:25 amplitudes) */
static inline void o_amplitudes(float cos_i, float n1, Oc n2, Oc* a) {
  float c = cos_i < 0.0f ? 0.0f : (cos_i > 1.0f ? 1.0f : cos_i);
  Oc c1 = oc(c, 0.0f), n1c = oc(n1, 0.0f);
  Oc n22 = oc_mul(n2, n2);
  Oc q = oc_decaying_sqrt(oc_sub(n22, oc_mul(oc_mul(n1c, n1c), oc(1.0f - c * c, 0.0f))));
  Oc ds = oc_add(oc_mul(n1c, c1), q);
  Oc dp = oc_add(oc_mul(n22, c1), oc_mul(n1c, q));
  int ok_s = oc_abs(ds) > O_FRESNEL_SMALL, ok_p = oc_abs(dp) > O_FRESNEL_SMALL;
  Oc two_n1c = oc_mul(oc(2.0f, 0.0f), oc_mul(n1c, c1));
  a[0] = ok_s ? oc_div(oc_sub(oc_mul(n1c, c1), q), ds) : oc(-1.0f, 0.0f);
  a[1] = ok_p ? oc_div(oc_sub(oc_mul(n22, c1), oc_mul(n1c, q)), dp) : oc(1.0f, 0.0f);
  a[2] = ok_s ? oc_div(two_n1c, ds) : oc(0.0f, 0.0f);
  a[3] = ok_p ? oc_div(oc_mul(two_n1c, n2), dp) : oc(0.0f, 0.0f);
}

/* ------------------------------------------------------------------------------------------- polarisation */
static inline void o_normalise(float* er, float* ei) {
  float s = o_dot(er, er) + o_dot(ei, ei);
  if (s > O_FLOOR32) {
    float r = 1.0f / sqrtf(s);
    for (int a = 0; a < 3; ++a) { er[a] = er[a] * r; ei[a] = ei[a] * r; }
  } else {
    for (int a = 0; a < 3; ++a) { er[a] = 0.0f; ei[a] = 0.0f; }
  }
}
/* an unpolarised state (E = 0) replaced by a random linear one (polar.py:57 fill) */
static inline void o_fill(const float* d, float* er, float* ei, float rand) {
  if (o_dot(er, er) + o_dot(ei, ei) < O_ZERO_STATE) {
    float t1[3], t2[3], s, c;
    o_basis(d, t1, t2);
    o_sincos2pi(rand, &s, &c);
    for (int a = 0; a < 3; ++a) { er[a] = c * t1[a] + s * t2[a]; ei[a] = 0.0f; }
  }
}
static inline void o_project(float* er, float* ei, const float* k) {
  float kr = o_dot(k, er), ki = o_dot(k, ei);
  for (int a = 0; a < 3; ++a) { er[a] = er[a] - kr * k[a]; ei[a] = ei[a] - ki * k[a]; }
  o_normalise(er, ei);
}
static inline void o_mirror(float* er, float* ei, const float* h) {
  float hr = o_dot(er, h), hi = o_dot(ei, h);
  for (int a = 0; a < 3; ++a) { er[a] = -er[a] + 2.0f * hr * h[a]; ei[a] = -ei[a] + 2.0f * hi * h[a]; }
}
/* the s axis unit(wi x n); at normal incidence basis(wi)'s first tangent (polar.py:100 s_axis) */
static inline void o_s_axis(const float* wi, const float* n, float* s) {
  float c[3];
  o_cross(wi, n, c);
  if (o_dot(c, c) > O_NORMAL_INCIDENCE) {
    s[0] = c[0]; s[1] = c[1]; s[2] = c[2];
    o_unit(s);
  } else {
    float t2[3];
    o_basis(wi, s, t2);
  }
}
static inline void o_components(const float* er, const float* ei, const float* wi, const float* s, Oc* es, Oc* ep) {
  float p[3];
  o_cross(wi, s, p);
  *es = oc(o_dot(er, s), o_dot(ei, s));
  *ep = oc(o_dot(er, p), o_dot(ei, p));
}
static inline void o_recombine(Oc es, Oc ep, Oc as, Oc ap, const float* s, const float* k, float* er, float* ei) {
  float p[3];
  o_cross(k, s, p);
  Oc cs = oc_mul(as, es), cp = oc_mul(ap, ep);
  for (int a = 0; a < 3; ++a) {
    er[a] = cs.re * s[a] + cp.re * p[a];
    ei[a] = cs.im * s[a] + cp.im * p[a];
  }
  o_normalise(er, ei);
}

/* --------------------------------------------------------------------------------------- the surface kernel */
typedef struct OEval {
  float probs[O_N_OUT];
  float detect;
  float sigma;
  Oc amps[4];
} OEval;

/* the tangent of one row column per gradient parameter: dcol[p][c] */
static inline float o_clip01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }
static inline float o_dclip01(float x, float dx) { return (x >= 0.0f && x <= 1.0f) ? dx : 0.0f; }

/* Geant4's chained cuts (types.py:211) of (p1..pk) -> k + 1 shares, with their tangents */
static inline void o_chained(int k, const float* p, const float* dp, float* out, float* dout) {
  float s = 0.0f, ds = 0.0f, prev = 0.0f, dprev = 0.0f;
  for (int j = 0; j < k; ++j) {
    s = j == 0 ? p[0] : s + p[j];
    ds = j == 0 ? dp[0] : ds + dp[j];
    float c = o_clip01(s), dc = o_dclip01(s, ds);
    out[j] = c - prev;
    dout[j] = dc - dprev;
    prev = c;
    dprev = dc;
  }
  out[k] = 1.0f - prev;
  dout[k] = -dprev;
}

/* the TypeEval of surface row `row` at a crossing (types.py:352 kernel, surface_event.py:58 type_probs); `grad`:
   the number of gradient parameters, dcolp[p * LUMEN_N_COL + c] the tangent of column c in parameter p, and
   dprobs[p * 6 + o], ddet[p] its outputs' tangents */
static inline void o_type_eval(const LumenSceneDesc* D, const float* pool, int row, float lam, const float* wi,
                               const float* n, float n1, float n2, const float* er, const float* ei, OEval* ev,
                               int grad, const float* dcolp, float* dprobs, float* ddet) {
  for (int o = 0; o < O_N_OUT; ++o) ev->probs[o] = 0.0f;
  ev->detect = 0.0f;
  ev->sigma = 0.1f;
  ev->amps[0] = oc(-1.0f, 0.0f); ev->amps[1] = oc(1.0f, 0.0f); ev->amps[2] = oc(1.0f, 0.0f); ev->amps[3] = oc(1.0f, 0.0f);
  for (int p = 0; p < grad; ++p) { for (int o = 0; o < O_N_OUT; ++o) dprobs[p * O_N_OUT + o] = 0.0f; ddet[p] = 0.0f; }
  if (row < 0) return;
  const int32_t* ri = D->row_i + (size_t)row * LUMEN_ROW_I;
  float E = O_HC / lam;
  float col[LUMEN_N_COL];
  for (int c = 0; c < LUMEN_N_COL; ++c) col[c] = o_tab(D, pool, ri[LUMEN_RI_COL + c], E, 0);
  int model = ri[LUMEN_RI_MODEL], normal = ri[LUMEN_RI_NORMAL];
  float cos_i = -(wi[0] * n[0] + wi[1] * n[1] + wi[2] * n[2]);
  cos_i = cos_i < 0.0f ? 0.0f : (cos_i > 1.0f ? 1.0f : cos_i);
  float Rc, split[5]; /* specular, glossy, backscatter, diffuse, refraction */
  float dRc[LUMEN_MAX_GRAD], dsplit[LUMEN_MAX_GRAD][5];
  if (model == 0) { /* _none: the reflection constants split R */
    float pc[3] = {col[LUMEN_COL_PSPIKE], col[LUMEN_COL_PLOBE], col[LUMEN_COL_PBACK]};
    float zero3[3] = {0.0f, 0.0f, 0.0f}, sh[4], dsh[4];
    o_chained(3, pc, zero3, sh, dsh);
    split[0] = normal ? sh[0] + sh[1] : sh[0];
    split[1] = normal ? 0.0f : sh[1];
    split[2] = sh[2];
    split[3] = sh[3];
    split[4] = 0.0f;
    Rc = col[LUMEN_COL_R];
    for (int p = 0; p < grad; ++p) {
      const float* dc = dcolp + p * LUMEN_N_COL;
      float dpc[3] = {dc[LUMEN_COL_PSPIKE], dc[LUMEN_COL_PLOBE], dc[LUMEN_COL_PBACK]};
      o_chained(3, pc, dpc, sh, dsh);
      dsplit[p][0] = normal ? dsh[0] + dsh[1] : dsh[0];
      dsplit[p][1] = normal ? 0.0f : dsh[1];
      dsplit[p][2] = dsh[2];
      dsplit[p][3] = dsh[3];
      dsplit[p][4] = 0.0f;
      dRc[p] = dc[LUMEN_COL_R];
    }
  } else if (model == 1) { /* _real: the two media's Fresnel interface */
    o_amplitudes(cos_i, n1, oc(n2, 0.0f), ev->amps);
    float F;
    if (er) {
      float s_ax[3];
      o_s_axis(wi, n, s_ax);
      Oc es, ep;
      o_components(er, ei, wi, s_ax, &es, &ep);
      F = oc_abs2(ev->amps[0]) * oc_abs2(es) + oc_abs2(ev->amps[1]) * oc_abs2(ep);
    } else { /* no state: the unpolarised reflectance, fractions (0.5, 0.5) (types.py:257 _real) */
      F = oc_abs2(ev->amps[0]) * 0.5f + oc_abs2(ev->amps[1]) * 0.5f;
    }
    F = o_clip01(F);
    split[0] = F; split[1] = 0.0f; split[2] = 0.0f; split[3] = 0.0f; split[4] = 1.0f - F;
    Rc = col[LUMEN_COL_R];
    for (int p = 0; p < grad; ++p) {
      for (int j = 0; j < 5; ++j) dsplit[p][j] = 0.0f;
      dRc[p] = dcolp[p * LUMEN_N_COL + LUMEN_COL_R];
    }
  } else { /* _complex: a complex index seen from a dielectric */
    o_amplitudes(cos_i, n1, oc(col[LUMEN_COL_NR], col[LUMEN_COL_NK]), ev->amps);
    if (er) {
      float s_ax[3];
      o_s_axis(wi, n, s_ax);
      Oc es, ep;
      o_components(er, ei, wi, s_ax, &es, &ep);
      Rc = o_clip01(oc_abs2(ev->amps[0]) * oc_abs2(es) + oc_abs2(ev->amps[1]) * oc_abs2(ep));
    } else { /* unpolarised (fresnel.py:53 unpolarised_absorbing_reflectance) */
      Rc = o_clip01(0.5f * (oc_abs2(ev->amps[0]) + oc_abs2(ev->amps[1])));
    }
    split[0] = 1.0f; split[1] = 0.0f; split[2] = 0.0f; split[3] = 0.0f; split[4] = 0.0f;
    for (int p = 0; p < grad; ++p) { for (int j = 0; j < 5; ++j) dsplit[p][j] = 0.0f; dRc[p] = 0.0f; }
  }
  /* Geant4's chain (types.py:277) */
  float cut[2] = {Rc, col[LUMEN_COL_T]}, zc[2] = {0.0f, 0.0f}, rta[3], drta[3];
  o_chained(2, cut, zc, rta, drta);
  float r = rta[0], t = rta[1], a = rta[2];
  ev->probs[O_REFRACT] = r * split[4];
  ev->probs[O_SPECULAR] = r * split[0];
  ev->probs[O_GLOSSY] = r * split[1];
  ev->probs[O_BACKSCATTER] = r * split[2];
  ev->probs[O_DIFFUSE] = r * split[3];
  ev->probs[O_STRAIGHT] = t;
  int far_opaque = ri[LUMEN_RI_FAR_OPAQUE];
  if (far_opaque) { ev->probs[O_STRAIGHT] = 0.0f; ev->probs[O_REFRACT] = 0.0f; }
  ev->detect = a * col[LUMEN_COL_EFF];
  ev->sigma = ri[LUMEN_RI_GLISUR] ? 1.0f - col[LUMEN_COL_POLISH] : col[LUMEN_COL_SIGMA];
  for (int p = 0; p < grad; ++p) {
    const float* dc = dcolp + p * LUMEN_N_COL;
    float dcut[2] = {dRc[p], dc[LUMEN_COL_T]};
    o_chained(2, cut, dcut, rta, drta);
    float dr = drta[0], dt = drta[1], da = drta[2];
    float* dp = dprobs + p * O_N_OUT;
    dp[O_REFRACT] = dr * split[4] + r * dsplit[p][4];
    dp[O_SPECULAR] = dr * split[0] + r * dsplit[p][0];
    dp[O_GLOSSY] = dr * split[1] + r * dsplit[p][1];
    dp[O_BACKSCATTER] = dr * split[2] + r * dsplit[p][2];
    dp[O_DIFFUSE] = dr * split[3] + r * dsplit[p][3];
    dp[O_STRAIGHT] = dt;
    if (far_opaque) { dp[O_STRAIGHT] = 0.0f; dp[O_REFRACT] = 0.0f; }
    ddet[p] = da * col[LUMEN_COL_EFF] + a * dc[LUMEN_COL_EFF];
  }
}

/* ------------------------------------------------------------------------------------------------- lobes */
/* Rayleigh: the dipole cosine's inverse CDF (phase.py:50 dipole_cos) and the polarised draw (phase.py:57) */
static inline float o_dipole_cos(float rand) {
  float x = 1.0f - 2.0f * rand;
  x = x < -1.0f ? -1.0f : (x > 1.0f ? 1.0f : x);
  float s, c;
  o_sincos((o_acos(x) - O_TWO_PI) / 3.0f, &s, &c);
  float r = 2.0f * c;
  return r < -1.0f ? -1.0f : (r > 1.0f ? 1.0f : r);
}
static inline void o_rayleigh_sample(const float* er, const float* ei, const float* rand, float* wo) {
  float a2 = o_dot(er, er);
  float norm2 = o_dot(er, er) + o_dot(ei, ei);
  float axis[3];
  const float* ax = (rand[2] * norm2 < a2) ? er : ei;
  axis[0] = ax[0]; axis[1] = ax[1]; axis[2] = ax[2];
  o_unit(axis);
  float c = o_dipole_cos(rand[0]);
  float s2 = 1.0f - c * c;
  float s = s2 > 0.0f ? sqrtf(s2) : 0.0f;
  float sp, cp;
  o_sincos2pi(rand[1], &sp, &cp);
  float l[3] = {s * cp, s * sp, c};
  o_to_world(l, axis, wo);
}
/* Lambert about the facing normal n (lobes.py:55 _cosine) */
static inline void o_lambert(const float* n, float r0, float r1, float* wo) {
  float r = sqrtf(r0);
  float sp, cp;
  o_sincos2pi(r1, &sp, &cp);
  float l[3] = {r * cp, r * sp, sqrtf(1.0f - r0)};
  o_to_world(l, n, wo);
}

/* ------------------------------------------------------------------------- Geant4's unified facet path (GLOSSY) */
#include "rng.h"
#define O_FACET_REDRAWS 4096 /* a facet draw is accepted with probability bounded below: never reached */
#define O_FACET_PATH 256     /* facets per path: the photon leaves with probability bounded below at each */

static inline void o_to_local(const float* v, const float* n, float* l) {
  float t1[3], t2[3];
  o_basis(n, t1, t2);
  l[0] = o_dot(v, t1); l[1] = o_dot(v, t2); l[2] = o_dot(v, n);
}
/* the half-width of the azimuth arc of facets at tilt a that face V (facets.py:311 _front_arc) */
static inline float o_front_arc(const float* V, float a) {
  float sv = sqrtf(V[0] * V[0] + V[1] * V[1]);
  float sa, ca;
  o_sincos(a, &sa, &ca);
  float ratio = V[2] * ca / o_max(sv * sa, O_FLOOR32);
  return o_acos(-o_min(ratio, 1.0f));
}
/* a unified facet normal (local frame) given V . m > 0 (facets.py:318 unified_facet): the tilt by rejection from a
   Rayleigh(sigma) proposal, the azimuth uniform in the front arc */
static inline void o_unified_facet(float sigma, const float* V, OKey key, float* m, int* capped) {
  float fmax = o_min(1.0f, 4.0f * sigma);
  float a = 0.0f, u2 = 0.5f;
  int ok = 0;
  for (uint32_t t = 0; t < O_FACET_REDRAWS && !ok; ++t) {
    OKey kt = o_fold_in(key, t);
    float u0 = o_uniform(kt, 0), u1 = o_uniform(kt, 1);
    float al = sigma * sqrtf(-2.0f * o_log(u0));
    if (al < 1.57079632679489661923f) {
      float sa, ca;
      o_sincos(al, &sa, &ca);
      ok = u1 * al * O_PI < o_min(sa, fmax) * o_front_arc(V, al);
    }
    a = al;
    u2 = o_uniform(kt, 2);
  }
  if (!ok) *capped = 1;
  float psi = (2.0f * u2 - 1.0f) * o_front_arc(V, a);
  float ph = o_atan2(V[1], V[0]) + psi;
  float sa, ca, sp, cp;
  o_sincos(a, &sa, &ca);
  o_sincos(ph, &sp, &cp);
  m[0] = sa * cp; m[1] = sa * sp; m[2] = ca;
}
/* a raw threefry key from the three lobe uniforms (facets.py:303 seed_key) */
static inline OKey o_seed_key(float r0, float r1, float r2) {
  uint32_t k0 = (uint32_t)(r0 * 8388608.0f), k1 = (uint32_t)(r1 * 8388608.0f), k2 = (uint32_t)(r2 * 8388608.0f);
  OKey k = {k0 | (k2 << 23), k1 | ((k2 >> 9) << 23)};
  return k;
}
/* ---- the unified lobe's tables, read as the reference reads them (facets.py:153-207): a C1 cubic Hermite of
   log zeta = log(Z / sigma^2) in y = log sigma, a bicubic Hermite of the facing share F in (x, y); each also returns
   its derivative(s) in the coordinates */
#define O_UNI_Y0 ((float)LUMEN_UNI_Y0)
#define O_UNI_DY ((float)LUMEN_UNI_DY)
#define O_HALF_PI 1.57079632679489661923f
#define O_LOG_TINY (-69.07755278982137f) /* log FLOOR32: a log density off the support (facets.py:61) */
#define O_LOG_2PI 1.83787706640934548356f

/* the cell of coordinate v among n nodes: index, offset t and dt / dv (0 where v is clamped) (facets.py:159 _cell) */
static inline void o_uni_cell(float v, int n, int* i, float* t, float* dt) {
  float top = (float)(n - 1);
  float f = v < 0.0f ? 0.0f : (v > top ? top : v);
  *dt = (v < 0.0f || v > top) ? 0.0f : 1.0f;
  int k = (int)floorf(f);
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  *i = k;
  *t = f - (float)k;
}
/* the cubic Hermite basis (a0, b0, a1, b1) at t and its derivative in t (facets.py:153 _hermite) */
static inline void o_hermite(float t, float* h, float* dh) {
  float t2 = t * t, t3 = t2 * t;
  h[0] = 2.0f * t3 - 3.0f * t2 + 1.0f;
  h[1] = t3 - 2.0f * t2 + t;
  h[2] = -2.0f * t3 + 3.0f * t2;
  h[3] = t3 - t2;
  dh[0] = 6.0f * t2 - 6.0f * t;
  dh[1] = 3.0f * t2 - 4.0f * t + 1.0f;
  dh[2] = -6.0f * t2 + 6.0f * t;
  dh[3] = 3.0f * t2 - 2.0f * t;
}
/* log zeta at y = log sigma and d / dy (facets.py:170 table_lz) */
static inline float o_table_lz(const float* U, float y, float* dy) {
  const float* v = U + 4 * LUMEN_UNI_NX * LUMEN_UNI_NY;
  const float* dv = v + LUMEN_UNI_NY;
  int j;
  float t, dt, h[4], dh[4];
  o_uni_cell((y - O_UNI_Y0) / O_UNI_DY - (float)LUMEN_UNI_J_LO, LUMEN_UNI_NY, &j, &t, &dt);
  o_hermite(t, h, dh);
  float out = h[0] * v[j] + h[2] * v[j + 1] + O_UNI_DY * (h[1] * dv[j] + h[3] * dv[j + 1]);
  float dout = dh[0] * v[j] + dh[2] * v[j + 1] + O_UNI_DY * (dh[1] * dv[j] + dh[3] * dv[j + 1]);
  *dy = dout * dt / O_UNI_DY;
  return out;
}
/* F at (x, y = log sigma) and its derivatives in x and y (facets.py:180 table_front) */
static inline float o_table_front(const float* U, float x, float y, float* dFx, float* dFy) {
  const int NY = LUMEN_UNI_NY, NN = LUMEN_UNI_NX * LUMEN_UNI_NY;
  const float* A[4] = {U, U + NN, U + 2 * NN, U + 3 * NN}; /* F, Fx, Fy, Fxy */
  int i, j;
  float tx, ty, dtx, dty, hx4[4], dhx4[4], hy4[4], dhy4[4];
  o_uni_cell(x * (float)(LUMEN_UNI_NX - 1), LUMEN_UNI_NX, &i, &tx, &dtx);
  o_uni_cell((y - O_UNI_Y0) / O_UNI_DY - (float)LUMEN_UNI_J_LO, NY, &j, &ty, &dty);
  const float hx = 1.0f / (float)(LUMEN_UNI_NX - 1);
  o_hermite(tx, hx4, dhx4);
  o_hermite(ty, hy4, dhy4);
  float out = 0.0f, ox = 0.0f, oy = 0.0f;
  for (int di = 0; di < 2; ++di)
    for (int dj = 0; dj < 2; ++dj) {
      int k = (i + di) * NY + (j + dj);
      float ax = hx4[2 * di], bx = hx4[2 * di + 1], ay = hy4[2 * dj], by = hy4[2 * dj + 1];
      float dax = dhx4[2 * di], dbx = dhx4[2 * di + 1], day = dhy4[2 * dj], dby = dhy4[2 * dj + 1];
      out = out + (ax * ay * A[0][k] + bx * ay * hx * A[1][k] + ax * by * O_UNI_DY * A[2][k] +
                   bx * by * hx * O_UNI_DY * A[3][k]);
      ox = ox + (dax * ay * A[0][k] + dbx * ay * hx * A[1][k] + dax * by * O_UNI_DY * A[2][k] +
                 dbx * by * hx * O_UNI_DY * A[3][k]);
      oy = oy + (ax * day * A[0][k] + bx * day * hx * A[1][k] + ax * dby * O_UNI_DY * A[2][k] +
                 bx * dby * hx * O_UNI_DY * A[3][k]);
    }
  *dFx = ox * dtx * (float)(LUMEN_UNI_NX - 1);
  *dFy = oy * dty / O_UNI_DY;
  return out;
}
/* log p1(w1 | w0) of one unified facet reflection at width sigma, D(h) / (4 F V . h) with h the half vector, and
   (dls, when given) its derivative in sigma; O_LOG_TINY off the support (facets.py:209 _unified_log_density, :248
   _half_vector, :259 unified_facet_logpdf) */
static inline float o_unified_logpdf(const float* U, float sigma, const float* w0, const float* n, const float* w1,
                                     float* dls) {
  float mw[3] = {-w0[0], -w0[1], -w0[2]};
  float V[3], W[3];
  o_to_local(mw, n, V);
  o_to_local(w1, n, W);
  float H[3] = {V[0] + W[0], V[1] + W[1], V[2] + W[2]};
  float vH = o_dot(V, H);
  if (!(H[2] > 0.0f && vH > 0.0f)) {
    if (dls) *dls = 0.0f;
    return O_LOG_TINY;
  }
  float inv = 1.0f / sqrtf(o_dot(H, H));
  float vh = vH * inv;
  float ch = H[2] * inv;
  float s = sqrtf(H[0] * H[0] + H[1] * H[1]) * inv; /* sin(alpha), from the tangential part */
  float alpha = o_atan2(s, ch);
  float l4 = o_log(4.0f * sigma);
  float lf = o_min(0.0f, l4); /* log f_max */
  float ef = o_exp(lf);
  float ls = o_log(s > ef ? s : ef);
  float cos_t = V[2], sin_t = sqrtf(V[0] * V[0] + V[1] * V[1]);
  float y = o_log(sigma);
  float dlz, dFx, dFy;
  float lz = o_table_lz(U, y, &dlz);
  float x = o_atan2(cos_t, sigma * sin_t) / O_HALF_PI;
  float F = o_table_front(U, x, y, &dFx, &dFy);
  float lp = -alpha * alpha / (2.0f * sigma * sigma) + (lf - ls) - O_LOG_2PI - 2.0f * y - lz - o_log(F);
  lp = lp - o_log(4.0f * vh);
  if (dls) {
    float is = 1.0f / sigma;
    float dlf = l4 < 0.0f ? is : (l4 == 0.0f ? 0.5f * is : 0.0f); /* a tie splits the derivative */
    float dsel = s > ef ? dlf : 0.0f;
    float sb = sigma * sin_t;
    float dx = -(cos_t * sin_t) / (cos_t * cos_t + sb * sb) / O_HALF_PI;
    *dls = alpha * alpha / (sigma * sigma * sigma) + dsel - 2.0f * is - dlz * is - (dFx * dx + dFy * is) / F;
  }
  return lp;
}

/* the facet path: a facet for the current direction and the mirror about it, until the direction leaves the surface
   (facets.py:372 _path_of, surface_event.py:106 _facet_path_branch: the Jones vector mirrored about each facet's half
   vector). With the tables U, each facet's log density is summed: at the live width into lp (its derivative in
   sigma into dls, when given) and, where weigh is set, at the drawn (reference) width into lr. */
static inline void o_facet_path(float sigma, const float* wi, const float* n, const float* rand, float* wo, float* er,
                                float* ei, int* capped, const float* U, float sig_live, int weigh, float* lp,
                                float* lr, float* dls) {
  OKey key = o_seed_key(rand[0], rand[1], rand[2]);
  float mwi[3] = {-wi[0], -wi[1], -wi[2]};
  float V[3];
  o_to_local(mwi, n, V);
  float w[3] = {wi[0], wi[1], wi[2]};
  for (uint32_t k = 0; k < O_FACET_PATH; ++k) {
    float m[3];
    o_unified_facet(sigma, V, o_fold_in(key, k), m, capped);
    float vm = o_dot(V, m);
    float L[3] = {2.0f * vm * m[0] - V[0], 2.0f * vm * m[1] - V[1], 2.0f * vm * m[2] - V[2]};
    o_to_world(L, n, wo);
    if (U) {
      float d = 0.0f;
      *lp = *lp + o_unified_logpdf(U, sig_live, w, n, wo, dls ? &d : 0);
      if (dls) *dls = *dls + d;
      if (weigh) *lr = *lr + o_unified_logpdf(U, sigma, w, n, wo, 0);
    }
    float h[3] = {wo[0] - w[0], wo[1] - w[1], wo[2] - w[2]};
    o_unit(h);
    o_mirror(er, ei, h);
    w[0] = wo[0]; w[1] = wo[1]; w[2] = wo[2];
    V[0] = -L[0]; V[1] = -L[1]; V[2] = -L[2];
    if (L[2] >= 0.0f) return;
    if (k + 1 == O_FACET_PATH) *capped = 1;
  }
}

/* ---------------------------------------------------------------------------------------- GLISUR facets */
#define O_SHELL_STREAM 0xFFFFFFFFu     /* the vertex key's fold choosing the facet's cover part (rng.py:31) */
#define O_FRESNEL_STREAM 0xFFFFFFFEu   /* a dielectric facet's reflect-or-refract uniform (rng.py:34) */
#define O_GLISUR_COVER 0.01f           /* the defensive share of the shell (src/lumen/rules/choices.py:113) */
#define O_INDEX_MATCH (128.0f * 1.1920928955078125e-7f) /* indices one at a facet (choices.py:98) */
#define O_PI 3.14159265358979323846f

/* a GLISUR facet normal (local frame): M = e_z + r s, s uniform in the unit ball (on its sphere when the facet's
   one cover draw says so), redrawn until V . M > 0 (facets.py:341 glisur_facet) */
static inline void o_glisur_facet(float r, const float* V, OKey key, float e, float* m, int* capped) {
  int shell = e > 0.0f && o_uniform(o_fold_in(key, O_SHELL_STREAM), 0) < e;
  float M[3] = {0.0f, 0.0f, 1.0f};
  int ok = 0;
  for (uint32_t t = 0; t < O_FACET_REDRAWS && !ok; ++t) {
    OKey kt = o_fold_in(key, t);
    float u0 = o_uniform(kt, 0), u1 = o_uniform(kt, 1), u2 = o_uniform(kt, 2);
    float z = 1.0f - 2.0f * u1;
    float s2 = 1.0f - z * z;
    float sxy = s2 > 0.0f ? sqrtf(s2) : 0.0f;
    float sp, cp;
    o_sincos2pi(u2, &sp, &cp);
    float rad = shell ? 1.0f : o_cbrt(u0);
    float C[3] = {0.0f + r * rad * (sxy * cp), 0.0f + r * rad * (sxy * sp), 1.0f + r * rad * z};
    if (o_dot(V, C) > 0.0f) { M[0] = C[0]; M[1] = C[1]; M[2] = C[2]; ok = 1; }
  }
  if (!ok) *capped = 1;
  float inv = 1.0f / sqrtf(o_dot(M, M));
  m[0] = M[0] * inv; m[1] = M[1] * inv; m[2] = M[2] * inv;
}
/* the log volume of the ball B(n, r) on the photon's side of V . M = 0 (h = V . n; facets.py:226), and d/dr */
static inline float o_glisur_log_volume(float r, float h, float* dr) {
  float d = o_max(r - h, 0.0f);
  float v = 4.0f / 3.0f * O_PI * r * r * r - O_PI * d * d * (2.0f * r + h) / 3.0f;
  if (dr) {
    float dd = r - h > 0.0f ? 1.0f : 0.0f;
    *dr = (4.0f * O_PI * r * r - O_PI * (2.0f * d * dd * (2.0f * r + h) + 2.0f * d * d) / 3.0f) / v;
  }
  return o_log(v);
}
/* the log area of the sphere |M - n| = r on the photon's side (facets.py:268) */
static inline float o_glisur_log_area(float r, float h) {
  return o_log(h >= r ? 4.0f * O_PI * r * r : 2.0f * O_PI * r * (r + o_min(h, r)));
}
/* (log p_m, on the support) of the facet direction M (any length) at width r (facets.py:232), d/dr when asked */
static inline float o_glisur_log_density(float r, const float* V, const float* M, int* ok, float* dr) {
  float m2 = o_dot(M, M);
  float inv = 1.0f / sqrtf(m2);
  float c = M[2] * inv;
  float s2 = (M[0] * M[0] + M[1] * M[1]) / m2;
  float q2 = r * r - s2;
  *ok = q2 > 0.0f && c > 0.0f && o_dot(V, M) > 0.0f;
  float q2s = *ok ? q2 : r * r;
  float cs = *ok ? c : 1.0f;
  float dv;
  float lp = O_LOG_2_3 + 0.5f * o_log(q2s) + o_log(3.0f * cs * cs + q2s) -
             o_glisur_log_volume(r, V[2], dr ? &dv : 0);
  if (dr) *dr = *ok ? r / q2s + 2.0f * r / (3.0f * cs * cs + q2s) - dv : 0.0f;
  return lp;
}
/* log(exp a + exp b), the larger first */
static inline float o_logaddexp(float a, float b) {
  float mx = o_max(a, b), mn = o_min(a, b);
  return mx + o_log1p(o_exp(mn - mx));
}
/* (log of (1 - e) p_m + e p_shell, on the support) for the facet direction M (facets.py:273) */
static inline float o_glisur_log_proposal(float r, const float* V, const float* M, float e, int* ok) {
  float lp = o_glisur_log_density(r, V, M, ok, 0);
  float m2 = o_dot(M, M);
  float c = *ok ? M[2] * (1.0f / sqrtf(m2)) : 1.0f;
  float q2 = *ok ? r * r - (M[0] * M[0] + M[1] * M[1]) / m2 : r * r;
  float ls = o_log(2.0f * r) + o_log(c * c + q2) - 0.5f * o_log(q2) - o_glisur_log_area(r, V[2]);
  return o_logaddexp(o_log1p(-e) + lp, o_log(e) + ls);
}
/* one GLISUR metal facet reflection's log density (exact, cover 0) or its cover's, LOG_TINY off the support
   (facets.py:283, :295), with d/dr of the exact one */
static inline float o_glisur_logpdf(float r, const float* w0, const float* n, const float* w1, float e, float* dr) {
  float mw[3] = {-w0[0], -w0[1], -w0[2]};
  float V[3], W[3];
  o_to_local(mw, n, V);
  o_to_local(w1, n, W);
  float H[3] = {V[0] + W[0], V[1] + W[1], V[2] + W[2]};
  int good = H[2] > 0.0f && o_dot(V, H) > 0.0f;
  if (dr) *dr = 0.0f;
  if (!good) return O_LOG_TINY;
  float vh = o_dot(V, H) * (1.0f / sqrtf(o_dot(H, H)));
  int ok;
  float lq = e > 0.0f ? o_glisur_log_proposal(r, V, H, e, &ok) : o_glisur_log_density(r, V, H, &ok, dr);
  if (!ok) {
    if (dr) *dr = 0.0f;
    return O_LOG_TINY;
  }
  return lq - o_log(4.0f * vh);
}
/* the GLISUR metal facet path drawn from the cover at the reference width r_ref, weighted by its exact path density
   at r_live over the cover's (surface_event.py:106 with the covered lobe); returns the weight, *on the drawn weight
   (the path on the cover's support), *dlr d/dr_live of the log weight */
static inline float o_glisur_metal_path(float r_ref, float r_live, const float* wi, const float* n, const float* rand,
                                        float e, float* wo, float* er, float* ei, int* capped, float* on_,
                                        float* dlr) {
  OKey key = o_seed_key(rand[0], rand[1], rand[2]);
  float mwi[3] = {-wi[0], -wi[1], -wi[2]};
  float V[3];
  o_to_local(mwi, n, V);
  float w[3] = {wi[0], wi[1], wi[2]};
  float lp = 0.0f, lr = 0.0f, dl = 0.0f;
  for (uint32_t k = 0; k < O_FACET_PATH; ++k) {
    float m[3];
    o_glisur_facet(r_ref, V, o_fold_in(key, k), e, m, capped);
    float vm = o_dot(V, m);
    float L[3] = {2.0f * vm * m[0] - V[0], 2.0f * vm * m[1] - V[1], 2.0f * vm * m[2] - V[2]};
    o_to_world(L, n, wo);
    float d;
    lp = lp + o_glisur_logpdf(r_live, w, n, wo, 0.0f, &d);
    dl = dl + d;
    lr = lr + o_glisur_logpdf(r_ref, w, n, wo, e, 0);
    float h[3] = {wo[0] - w[0], wo[1] - w[1], wo[2] - w[2]};
    o_unit(h);
    o_mirror(er, ei, h);
    w[0] = wo[0]; w[1] = wo[1]; w[2] = wo[2];
    V[0] = -L[0]; V[1] = -L[1]; V[2] = -L[2];
    if (L[2] >= 0.0f) break;
    if (k + 1 == O_FACET_PATH) *capped = 1;
  }
  int on = lr > 0.5f * O_LOG_TINY;
  *on_ = on ? 1.0f : 0.0f;
  *dlr = on ? dl : 0.0f;
  return on ? o_exp(lp - lr) : 0.0f;
}

/* ---- the GLISUR dielectric facet path (facets.py:487 _dielectric_path_of, :453 dielectric_event_logpdf) */
static inline int o_matched(float na, float nb) { return fabsf(na - nb) <= O_INDEX_MATCH * o_max(na, nb); }
/* (R, s axis, components, amplitudes) of the state going w0 onto the facet m from n_a into n_b (facets.py:443) */
static inline float o_interface(const float* w0, const float* m, float na, float nb, const float* er, const float* ei,
                                float* s_ax, Oc* es, Oc* ep, Oc* amps) {
  o_s_axis(w0, m, s_ax);
  o_components(er, ei, w0, s_ax, es, ep);
  o_amplitudes(-o_dot(w0, m), na, oc(nb, 0.0f), amps);
  float R = oc_abs2(amps[0]) * oc_abs2(*es) + oc_abs2(amps[1]) * oc_abs2(*ep);
  return R < 0.0f ? 0.0f : (R > 1.0f ? 1.0f : R);
}
/* Snell's refraction of w at facing normal m (outcomes.py:36 refract), the mirror under total reflection */
static inline void o_refract_dir(const float* w, const float* m, float eta, float* wo) {
  float cos_i = -o_dot(w, m);
  float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
  if (sin2_t >= 1.0f) {
    for (int a = 0; a < 3; ++a) wo[a] = w[a] + 2.0f * cos_i * m[a];
    return;
  }
  float ct2 = 1.0f - sin2_t;
  float cos_t = ct2 > 0.0f ? sqrtf(ct2) : 0.0f;
  float k = eta * cos_i - cos_t;
  for (int a = 0; a < 3; ++a) wo[a] = eta * w[a] + k * m[a];
  o_unit(wo);
}
/* one dielectric facet event's log density (exact or the cover's), the Jones vector after it, d/dr (exact) */
static inline float o_dielectric_event_lp(float r, float n1, float n2, const float* n, const float* w0,
                                          const float* w1, int refracted, float side, float e, const float* er,
                                          const float* ei, float* er1, float* ei1, float* dr) {
  float na = side > 0.0f ? n1 : n2, nb = side > 0.0f ? n2 : n1;
  float N[3] = {side * n[0], side * n[1], side * n[2]};
  int matched = o_matched(na, nb);
  float m[3];
  if (refracted && !matched) {
    float sg = nb - na > 0.0f ? 1.0f : (nb - na < 0.0f ? -1.0f : 0.0f);
    float u[3] = {na * w0[0] - nb * w1[0], na * w0[1] - nb * w1[1], na * w0[2] - nb * w1[2]};
    o_unit(u);
    m[0] = u[0] * sg; m[1] = u[1] * sg; m[2] = u[2] * sg;
  } else {
    m[0] = w1[0] - w0[0]; m[1] = w1[1] - w0[1]; m[2] = w1[2] - w0[2];
    o_unit(m);
  }
  float cos1 = -o_dot(w0, m), cos2 = -o_dot(w1, m);
  float mw[3] = {-w0[0], -w0[1], -w0[2]}, Vl[3], Ml[3];
  o_to_local(mw, N, Vl);
  o_to_local(m, N, Ml);
  int ok;
  float lpm = e > 0.0f ? o_glisur_log_proposal(r, Vl, Ml, e, &ok) : o_glisur_log_density(r, Vl, Ml, &ok, dr);
  float s_ax[3];
  Oc es, ep, amps[4];
  float R = o_interface(w0, m, na, nb, er, ei, s_ax, &es, &ep, amps);
  ok = ok && cos1 > 0.0f && (refracted ? cos2 > 0.0f : cos2 < 0.0f);
  float c1 = ok ? cos1 : 1.0f, c2 = ok ? fabsf(cos2) : 1.0f;
  float lrf = lpm + o_log(o_max(R, O_FLOOR32)) - o_log(4.0f * c1);
  float gap = (ok && !matched) ? fabsf(nb * c2 - na * c1) : 1.0f;
  float lt = lpm + o_log(o_max(1.0f - R, O_FLOOR32)) + 2.0f * o_log(nb) + o_log(c2) - 2.0f * o_log(gap);
  float lp = refracted ? (matched ? 0.0f : lt) : lrf;
  ok = ok || (refracted && matched);
  int straight = refracted && matched;
  if (straight) {
    for (int a = 0; a < 3; ++a) { er1[a] = er[a]; ei1[a] = ei[a]; }
  } else {
    o_recombine(es, ep, refracted ? amps[2] : amps[0], refracted ? amps[3] : amps[1], s_ax, w1, er1, ei1);
  }
  if (dr && (!ok || straight)) *dr = 0.0f;
  return ok ? lp : O_LOG_TINY;
}
/* the GLISUR dielectric facet path drawn from the cover at the reference width, at the live indices (n1 the incident
   medium's, n2 the far one's) and state; weighted by its exact path density at r_live over the cover's at r_ref,
   its Jones vector the live one (surface_event.py:137 _dielectric_path_branch); *far: it ends beyond the surface */
static inline float o_glisur_dielectric_path(float r_ref, float r_live, float n1, float n2, const float* wi,
                                             const float* n, const float* rand, float e, float* wo, float* er,
                                             float* ei, int* far_, int* capped, float* on_, float* dlr) {
  OKey key = o_seed_key(rand[0], rand[1], rand[2]);
  float w[3] = {wi[0], wi[1], wi[2]}, wv[3] = {wi[0], wi[1], wi[2]};
  float side = 1.0f;
  float er_d[3] = {er[0], er[1], er[2]}, ei_d[3] = {ei[0], ei[1], ei[2]}; /* the draw's state */
  float er_r[3] = {er[0], er[1], er[2]}, ei_r[3] = {ei[0], ei[1], ei[2]}; /* the cover's density's state */
  float lp = 0.0f, lr = 0.0f, dl = 0.0f;
  int far = 0;
  for (uint32_t k = 0; k < O_FACET_PATH; ++k) {
    float N[3] = {side * n[0], side * n[1], side * n[2]};
    float na = side > 0.0f ? n1 : n2, nb = side > 0.0f ? n2 : n1;
    OKey kk = o_fold_in(key, k);
    float mw[3] = {-w[0], -w[1], -w[2]}, Vl[3];
    o_to_local(mw, N, Vl);
    if (!(Vl[2] > 0.0f)) { Vl[0] = 0.0f; Vl[1] = 0.0f; Vl[2] = 1.0f; }
    float ml[3], m[3];
    o_glisur_facet(r_ref, Vl, kk, e, ml, capped);
    o_to_world(ml, N, m);
    float s_ax[3];
    Oc es, ep, amps[4];
    float R = o_interface(w, m, na, nb, er_d, ei_d, s_ax, &es, &ep, amps);
    int refr = o_uniform(o_fold_in(kk, O_FRESNEL_STREAM), 0) >= R;
    float w1[3];
    if (refr) {
      if (o_matched(na, nb)) { w1[0] = w[0]; w1[1] = w[1]; w1[2] = w[2]; }
      else o_refract_dir(w, m, na / nb, w1);
    } else {
      float wm = o_dot(w, m);
      for (int a = 0; a < 3; ++a) w1[a] = w[a] - 2.0f * wm * m[a];
    }
    float er1[3], ei1[3];
    o_recombine(es, ep, refr ? amps[2] : amps[0], refr ? amps[3] : amps[1], s_ax, w1, er1, ei1);
    float dot = o_dot(w1, N);
    int end = refr ? dot <= 0.0f : dot >= 0.0f;
    /* the visit: the live density with the live state, the cover's with its own state */
    float d, erl[3], eil[3], err2[3], eir2[3];
    lp = lp + o_dielectric_event_lp(r_live, n1, n2, n, wv, w1, refr, side, 0.0f, er, ei, erl, eil, &d);
    dl = dl + d;
    lr = lr + o_dielectric_event_lp(r_ref, n1, n2, n, wv, w1, refr, side, e, er_r, ei_r, err2, eir2, 0);
    for (int a = 0; a < 3; ++a) { er[a] = erl[a]; ei[a] = eil[a]; er_r[a] = err2[a]; ei_r[a] = eir2[a]; }
    for (int a = 0; a < 3; ++a) { er_d[a] = er1[a]; ei_d[a] = ei1[a]; w[a] = w1[a]; wv[a] = w1[a]; wo[a] = w1[a]; }
    if (refr && !end) side = -side;
    far = far ^ refr;
    if (end) break;
    if (k + 1 == O_FACET_PATH) *capped = 1;
  }
  *far_ = far;
  int on = lr > 0.5f * O_LOG_TINY;
  *on_ = on ? 1.0f : 0.0f;
  *dlr = on ? dl : 0.0f;
  return on ? o_exp(lp - lr) : 0.0f;
}

/* the cumulative draw (estimator.py:62 choose): index drawn from q with one uniform, -1 if q is all 0 */
static inline int o_choose(const float* q, int k, float rand) {
  float c[8];
  float s = 0.0f;
  for (int j = 0; j < k; ++j) { s = j == 0 ? q[0] : s + q[j]; c[j] = s; }
  if (!(c[k - 1] > 0.0f)) return -1;
  float thr = rand * c[k - 1];
  for (int j = 0; j < k; ++j) if (c[j] > thr) return j;
  return 0;
}

#endif
