// Optics on the device: tables, media, the surface kernel with its tangents, Fresnel amplitudes, polarisation and
// the bulk / surface lobes. Semantics: src/lumen/media/laws.py:86 (_table), :156-183 (Geant4's GROUPVEL group
// index), bulk.py:76-88, transport/medium.py:27, surfaces/types.py:211-388 (chained cuts, the three Fresnel
// branches, Geant4's chain, kernel), fresnel.py:14-75, polar.py, outcomes.py:36, lobes.py:55, media/phase.py:43-57,
// _core/frames.py. Arithmetic operation for operation the CPU checker's.
#pragma once
#include "dgeom.cuh"

namespace lb {

#define D_HC 1239.84198433200208f
#define D_C_VACUUM 0.299792458f
#define D_FLOOR32 1e-30f
#define D_FLT_TINY 1.17549435e-38f
#define D_FRESNEL_SMALL 1e-12f
#define D_NORMAL_INCIDENCE 1.42108547152020037e-14f
#define D_ZERO_STATE 0.5f

enum { STRAIGHT = 0, REFRACT, SPECULAR, BACKSCATTER, GLOSSY, DIFFUSE, N_OUT };

L_DEV float d_tab(const DScene& S, const float* __restrict__ pool, int t, float E) {
  int off = __ldg(S.tab + 2 * t), k = __ldg(S.tab + 2 * t + 1);
  const float* xe = pool + off;
  const float* fv = pool + off + k;
  if (k == 1 || E <= __ldg(xe)) return __ldg(fv);
  if (E >= __ldg(xe + k - 1)) return __ldg(fv + k - 1);
  int i = 1;
  while (i < k - 1 && __ldg(xe + i) <= E) ++i;
  float x0 = __ldg(xe + i - 1), x1 = __ldg(xe + i);
  float f0 = __ldg(fv + i - 1), f1 = __ldg(fv + i);
  float dx = x1 - x0;
  float df = f1 - f0;
  return f0 + (E - x0) / dx * df;
}

L_DEV float d_rate(float L) { return L >= D_FLT_TINY ? 1.0f / L : 1.0f / D_FLT_TINY; }

L_DEV float d_g4_group_knot(const float* e, const float* n, int k, int j) {
  int s = j - 1 < 0 ? 0 : (j - 1 > k - 1 ? k - 1 : j - 1);
  float slope = (__ldg(n + s + 1) - __ldg(n + s)) / l_log(__ldg(e + s + 1) / __ldg(e + s));
  float base = (j == 0 || j == k) ? __ldg(n + j) : 0.5f * (__ldg(n + s) + __ldg(n + s + 1));
  float g = base + slope;
  return g > base ? g : base;
}
// the midpoint knot eg[j] of Geant4's GROUPVEL table (e0, segment midpoints 0 .. k-2, e_k)
L_DEV float d_eg(const float* e, int k, int j) {
  if (j == 0) return __ldg(e);
  if (j == k) return __ldg(e + k);
  return 0.5f * (__ldg(e + j - 1) + __ldg(e + j));
}
L_DEV float d_group_index(const DScene& S, const float* __restrict__ pool, int t, float E) {
  int off = __ldg(S.tab + 2 * t), kk = __ldg(S.tab + 2 * t + 1);
  const float* e = pool + off;
  const float* n = pool + off + kk;
  if (kk == 1) return __ldg(n);
  int k = kk - 1;
  int p = 0;
  while (p < k + 1 && d_eg(e, k, p) <= E) ++p;
  p = p < 1 ? 1 : (p > k ? k : p);
  float x0 = d_eg(e, k, p - 1), x1 = d_eg(e, k, p);
  float f0 = 1.0f / d_g4_group_knot(e, n, k, p - 1), f1 = 1.0f / d_g4_group_knot(e, n, k, p);
  float f;
  if (E < x0) f = f0;
  else if (E > x1) f = f1;
  else {
    float dx = x1 - x0;
    f = fabsf(dx) <= 1.4e-45f ? f0 : f0 + (E - x0) / dx * (f1 - f0);
  }
  return 1.0f / f;
}

struct Med { float n, ng, mu_abs, mu_c; };  // mu_c: the channels' rates summed

// the length table of channel c (Rayleigh, Mie, WLS: bulk.py:21 CHANNEL_ORDER) of a medium record, -1 if absent
L_DEV int d_channel_tab(const int32_t* m, int c) {
  return __ldg(m + (c == 0 ? LUMEN_MI_RAY : (c == 1 ? LUMEN_MI_MIE : LUMEN_MI_WLS)));
}

// the channels' rates of medium mi at lam (bulk.py:88 evaluate's mu), 0 for an absent channel
L_DEV void d_channel_rates(const DScene& S, const float* __restrict__ pool, float lam, int mi, float* ch) {
  const int32_t* m = S.med_i + (size_t)mi * LUMEN_MED_I;
  float E = D_HC / lam;
#pragma unroll
  for (int c = 0; c < LUMEN_N_CHANNEL; ++c) {
    int t = d_channel_tab(m, c);
    ch[c] = t >= 0 ? d_rate(d_tab(S, pool, t, E)) : 0.0f;
  }
}

// (n, n_g, mu_abs, the channels' rates summed) of medium mi at lam (medium.py:27, bulk.py:88 evaluate); a bulk event
// reads the channels' own rates again (d_channel_rates: the same values)
L_DEV Med d_medium_at(const DScene& S, const float* __restrict__ pool, float lam, int mi) {
  const int32_t* m = S.med_i + (size_t)mi * LUMEN_MED_I;
  float E = D_HC / lam;
  Med r = {1.0f, 1.0f, 0.0f, 0.0f};
  int ti = __ldg(m + LUMEN_MI_INDEX), ta = __ldg(m + LUMEN_MI_ABS);
  if (ti >= 0) {
    r.n = d_tab(S, pool, ti, E);
    r.ng = d_group_index(S, pool, ti, E);
  }
  if (ta >= 0) r.mu_abs = d_rate(d_tab(S, pool, ta, E));
  float ch[LUMEN_N_CHANNEL];
  d_channel_rates(S, pool, lam, mi, ch);
  r.mu_c = (ch[0] + ch[1]) + ch[2];
  return r;
}
L_DEV float d_index_at(const DScene& S, const float* __restrict__ pool, float lam, int mi) {
  int ti = __ldg(S.med_i + (size_t)mi * LUMEN_MED_I + LUMEN_MI_INDEX);
  if (ti < 0) return 1.0f;
  return d_tab(S, pool, ti, D_HC / lam);
}

// ------------------------------------------------------------------------------------------------ vectors
L_DEV void d_unit(float* v) {
  float s = d_dot(v, v);
  if (s > 0.0f) {
    float r = sqrtf(s);
    v[0] = v[0] / r; v[1] = v[1] / r; v[2] = v[2] / r;
  }
}
L_DEV void d_cross(const float* a, const float* b, float* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
L_DEV void d_basis(const float* n, float* t1, float* t2) {
  float sign = n[2] >= 0.0f ? 1.0f : -1.0f;
  float a = -1.0f / (sign + n[2]);
  float b = n[0] * n[1] * a;
  t1[0] = 1.0f + sign * (n[0] * n[0]) * a; t1[1] = sign * b; t1[2] = -sign * n[0];
  t2[0] = b; t2[1] = sign + (n[1] * n[1]) * a; t2[2] = -n[1];
}
L_DEV void d_to_world(const float* l, const float* n, float* w) {
  float t1[3], t2[3];
  d_basis(n, t1, t2);
#pragma unroll
  for (int a = 0; a < 3; ++a) w[a] = l[0] * t1[a] + l[1] * t2[a] + l[2] * n[a];
}

// ------------------------------------------------------------------------------------------- complex float
struct Cf { float re, im; };
L_DEV Cf cf(float r, float i) { Cf z; z.re = r; z.im = i; return z; }
L_DEV Cf c_add(Cf a, Cf b) { return cf(a.re + b.re, a.im + b.im); }
L_DEV Cf c_sub(Cf a, Cf b) { return cf(a.re - b.re, a.im - b.im); }
L_DEV Cf c_mul(Cf a, Cf b) { return cf(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re); }
L_DEV Cf c_div(Cf a, Cf b) {
  float den = b.re * b.re + b.im * b.im;
  return cf((a.re * b.re + a.im * b.im) / den, (a.im * b.re - a.re * b.im) / den);
}
L_DEV float c_abs2(Cf a) { return a.re * a.re + a.im * a.im; }
L_DEV float c_abs(Cf a) { return sqrtf(c_abs2(a)); }
L_DEV Cf c_sqrt(Cf z) {
  float r = c_abs(z);
  if (r == 0.0f) return cf(0.0f, 0.0f);
  if (z.re >= 0.0f) {
    float t = sqrtf((r + z.re) * 0.5f);
    return cf(t, z.im / (2.0f * t));
  }
  float t = sqrtf((r - z.re) * 0.5f);
  return cf(fabsf(z.im) / (2.0f * t), z.im < 0.0f ? -t : t);
}
L_DEV Cf c_decaying_sqrt(Cf z) {
  if (c_abs(z) < D_FRESNEL_SMALL) return cf(0.0f, 0.0f);
  Cf q = c_sqrt(z);
  if (q.im < 0.0f) q = cf(-q.re, -q.im);
  return q;
}

L_DEV void d_amplitudes(float cos_i, float n1, Cf n2, Cf* a) {
  float c = cos_i < 0.0f ? 0.0f : (cos_i > 1.0f ? 1.0f : cos_i);
  Cf c1 = cf(c, 0.0f), n1c = cf(n1, 0.0f);
  Cf n22 = c_mul(n2, n2);
  Cf q = c_decaying_sqrt(c_sub(n22, c_mul(c_mul(n1c, n1c), cf(1.0f - c * c, 0.0f))));
  Cf ds = c_add(c_mul(n1c, c1), q);
  Cf dp = c_add(c_mul(n22, c1), c_mul(n1c, q));
  int ok_s = c_abs(ds) > D_FRESNEL_SMALL, ok_p = c_abs(dp) > D_FRESNEL_SMALL;
  Cf two_n1c = c_mul(cf(2.0f, 0.0f), c_mul(n1c, c1));
  a[0] = ok_s ? c_div(c_sub(c_mul(n1c, c1), q), ds) : cf(-1.0f, 0.0f);
  a[1] = ok_p ? c_div(c_sub(c_mul(n22, c1), c_mul(n1c, q)), dp) : cf(1.0f, 0.0f);
  a[2] = ok_s ? c_div(two_n1c, ds) : cf(0.0f, 0.0f);
  a[3] = ok_p ? c_div(c_mul(two_n1c, n2), dp) : cf(0.0f, 0.0f);
}

// ------------------------------------------------------------------------------------------- polarisation
L_DEV void d_normalise(float* er, float* ei) {
  float s = d_dot(er, er) + d_dot(ei, ei);
  if (s > D_FLOOR32) {
    float r = 1.0f / sqrtf(s);
#pragma unroll
    for (int a = 0; a < 3; ++a) { er[a] = er[a] * r; ei[a] = ei[a] * r; }
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) { er[a] = 0.0f; ei[a] = 0.0f; }
  }
}
L_DEV void d_fill(const float* d, float* er, float* ei, float rand) {
  float t1[3], t2[3], s, c;
  d_basis(d, t1, t2);
  l_sincos2pi(rand, &s, &c);
#pragma unroll
  for (int a = 0; a < 3; ++a) { er[a] = c * t1[a] + s * t2[a]; ei[a] = 0.0f; }
}
L_DEV void d_project(float* er, float* ei, const float* k) {
  float kr = d_dot(k, er), ki = d_dot(k, ei);
#pragma unroll
  for (int a = 0; a < 3; ++a) { er[a] = er[a] - kr * k[a]; ei[a] = ei[a] - ki * k[a]; }
  d_normalise(er, ei);
}
L_DEV void d_mirror(float* er, float* ei, const float* h) {
  float hr = d_dot(er, h), hi = d_dot(ei, h);
#pragma unroll
  for (int a = 0; a < 3; ++a) { er[a] = -er[a] + 2.0f * hr * h[a]; ei[a] = -ei[a] + 2.0f * hi * h[a]; }
}
L_DEV void d_s_axis(const float* wi, const float* n, float* s) {
  float c[3];
  d_cross(wi, n, c);
  if (d_dot(c, c) > D_NORMAL_INCIDENCE) {
    s[0] = c[0]; s[1] = c[1]; s[2] = c[2];
    d_unit(s);
  } else {
    float t2[3];
    d_basis(wi, s, t2);
  }
}
L_DEV void d_components(const float* er, const float* ei, const float* wi, const float* s, Cf* es, Cf* ep) {
  float p[3];
  d_cross(wi, s, p);
  *es = cf(d_dot(er, s), d_dot(ei, s));
  *ep = cf(d_dot(er, p), d_dot(ei, p));
}
L_DEV void d_recombine(Cf es, Cf ep, Cf as, Cf ap, const float* s, const float* k, float* er, float* ei) {
  float p[3];
  d_cross(k, s, p);
  Cf cs = c_mul(as, es), cp = c_mul(ap, ep);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    er[a] = cs.re * s[a] + cp.re * p[a];
    ei[a] = cs.im * s[a] + cp.im * p[a];
  }
  d_normalise(er, ei);
}

// -------------------------------------------------------------------------------------- the surface kernel
struct Eval {
  float probs[N_OUT];
  float detect;
  float sigma;
  Cf amps[4];
};

L_DEV float d_clip01(float x) { return x < 0.0f ? 0.0f : (x > 1.0f ? 1.0f : x); }
L_DEV float d_dclip01(float x, float dx) { return (x >= 0.0f && x <= 1.0f) ? dx : 0.0f; }

template <int K>
L_DEV void d_chained(const float* p, const float* dp, float* out, float* dout) {
  float s = 0.0f, ds = 0.0f, prev = 0.0f, dprev = 0.0f;
#pragma unroll
  for (int j = 0; j < K; ++j) {
    s = j == 0 ? p[0] : s + p[j];
    ds = j == 0 ? dp[0] : ds + dp[j];
    float c = d_clip01(s), dc = d_dclip01(s, ds);
    out[j] = c - prev;
    dout[j] = dc - dprev;
    prev = c;
    dprev = dc;
  }
  out[K] = 1.0f - prev;
  dout[K] = -dprev;
}

// the TypeEval of a surface row (types.py:352 kernel); with G > 0 gradient parameters, gt[p] the table each moves,
// the tangents dprobs[p][o], ddet[p] (a column's value moves with its table)
// UNPOL: no polarisation state (er, ei unread): the unpolarised reflectances (a photon born in a sensor, step.py:589)
template <int G, bool UNPOL = false>
L_DEV void d_type_eval(const DScene& S, const float* __restrict__ pool, int row, float lam, const float* wi,
                       const float* n, float n1, float n2, const float* er, const float* ei, Eval& ev, int P,
                       const int* gt, float (*dprobs)[N_OUT], float* ddet) {
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) ev.probs[o] = 0.0f;
  ev.detect = 0.0f;
  ev.sigma = 0.1f;
  ev.amps[0] = cf(-1.0f, 0.0f); ev.amps[1] = cf(1.0f, 0.0f); ev.amps[2] = cf(1.0f, 0.0f); ev.amps[3] = cf(1.0f, 0.0f);
  if (G > 0)
    for (int p = 0; p < P; ++p) {
#pragma unroll
      for (int o = 0; o < N_OUT; ++o) dprobs[p][o] = 0.0f;
      ddet[p] = 0.0f;
    }
  if (row < 0) return;
  const int32_t* ri = S.row_i + (size_t)row * LUMEN_ROW_I;
  float E = D_HC / lam;
  float col[LUMEN_N_COL];
  int ct[LUMEN_N_COL];
#pragma unroll
  for (int c = 0; c < LUMEN_N_COL; ++c) {
    ct[c] = __ldg(ri + LUMEN_RI_COL + c);
    col[c] = d_tab(S, pool, ct[c], E);
  }
  int model = __ldg(ri + LUMEN_RI_MODEL), normal = __ldg(ri + LUMEN_RI_NORMAL);
  float cos_i = -(wi[0] * n[0] + wi[1] * n[1] + wi[2] * n[2]);
  cos_i = cos_i < 0.0f ? 0.0f : (cos_i > 1.0f ? 1.0f : cos_i);
  float Rc, split[5];
  if (model == 0) {
    float pc[3] = {col[LUMEN_COL_PSPIKE], col[LUMEN_COL_PLOBE], col[LUMEN_COL_PBACK]};
    float zero3[3] = {0.0f, 0.0f, 0.0f}, sh[4], dsh[4];
    d_chained<3>(pc, zero3, sh, dsh);
    split[0] = normal ? sh[0] + sh[1] : sh[0];
    split[1] = normal ? 0.0f : sh[1];
    split[2] = sh[2];
    split[3] = sh[3];
    split[4] = 0.0f;
    Rc = col[LUMEN_COL_R];
  } else if (model == 1) {
    d_amplitudes(cos_i, n1, cf(n2, 0.0f), ev.amps);
    float F;
    if constexpr (!UNPOL) {
      float s_ax[3];
      d_s_axis(wi, n, s_ax);
      Cf es, ep;
      d_components(er, ei, wi, s_ax, &es, &ep);
      F = c_abs2(ev.amps[0]) * c_abs2(es) + c_abs2(ev.amps[1]) * c_abs2(ep);
    } else {  // no state: the unpolarised reflectance, fractions (0.5, 0.5) (types.py:257 _real)
      F = c_abs2(ev.amps[0]) * 0.5f + c_abs2(ev.amps[1]) * 0.5f;
    }
    F = d_clip01(F);
    split[0] = F; split[1] = 0.0f; split[2] = 0.0f; split[3] = 0.0f; split[4] = 1.0f - F;
    Rc = col[LUMEN_COL_R];
  } else {
    d_amplitudes(cos_i, n1, cf(col[LUMEN_COL_NR], col[LUMEN_COL_NK]), ev.amps);
    if constexpr (!UNPOL) {
      float s_ax[3];
      d_s_axis(wi, n, s_ax);
      Cf es, ep;
      d_components(er, ei, wi, s_ax, &es, &ep);
      Rc = d_clip01(c_abs2(ev.amps[0]) * c_abs2(es) + c_abs2(ev.amps[1]) * c_abs2(ep));
    } else {  // unpolarised (fresnel.py:53 unpolarised_absorbing_reflectance)
      Rc = d_clip01(0.5f * (c_abs2(ev.amps[0]) + c_abs2(ev.amps[1])));
    }
    split[0] = 1.0f; split[1] = 0.0f; split[2] = 0.0f; split[3] = 0.0f; split[4] = 0.0f;
  }
  float cut[2] = {Rc, col[LUMEN_COL_T]}, zc[2] = {0.0f, 0.0f}, rta[3], drta[3];
  d_chained<2>(cut, zc, rta, drta);
  float r = rta[0], t = rta[1], a = rta[2];
  ev.probs[REFRACT] = r * split[4];
  ev.probs[SPECULAR] = r * split[0];
  ev.probs[GLOSSY] = r * split[1];
  ev.probs[BACKSCATTER] = r * split[2];
  ev.probs[DIFFUSE] = r * split[3];
  ev.probs[STRAIGHT] = t;
  int far_opaque = __ldg(ri + LUMEN_RI_FAR_OPAQUE);
  if (far_opaque) { ev.probs[STRAIGHT] = 0.0f; ev.probs[REFRACT] = 0.0f; }
  ev.detect = a * col[LUMEN_COL_EFF];
  ev.sigma = __ldg(ri + LUMEN_RI_GLISUR) ? 1.0f - col[LUMEN_COL_POLISH] : col[LUMEN_COL_SIGMA];
  if (G > 0) {
    for (int p = 0; p < P; ++p) {
      float dc[LUMEN_N_COL];
#pragma unroll
      for (int c = 0; c < LUMEN_N_COL; ++c) dc[c] = ct[c] == gt[p] ? 1.0f : 0.0f;
      float dsplit[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f}, dRc = 0.0f;
      if (model == 0) {
        float pc[3] = {col[LUMEN_COL_PSPIKE], col[LUMEN_COL_PLOBE], col[LUMEN_COL_PBACK]};
        float dpc[3] = {dc[LUMEN_COL_PSPIKE], dc[LUMEN_COL_PLOBE], dc[LUMEN_COL_PBACK]}, sh[4], dsh[4];
        d_chained<3>(pc, dpc, sh, dsh);
        dsplit[0] = normal ? dsh[0] + dsh[1] : dsh[0];
        dsplit[1] = normal ? 0.0f : dsh[1];
        dsplit[2] = dsh[2];
        dsplit[3] = dsh[3];
        dRc = dc[LUMEN_COL_R];
      } else if (model == 1) {
        dRc = dc[LUMEN_COL_R];
      }
      float dcut[2] = {dRc, dc[LUMEN_COL_T]};
      d_chained<2>(cut, dcut, rta, drta);
      float dr = drta[0], dt = drta[1], da = drta[2];
      float* dp = dprobs[p];
      dp[REFRACT] = dr * split[4] + r * dsplit[4];
      dp[SPECULAR] = dr * split[0] + r * dsplit[0];
      dp[GLOSSY] = dr * split[1] + r * dsplit[1];
      dp[BACKSCATTER] = dr * split[2] + r * dsplit[2];
      dp[DIFFUSE] = dr * split[3] + r * dsplit[3];
      dp[STRAIGHT] = dt;
      if (far_opaque) { dp[STRAIGHT] = 0.0f; dp[REFRACT] = 0.0f; }
      ddet[p] = da * col[LUMEN_COL_EFF] + a * dc[LUMEN_COL_EFF];
    }
  }
}

// ------------------------------------------------------------------------------------------------- lobes
L_DEV float d_dipole_cos(float rand) {
  float x = 1.0f - 2.0f * rand;
  x = x < -1.0f ? -1.0f : (x > 1.0f ? 1.0f : x);
  float s, c;
  l_sincos((l_acos(x) - 6.28318530717958647692f) / 3.0f, &s, &c);
  float r = 2.0f * c;
  return r < -1.0f ? -1.0f : (r > 1.0f ? 1.0f : r);
}
L_DEV void d_rayleigh_sample(const float* er, const float* ei, float r0, float r1, float r2, float* wo) {
  float a2 = d_dot(er, er);
  float norm2 = d_dot(er, er) + d_dot(ei, ei);
  float axis[3];
  int use_r = r2 * norm2 < a2;
#pragma unroll
  for (int a = 0; a < 3; ++a) axis[a] = use_r ? er[a] : ei[a];
  d_unit(axis);
  float c = d_dipole_cos(r0);
  float s2 = 1.0f - c * c;
  float s = s2 > 0.0f ? sqrtf(s2) : 0.0f;
  float sp, cp;
  l_sincos2pi(r1, &sp, &cp);
  float l[3] = {s * cp, s * sp, c};
  d_to_world(l, axis, wo);
}
L_DEV void d_lambert(const float* n, float r0, float r1, float* wo) {
  float r = sqrtf(r0);
  float sp, cp;
  l_sincos2pi(r1, &sp, &cp);
  float l[3] = {r * cp, r * sp, sqrtf(1.0f - r0)};
  d_to_world(l, n, wo);
}
// ---------------------------------------------------------------- Geant4's unified facet path (GLOSSY), facets.py
#define D_FACET_REDRAWS 4096  // a facet draw is accepted with a probability bounded below: never reached
#define D_FACET_PATH 256      // facets per path: the photon leaves with a probability bounded below at each

L_DEV void d_to_local(const float* v, const float* n, float* l) {
  float t1[3], t2[3];
  d_basis(n, t1, t2);
  l[0] = d_dot(v, t1); l[1] = d_dot(v, t2); l[2] = d_dot(v, n);
}
L_DEV float d_front_arc(const float* V, float a) {
  float sv = sqrtf(V[0] * V[0] + V[1] * V[1]);
  float sa, ca;
  l_sincos(a, &sa, &ca);
  float ratio = V[2] * ca / d_max(sv * sa, D_FLOOR32);
  return l_acos(-d_min(ratio, 1.0f));
}
L_DEV void d_unified_facet(float sigma, const float* V, Key key, float* m, int* capped) {
  float fmax = d_min(1.0f, 4.0f * sigma);
  float a = 0.0f, u2 = 0.5f;
  int ok = 0;
  for (uint32_t t = 0; t < D_FACET_REDRAWS && !ok; ++t) {
    Key kt = fold_in(key, t);
    float u0 = uniform(kt, 0), u1 = uniform(kt, 1);
    float al = sigma * sqrtf(-2.0f * l_log(u0));
    if (al < 1.57079632679489661923f) {
      float sa, ca;
      l_sincos(al, &sa, &ca);
      ok = u1 * al * 3.14159265358979323846f < d_min(sa, fmax) * d_front_arc(V, al);
    }
    a = al;
    u2 = uniform(kt, 2);
  }
  if (!ok) *capped = 1;
  float psi = (2.0f * u2 - 1.0f) * d_front_arc(V, a);
  float ph = l_atan2(V[1], V[0]) + psi;
  float sa, ca, sp, cp;
  l_sincos(a, &sa, &ca);
  l_sincos(ph, &sp, &cp);
  m[0] = sa * cp; m[1] = sa * sp; m[2] = ca;
}
L_DEV Key d_seed_key(float r0, float r1, float r2) {
  uint32_t k0 = (uint32_t)(r0 * 8388608.0f), k1 = (uint32_t)(r1 * 8388608.0f), k2 = (uint32_t)(r2 * 8388608.0f);
  Key k;
  k.k0 = k0 | (k2 << 23);
  k.k1 = k1 | ((k2 >> 9) << 23);
  return k;
}
// ---- the unified lobe's tables (facets.py:153-207): C1 cubic Hermite of log zeta in y = log sigma, bicubic Hermite
// of the facing share F in (x, y), each with its derivative(s) in the coordinates
#define D_UNI_Y0 ((float)LUMEN_UNI_Y0)
#define D_UNI_DY ((float)LUMEN_UNI_DY)
#define D_HALF_PI 1.57079632679489661923f
#define D_LOG_TINY (-69.07755278982137f)  // log FLOOR32: a log density off the support (facets.py:61)
#define D_LOG_2PI 1.83787706640934548356f

L_DEV void d_uni_cell(float v, int n, int* i, float* t, float* dt) {
  float top = (float)(n - 1);
  float f = v < 0.0f ? 0.0f : (v > top ? top : v);
  *dt = (v < 0.0f || v > top) ? 0.0f : 1.0f;
  int k = (int)floorf(f);
  k = k < 0 ? 0 : (k > n - 2 ? n - 2 : k);
  *i = k;
  *t = f - (float)k;
}
L_DEV void d_hermite(float t, float* h, float* dh) {
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
L_DEV float d_table_lz(const float* __restrict__ U, float y, float* dy) {
  const float* v = U + 4 * LUMEN_UNI_NX * LUMEN_UNI_NY;
  const float* dv = v + LUMEN_UNI_NY;
  int j;
  float t, dt, h[4], dh[4];
  d_uni_cell((y - D_UNI_Y0) / D_UNI_DY - (float)LUMEN_UNI_J_LO, LUMEN_UNI_NY, &j, &t, &dt);
  d_hermite(t, h, dh);
  float v0 = __ldg(v + j), v1 = __ldg(v + j + 1), d0 = __ldg(dv + j), d1 = __ldg(dv + j + 1);
  float out = h[0] * v0 + h[2] * v1 + D_UNI_DY * (h[1] * d0 + h[3] * d1);
  float dout = dh[0] * v0 + dh[2] * v1 + D_UNI_DY * (dh[1] * d0 + dh[3] * d1);
  *dy = dout * dt / D_UNI_DY;
  return out;
}
L_DEV float d_table_front(const float* __restrict__ U, float x, float y, float* dFx, float* dFy) {
  const int NY = LUMEN_UNI_NY, NN = LUMEN_UNI_NX * LUMEN_UNI_NY;
  int i, j;
  float tx, ty, dtx, dty, hx4[4], dhx4[4], hy4[4], dhy4[4];
  d_uni_cell(x * (float)(LUMEN_UNI_NX - 1), LUMEN_UNI_NX, &i, &tx, &dtx);
  d_uni_cell((y - D_UNI_Y0) / D_UNI_DY - (float)LUMEN_UNI_J_LO, NY, &j, &ty, &dty);
  const float hx = 1.0f / (float)(LUMEN_UNI_NX - 1);
  d_hermite(tx, hx4, dhx4);
  d_hermite(ty, hy4, dhy4);
  float out = 0.0f, ox = 0.0f, oy = 0.0f;
#pragma unroll
  for (int di = 0; di < 2; ++di)
#pragma unroll
    for (int dj = 0; dj < 2; ++dj) {
      int k = (i + di) * NY + (j + dj);
      float a0 = __ldg(U + k), a1 = __ldg(U + NN + k), a2 = __ldg(U + 2 * NN + k), a3 = __ldg(U + 3 * NN + k);
      float ax = hx4[2 * di], bx = hx4[2 * di + 1], ay = hy4[2 * dj], by = hy4[2 * dj + 1];
      float dax = dhx4[2 * di], dbx = dhx4[2 * di + 1], day = dhy4[2 * dj], dby = dhy4[2 * dj + 1];
      out = out + (ax * ay * a0 + bx * ay * hx * a1 + ax * by * D_UNI_DY * a2 + bx * by * hx * D_UNI_DY * a3);
      ox = ox + (dax * ay * a0 + dbx * ay * hx * a1 + dax * by * D_UNI_DY * a2 + dbx * by * hx * D_UNI_DY * a3);
      oy = oy + (ax * day * a0 + bx * day * hx * a1 + ax * dby * D_UNI_DY * a2 + bx * dby * hx * D_UNI_DY * a3);
    }
  *dFx = ox * dtx * (float)(LUMEN_UNI_NX - 1);
  *dFy = oy * dty / D_UNI_DY;
  return out;
}
// log p1(w1 | w0) of one unified facet reflection at width sigma and (want_d) its derivative in sigma
// (facets.py:209 _unified_log_density, :248 _half_vector, :259 unified_facet_logpdf)
L_DEV float d_unified_logpdf(const float* __restrict__ U, float sigma, const float* w0, const float* n,
                              const float* w1, int want_d, float* dls) {
  float mw[3] = {-w0[0], -w0[1], -w0[2]};
  float V[3], W[3];
  d_to_local(mw, n, V);
  d_to_local(w1, n, W);
  float H[3] = {V[0] + W[0], V[1] + W[1], V[2] + W[2]};
  float vH = d_dot(V, H);
  *dls = 0.0f;
  if (!(H[2] > 0.0f && vH > 0.0f)) return D_LOG_TINY;
  float inv = 1.0f / sqrtf(d_dot(H, H));
  float vh = vH * inv;
  float ch = H[2] * inv;
  float s = sqrtf(H[0] * H[0] + H[1] * H[1]) * inv;
  float alpha = l_atan2(s, ch);
  float l4 = l_log(4.0f * sigma);
  float lf = d_min(0.0f, l4);
  float ef = l_exp(lf);
  float ls = l_log(s > ef ? s : ef);
  float cos_t = V[2], sin_t = sqrtf(V[0] * V[0] + V[1] * V[1]);
  float y = l_log(sigma);
  float dlz, dFx, dFy;
  float lz = d_table_lz(U, y, &dlz);
  float x = l_atan2(cos_t, sigma * sin_t) / D_HALF_PI;
  float F = d_table_front(U, x, y, &dFx, &dFy);
  float lp = -alpha * alpha / (2.0f * sigma * sigma) + (lf - ls) - D_LOG_2PI - 2.0f * y - lz - l_log(F);
  lp = lp - l_log(4.0f * vh);
  if (want_d) {
    float is = 1.0f / sigma;
    float dlf = l4 < 0.0f ? is : (l4 == 0.0f ? 0.5f * is : 0.0f);
    float dsel = s > ef ? dlf : 0.0f;
    float sb = sigma * sin_t;
    float dx = -(cos_t * sin_t) / (cos_t * cos_t + sb * sb) / D_HALF_PI;
    *dls = alpha * alpha / (sigma * sigma * sigma) + dsel - 2.0f * is - dlz * is - (dFx * dx + dFy * is) / F;
  }
  return lp;
}

// the facet path (facets.py:372 _path_of; the Jones vector mirrored about each facet's half vector,
// surface_event.py:106 _facet_path_branch). With the tables U each facet's log density is summed: at the live width
// into lp (with its derivative in sigma into dls where want_d), and where weigh is set at the drawn width into lr.
L_DEV void d_facet_path(float sigma, const float* wi, const float* n, float r0, float r1, float r2, float* wo,
                         float* er, float* ei, int* capped, const float* __restrict__ U, float sig_live, int weigh,
                         int want_d, float* lp, float* lr, float* dls) {
  Key key = d_seed_key(r0, r1, r2);
  float mwi[3] = {-wi[0], -wi[1], -wi[2]};
  float V[3];
  d_to_local(mwi, n, V);
  float w[3] = {wi[0], wi[1], wi[2]};
  for (uint32_t k = 0; k < D_FACET_PATH; ++k) {
    float m[3];
    d_unified_facet(sigma, V, fold_in(key, k), m, capped);
    float vm = d_dot(V, m);
    float L[3] = {2.0f * vm * m[0] - V[0], 2.0f * vm * m[1] - V[1], 2.0f * vm * m[2] - V[2]};
    d_to_world(L, n, wo);
    if (U) {
      float d;
      *lp = *lp + d_unified_logpdf(U, sig_live, w, n, wo, want_d, &d);
      if (want_d) *dls = *dls + d;
      if (weigh) *lr = *lr + d_unified_logpdf(U, sigma, w, n, wo, 0, &d);
    }
    float h[3] = {wo[0] - w[0], wo[1] - w[1], wo[2] - w[2]};
    d_unit(h);
    d_mirror(er, ei, h);
    w[0] = wo[0]; w[1] = wo[1]; w[2] = wo[2];
    V[0] = -L[0]; V[1] = -L[1]; V[2] = -L[2];
    if (L[2] >= 0.0f) return;
    if (k + 1 == D_FACET_PATH) *capped = 1;
  }
}

// -------------------------------------------------------------------------------------------- GLISUR facets
#define D_SHELL_STREAM 0xFFFFFFFFu    // the facet key's fold choosing the cover part (rng.py:31)
#define D_FRESNEL_STREAM 0xFFFFFFFEu  // a dielectric facet's reflect-or-refract uniform (rng.py:34)
#define D_GLISUR_COVER 0.01f          // the defensive share of the shell (src/lumen/rules/choices.py:113)
#define D_INDEX_MATCH (128.0f * 1.1920928955078125e-7f)  // indices one at a facet (choices.py:98)
#define D_PI 3.14159265358979323846f
#define D_LOG_2_3 (-0.405465108108164381978f)

L_DEV float l_log1p(float x) {
  float u = 1.0f + x;
  if (u == 1.0f) return x;
  return l_log(u) * x / (u - 1.0f);
}
L_DEV float l_expm1(float y) {
  float u = l_exp(y);
  if (u == 1.0f) return y;
  float um = u - 1.0f;
  if (um == -1.0f) return -1.0f;
  return um * y / l_log(u);
}

// a GLISUR facet normal (local frame): M = e_z + r s, s uniform in the unit ball (on its sphere when the facet's
// cover draw says so), redrawn until V . M > 0 (facets.py:341 glisur_facet)
L_DEV void d_glisur_facet(float r, const float* V, Key key, float e, float* m, int* capped) {
  int shell = e > 0.0f && uniform(fold_in(key, D_SHELL_STREAM), 0) < e;
  float M[3] = {0.0f, 0.0f, 1.0f};
  int ok = 0;
  for (uint32_t t = 0; t < D_FACET_REDRAWS && !ok; ++t) {
    Key kt = fold_in(key, t);
    float u0 = uniform(kt, 0), u1 = uniform(kt, 1), u2 = uniform(kt, 2);
    float z = 1.0f - 2.0f * u1;
    float s2 = 1.0f - z * z;
    float sxy = s2 > 0.0f ? sqrtf(s2) : 0.0f;
    float sp, cp;
    l_sincos2pi(u2, &sp, &cp);
    float rad = shell ? 1.0f : l_cbrt(u0);
    float C[3] = {0.0f + r * rad * (sxy * cp), 0.0f + r * rad * (sxy * sp), 1.0f + r * rad * z};
    if (d_dot(V, C) > 0.0f) { M[0] = C[0]; M[1] = C[1]; M[2] = C[2]; ok = 1; }
  }
  if (!ok) *capped = 1;
  float inv = 1.0f / sqrtf(d_dot(M, M));
  m[0] = M[0] * inv; m[1] = M[1] * inv; m[2] = M[2] * inv;
}
L_DEV float d_glisur_log_volume(float r, float h, float* dr) {
  float d = d_max(r - h, 0.0f);
  float v = 4.0f / 3.0f * D_PI * r * r * r - D_PI * d * d * (2.0f * r + h) / 3.0f;
  if (dr) {
    float dd = r - h > 0.0f ? 1.0f : 0.0f;
    *dr = (4.0f * D_PI * r * r - D_PI * (2.0f * d * dd * (2.0f * r + h) + 2.0f * d * d) / 3.0f) / v;
  }
  return l_log(v);
}
L_DEV float d_glisur_log_area(float r, float h) {
  return l_log(h >= r ? 4.0f * D_PI * r * r : 2.0f * D_PI * r * (r + d_min(h, r)));
}
L_DEV float d_glisur_log_density(float r, const float* V, const float* M, int* ok, float* dr) {
  float m2 = d_dot(M, M);
  float inv = 1.0f / sqrtf(m2);
  float c = M[2] * inv;
  float s2 = (M[0] * M[0] + M[1] * M[1]) / m2;
  float q2 = r * r - s2;
  *ok = q2 > 0.0f && c > 0.0f && d_dot(V, M) > 0.0f;
  float q2s = *ok ? q2 : r * r;
  float cs = *ok ? c : 1.0f;
  float dv;
  float lp = D_LOG_2_3 + 0.5f * l_log(q2s) + l_log(3.0f * cs * cs + q2s) - d_glisur_log_volume(r, V[2], dr ? &dv : nullptr);
  if (dr) *dr = *ok ? r / q2s + 2.0f * r / (3.0f * cs * cs + q2s) - dv : 0.0f;
  return lp;
}
L_DEV float d_logaddexp(float a, float b) {
  float mx = d_max(a, b), mn = d_min(a, b);
  return mx + l_log1p(l_exp(mn - mx));
}
L_DEV float d_glisur_log_proposal(float r, const float* V, const float* M, float e, int* ok) {
  float lp = d_glisur_log_density(r, V, M, ok, nullptr);
  float m2 = d_dot(M, M);
  float c = *ok ? M[2] * (1.0f / sqrtf(m2)) : 1.0f;
  float q2 = *ok ? r * r - (M[0] * M[0] + M[1] * M[1]) / m2 : r * r;
  float ls = l_log(2.0f * r) + l_log(c * c + q2) - 0.5f * l_log(q2) - d_glisur_log_area(r, V[2]);
  return d_logaddexp(l_log1p(-e) + lp, l_log(e) + ls);
}
L_DEV float d_glisur_logpdf(float r, const float* w0, const float* n, const float* w1, float e, float* dr) {
  float mw[3] = {-w0[0], -w0[1], -w0[2]};
  float V[3], W[3];
  d_to_local(mw, n, V);
  d_to_local(w1, n, W);
  float H[3] = {V[0] + W[0], V[1] + W[1], V[2] + W[2]};
  int good = H[2] > 0.0f && d_dot(V, H) > 0.0f;
  if (dr) *dr = 0.0f;
  if (!good) return D_LOG_TINY;
  float vh = d_dot(V, H) * (1.0f / sqrtf(d_dot(H, H)));
  int ok;
  float lq = e > 0.0f ? d_glisur_log_proposal(r, V, H, e, &ok) : d_glisur_log_density(r, V, H, &ok, dr);
  if (!ok) {
    if (dr) *dr = 0.0f;
    return D_LOG_TINY;
  }
  return lq - l_log(4.0f * vh);
}
// the GLISUR metal facet path drawn from the cover at r_ref, weighted by its exact path density at r_live over the
// cover's (surface_event.py:106 with the covered lobe); *on the drawn weight, *dlr d/dr_live of the log weight
L_DEV float d_glisur_metal_path(float r_ref, float r_live, const float* wi, const float* n, float r0, float r1,
                                 float r2, float e, float* wo, float* er, float* ei, int* capped, float* on_,
                                 float* dlr) {
  Key key = d_seed_key(r0, r1, r2);
  float mwi[3] = {-wi[0], -wi[1], -wi[2]};
  float V[3];
  d_to_local(mwi, n, V);
  float w[3] = {wi[0], wi[1], wi[2]};
  float lp = 0.0f, lr = 0.0f, dl = 0.0f;
  for (uint32_t k = 0; k < D_FACET_PATH; ++k) {
    float m[3];
    d_glisur_facet(r_ref, V, fold_in(key, k), e, m, capped);
    float vm = d_dot(V, m);
    float L[3] = {2.0f * vm * m[0] - V[0], 2.0f * vm * m[1] - V[1], 2.0f * vm * m[2] - V[2]};
    d_to_world(L, n, wo);
    float d;
    lp = lp + d_glisur_logpdf(r_live, w, n, wo, 0.0f, &d);
    dl = dl + d;
    lr = lr + d_glisur_logpdf(r_ref, w, n, wo, e, nullptr);
    float h[3] = {wo[0] - w[0], wo[1] - w[1], wo[2] - w[2]};
    d_unit(h);
    d_mirror(er, ei, h);
    w[0] = wo[0]; w[1] = wo[1]; w[2] = wo[2];
    V[0] = -L[0]; V[1] = -L[1]; V[2] = -L[2];
    if (L[2] >= 0.0f) break;
    if (k + 1 == D_FACET_PATH) *capped = 1;
  }
  int on = lr > 0.5f * D_LOG_TINY;
  *on_ = on ? 1.0f : 0.0f;
  *dlr = on ? dl : 0.0f;
  return on ? l_exp(lp - lr) : 0.0f;
}

// ---- the GLISUR dielectric facet path (facets.py:487 _dielectric_path_of, :453 dielectric_event_logpdf)
L_DEV int d_matched(float na, float nb) { return fabsf(na - nb) <= D_INDEX_MATCH * d_max(na, nb); }
L_DEV float d_interface(const float* w0, const float* m, float na, float nb, const float* er, const float* ei,
                        float* s_ax, Cf* es, Cf* ep, Cf* amps) {
  d_s_axis(w0, m, s_ax);
  d_components(er, ei, w0, s_ax, es, ep);
  d_amplitudes(-d_dot(w0, m), na, cf(nb, 0.0f), amps);
  float R = c_abs2(amps[0]) * c_abs2(*es) + c_abs2(amps[1]) * c_abs2(*ep);
  return R < 0.0f ? 0.0f : (R > 1.0f ? 1.0f : R);
}
L_DEV void d_refract_dir(const float* w, const float* m, float eta, float* wo) {
  float cos_i = -d_dot(w, m);
  float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
  if (sin2_t >= 1.0f) {
    for (int a = 0; a < 3; ++a) wo[a] = w[a] + 2.0f * cos_i * m[a];
    return;
  }
  float ct2 = 1.0f - sin2_t;
  float cos_t = ct2 > 0.0f ? sqrtf(ct2) : 0.0f;
  float k = eta * cos_i - cos_t;
  for (int a = 0; a < 3; ++a) wo[a] = eta * w[a] + k * m[a];
  d_unit(wo);
}
L_DEV float d_dielectric_event_lp(float r, float n1, float n2, const float* n, const float* w0, const float* w1,
                                   int refracted, float side, float e, const float* er, const float* ei, float* er1,
                                   float* ei1, float* dr) {
  float na = side > 0.0f ? n1 : n2, nb = side > 0.0f ? n2 : n1;
  float N[3] = {side * n[0], side * n[1], side * n[2]};
  int matched = d_matched(na, nb);
  float m[3];
  if (refracted && !matched) {
    float sg = nb - na > 0.0f ? 1.0f : (nb - na < 0.0f ? -1.0f : 0.0f);
    float u[3] = {na * w0[0] - nb * w1[0], na * w0[1] - nb * w1[1], na * w0[2] - nb * w1[2]};
    d_unit(u);
    m[0] = u[0] * sg; m[1] = u[1] * sg; m[2] = u[2] * sg;
  } else {
    m[0] = w1[0] - w0[0]; m[1] = w1[1] - w0[1]; m[2] = w1[2] - w0[2];
    d_unit(m);
  }
  float cos1 = -d_dot(w0, m), cos2 = -d_dot(w1, m);
  float mw[3] = {-w0[0], -w0[1], -w0[2]}, Vl[3], Ml[3];
  d_to_local(mw, N, Vl);
  d_to_local(m, N, Ml);
  int ok;
  float lpm = e > 0.0f ? d_glisur_log_proposal(r, Vl, Ml, e, &ok) : d_glisur_log_density(r, Vl, Ml, &ok, dr);
  float s_ax[3];
  Cf es, ep, amps[4];
  float R = d_interface(w0, m, na, nb, er, ei, s_ax, &es, &ep, amps);
  ok = ok && cos1 > 0.0f && (refracted ? cos2 > 0.0f : cos2 < 0.0f);
  float c1 = ok ? cos1 : 1.0f, c2 = ok ? fabsf(cos2) : 1.0f;
  float lrf = lpm + l_log(d_max(R, D_FLOOR32)) - l_log(4.0f * c1);
  float gap = (ok && !matched) ? fabsf(nb * c2 - na * c1) : 1.0f;
  float lt = lpm + l_log(d_max(1.0f - R, D_FLOOR32)) + 2.0f * l_log(nb) + l_log(c2) - 2.0f * l_log(gap);
  float lp = refracted ? (matched ? 0.0f : lt) : lrf;
  ok = ok || (refracted && matched);
  int straight = refracted && matched;
  if (straight) {
    for (int a = 0; a < 3; ++a) { er1[a] = er[a]; ei1[a] = ei[a]; }
  } else {
    d_recombine(es, ep, refracted ? amps[2] : amps[0], refracted ? amps[3] : amps[1], s_ax, w1, er1, ei1);
  }
  if (dr && (!ok || straight)) *dr = 0.0f;
  return ok ? lp : D_LOG_TINY;
}
// the GLISUR dielectric facet path drawn from the cover at r_ref, at the live indices (n1 incident, n2 far) and state;
// weighted by its exact path density at r_live over the cover's at r_ref, its Jones vector the live one
// (surface_event.py:137 _dielectric_path_branch); *far: it ends beyond the surface
L_DEV float d_glisur_dielectric_path(float r_ref, float r_live, float n1, float n2, const float* wi, const float* n,
                                      float r0, float r1, float r2, float e, float* wo, float* er, float* ei,
                                      int* far_, int* capped, float* on_, float* dlr) {
  Key key = d_seed_key(r0, r1, r2);
  float w[3] = {wi[0], wi[1], wi[2]}, wv[3] = {wi[0], wi[1], wi[2]};
  float side = 1.0f;
  float er_d[3] = {er[0], er[1], er[2]}, ei_d[3] = {ei[0], ei[1], ei[2]};
  float er_r[3] = {er[0], er[1], er[2]}, ei_r[3] = {ei[0], ei[1], ei[2]};
  float lp = 0.0f, lr = 0.0f, dl = 0.0f;
  int far = 0;
  for (uint32_t k = 0; k < D_FACET_PATH; ++k) {
    float N[3] = {side * n[0], side * n[1], side * n[2]};
    float na = side > 0.0f ? n1 : n2, nb = side > 0.0f ? n2 : n1;
    Key kk = fold_in(key, k);
    float mw[3] = {-w[0], -w[1], -w[2]}, Vl[3];
    d_to_local(mw, N, Vl);
    if (!(Vl[2] > 0.0f)) { Vl[0] = 0.0f; Vl[1] = 0.0f; Vl[2] = 1.0f; }
    float ml[3], m[3];
    d_glisur_facet(r_ref, Vl, kk, e, ml, capped);
    d_to_world(ml, N, m);
    float s_ax[3];
    Cf es, ep, amps[4];
    float R = d_interface(w, m, na, nb, er_d, ei_d, s_ax, &es, &ep, amps);
    int refr = uniform(fold_in(kk, D_FRESNEL_STREAM), 0) >= R;
    float w1[3];
    if (refr) {
      if (d_matched(na, nb)) { w1[0] = w[0]; w1[1] = w[1]; w1[2] = w[2]; }
      else d_refract_dir(w, m, na / nb, w1);
    } else {
      float wm = d_dot(w, m);
      for (int a = 0; a < 3; ++a) w1[a] = w[a] - 2.0f * wm * m[a];
    }
    float er1[3], ei1[3];
    d_recombine(es, ep, refr ? amps[2] : amps[0], refr ? amps[3] : amps[1], s_ax, w1, er1, ei1);
    float dot = d_dot(w1, N);
    int end = refr ? dot <= 0.0f : dot >= 0.0f;
    float d, erl[3], eil[3], err2[3], eir2[3];
    lp = lp + d_dielectric_event_lp(r_live, n1, n2, n, wv, w1, refr, side, 0.0f, er, ei, erl, eil, &d);
    dl = dl + d;
    lr = lr + d_dielectric_event_lp(r_ref, n1, n2, n, wv, w1, refr, side, e, er_r, ei_r, err2, eir2, nullptr);
    for (int a = 0; a < 3; ++a) { er[a] = erl[a]; ei[a] = eil[a]; er_r[a] = err2[a]; ei_r[a] = eir2[a]; }
    for (int a = 0; a < 3; ++a) { er_d[a] = er1[a]; ei_d[a] = ei1[a]; w[a] = w1[a]; wv[a] = w1[a]; wo[a] = w1[a]; }
    if (refr && !end) side = -side;
    far = far ^ refr;
    if (end) break;
    if (k + 1 == D_FACET_PATH) *capped = 1;
  }
  *far_ = far;
  int on = lr > 0.5f * D_LOG_TINY;
  *on_ = on ? 1.0f : 0.0f;
  *dlr = on ? dl : 0.0f;
  return on ? l_exp(lp - lr) : 0.0f;
}

L_DEV int d_choose6(const float* q, float rand) {
  float c[N_OUT];
  float s = 0.0f;
#pragma unroll
  for (int j = 0; j < N_OUT; ++j) { s = j == 0 ? q[0] : s + q[j]; c[j] = s; }
  if (!(c[N_OUT - 1] > 0.0f)) return -1;
  float thr = rand * c[N_OUT - 1];
#pragma unroll
  for (int j = 0; j < N_OUT; ++j)
    if (c[j] > thr) return j;
  return 0;
}

}  // namespace lb
