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
L_CALL float d_group_index(const DScene& S, const float* __restrict__ pool, int t, float E) {
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

struct Med { float n, ng, mu_abs, mu_c; };

L_CALL Med d_medium_at(const DScene& S, const float* __restrict__ pool, float lam, int mi) {
  const int32_t* m = S.med_i + (size_t)mi * LUMEN_MED_I;
  float E = D_HC / lam;
  Med r = {1.0f, 1.0f, 0.0f, 0.0f};
  int ti = __ldg(m + LUMEN_MI_INDEX), ta = __ldg(m + LUMEN_MI_ABS), tr = __ldg(m + LUMEN_MI_RAY);
  if (ti >= 0) {
    r.n = d_tab(S, pool, ti, E);
    r.ng = d_group_index(S, pool, ti, E);
  }
  if (ta >= 0) r.mu_abs = d_rate(d_tab(S, pool, ta, E));
  if (tr >= 0) r.mu_c = d_rate(d_tab(S, pool, tr, E));
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

L_CALL void d_amplitudes(float cos_i, float n1, Cf n2, Cf* a) {
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
template <int G>
L_CALL void d_type_eval(const DScene& S, const float* __restrict__ pool, int row, float lam, const float* wi,
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
    float s_ax[3];
    d_s_axis(wi, n, s_ax);
    Cf es, ep;
    d_components(er, ei, wi, s_ax, &es, &ep);
    float F = c_abs2(ev.amps[0]) * c_abs2(es) + c_abs2(ev.amps[1]) * c_abs2(ep);
    F = d_clip01(F);
    split[0] = F; split[1] = 0.0f; split[2] = 0.0f; split[3] = 0.0f; split[4] = 1.0f - F;
    Rc = col[LUMEN_COL_R];
  } else {
    d_amplitudes(cos_i, n1, cf(col[LUMEN_COL_NR], col[LUMEN_COL_NK]), ev.amps);
    float s_ax[3];
    d_s_axis(wi, n, s_ax);
    Cf es, ep;
    d_components(er, ei, wi, s_ax, &es, &ep);
    Rc = d_clip01(c_abs2(ev.amps[0]) * c_abs2(es) + c_abs2(ev.amps[1]) * c_abs2(ep));
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
L_CALL void d_rayleigh_sample(const float* er, const float* ei, float r0, float r1, float r2, float* wo) {
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
