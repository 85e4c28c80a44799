/*
 * ORACLE (test infrastructure): the reference's navigator and CSG evaluator, restated for one ray on the CPU.
 *
 * Follows src/lumen/geometry/csg.py (leaf intervals, the postfix boolean, first_change), leaf_kernels.py (quadric
 * pieces), navigate.py (Geant4 volume tracking with surface identity) and surface_id.py. Candidates are scanned by
 * brute force over each volume's daughters (no acceleration structure), so the engine's BVH is checked against it.
 * Scope: quadric / plane leaves (no torus), no meshes, volumes nested in a tree (no overlap owners, no ancestor
 * clipping, no frame groups), plain vertex table (a crossing is visible where the class changes).
 */
#ifndef LUMEN_ORACLE_GEOM_H
#define LUMEN_ORACLE_GEOM_H

#include <algorithm>

#include "../include/lumen_b200.h"
#include "lmath.h"

#define O_HUGE 1e30f
#define O_BIG 1e29f
#define O_EPS32 1.1920928955078125e-7f
#define O_BAND_ULPS_EPS 9.5367431640625e-07f /* BAND_ULPS (8) x eps32 (src/lumen/rules/tolerances.py:76) */
#define O_BAND_FLOOR 1e-9f
#define O_K_ON 4.0f
#define O_RELOCATE_BANDS 0.25f
#define O_ZERO_STEP_BANDS 0.125f
#define O_PUSH_BANDS 8.0f
#define O_TANGENT_ULPS 16.0f
#define O_DIVISOR_FLOOR 1e-30f
#define O_TINY_DIR 1e-30f
#define O_LINEAR_REL 1e-12f
#define O_PARALLEL 1e-12f
#define O_GRAZE 256.0f
#define O_ZSBP 10 /* ZERO_STEPS_BEFORE_PUSH */
#define O_ZSBK 25 /* ZERO_STEPS_BEFORE_KILL */
#define O_MAX_SCAN_PER_LEAF 4
#define O_MAX_SCAN_EXTRA 5
#define O_TINY_NORMAL 1.17549435e-38f

typedef struct OScene {
  const LumenSceneDesc* D;
  int n;      /* volumes; n = the outside */
  int LM, FM; /* most leaves of a kind, most faces of a leaf (1 + planes) */
  int SU;     /* first face code: a code below it is a plain item */
} OScene;

/* ------------------------------------------------------------------------------------------- small vector math */
static inline float o_dot(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline float o_maxabs3(const float* a) {
  float m = fabsf(a[0]);
  if (fabsf(a[1]) > m) m = fabsf(a[1]);
  if (fabsf(a[2]) > m) m = fabsf(a[2]);
  return m;
}
static inline float o_min(float a, float b) { return a < b ? a : b; }
static inline float o_max(float a, float b) { return a > b ? a : b; }
/* band(scale) = BAND_ULPS eps scale + BAND_FLOOR (src/lumen/rules/navigation.py:121) */
static inline float o_band(float scale) { return O_BAND_ULPS_EPS * scale + O_BAND_FLOOR; }
static inline float o_safe_norm(const float* v) { return sqrtf(o_max(o_dot(v, v), O_TINY_NORMAL)); }

/* ------------------------------------------------------------------------------------------------ accessors */
static inline const int32_t* o_vi(const OScene* S, int v) { return S->D->vol_i + (size_t)v * LUMEN_VOL_I; }
static inline const float* o_vf(const OScene* S, int v) { return S->D->vol_f + (size_t)v * LUMEN_VOL_F; }
static inline const int32_t* o_ki(const OScene* S, int k) { return S->D->kind_i + (size_t)k * LUMEN_KIND_I; }
static inline const float* o_lf(const OScene* S, int g) { return S->D->leaf_f + (size_t)g * LUMEN_LEAF_F; }
static inline const int32_t* o_li(const OScene* S, int g) { return S->D->leaf_i + (size_t)g * LUMEN_LEAF_I; }
static inline const float* o_pl(const OScene* S, int q) { return S->D->plane_f + (size_t)q * LUMEN_PLANE_F; }
static inline int o_cls(const OScene* S, int v) { return o_vi(S, v)[LUMEN_VI_CLS]; }
static inline int o_parent(const OScene* S, int v) { return o_vi(S, v)[LUMEN_VI_PARENT]; }
/* rank of a candidate: minus its place in the rule's order (navigate.py:208) */
static inline int o_rank(const OScene* S, int i) { return i >= 0 ? -o_vi(S, i)[LUMEN_VI_PRIO] : 0; }

/* the ray in volume i's frame: local = R^T (x - t) (navigate.py:151) */
static inline void o_to_local_pt(const OScene* S, int i, const float* x, float* xl) {
  const float* f = o_vf(S, i);
  const float* R = f + LUMEN_VF_R;
  float v0 = x[0] - f[LUMEN_VF_T], v1 = x[1] - f[LUMEN_VF_T + 1], v2 = x[2] - f[LUMEN_VF_T + 2];
  for (int a = 0; a < 3; ++a) xl[a] = R[a] * v0 + R[3 + a] * v1 + R[6 + a] * v2;
}
static inline void o_to_local_dir(const OScene* S, int i, const float* d, float* dl) {
  const float* R = o_vf(S, i) + LUMEN_VF_R;
  for (int a = 0; a < 3; ++a) dl[a] = R[a] * d[0] + R[3 + a] * d[1] + R[6 + a] * d[2];
}
static inline void o_to_world_dir(const OScene* S, int i, const float* g, float* gw) {
  const float* R = o_vf(S, i) + LUMEN_VF_R;
  for (int a = 0; a < 3; ++a) gw[a] = R[3 * a] * g[0] + R[3 * a + 1] * g[1] + R[3 * a + 2] * g[2];
}

/* ------------------------------------------------------------------------------- one leaf along a line (csg.py) */
typedef struct OIv { float lo0, hi0; int f_lo0, f_hi0; float lo1, hi1; int f_lo1, f_hi1; } OIv;

static inline void o_Av(const float* A, const float* v, float* out) {
  for (int a = 0; a < 3; ++a) out[a] = A[3 * a] * v[0] + A[3 * a + 1] * v[1] + A[3 * a + 2] * v[2];
}

/* quadric pieces [L0, R0], [L1, inf) along y + t d (leaf_kernels.py:81 quad_line, :41 _roots, :60 _pieces) */
static inline void o_quad_line(const float* lf, const float* y, const float* d, float* L0, float* R0, int* L0q,
                               int* R0q, float* L1, float* R1) {
  const float* A = lf + LUMEN_LF_A;
  const float* b = lf + LUMEN_LF_B;
  float c = lf[LUMEN_LF_C], sa = lf[LUMEN_LF_SA];
  const float inf = O_HUGE;
  float t_o = -o_dot(y, d);
  float y0[3] = {y[0] + t_o * d[0], y[1] + t_o * d[1], y[2] + t_o * d[2]};
  float Ad[3];
  o_Av(A, d, Ad);
  float alpha = o_dot(Ad, d);
  int lin = fabsf(alpha) < o_max(O_LINEAR_REL * sa, O_DIVISOR_FLOOR);
  float bdd = o_dot(b, d);
  float Ay0[3];
  o_Av(A, y0, Ay0);
  float beta0 = o_dot(Ay0, d) + bdd;
  float gam0 = (o_dot(y0, Ay0) + 2.0f * o_dot(b, y0)) + c;
  int near_ = !lin && (alpha * gam0 > 0.5f * beta0 * beta0);
  float t_c = t_o + (near_ ? -beta0 / alpha : 0.0f);
  float yc[3] = {y[0] + t_c * d[0], y[1] + t_c * d[1], y[2] + t_c * d[2]};
  float Ayc[3];
  o_Av(A, yc, Ayc);
  float beta = o_dot(Ayc, d) + bdd;
  float gam = (o_dot(yc, Ayc) + 2.0f * o_dot(b, yc)) + c;
  /* _roots */
  float D = beta * beta - alpha * gam;
  int Dpos = D > O_TANGENT_ULPS * O_EPS32 * (beta * beta + fabsf(alpha * gam));
  float sD = sqrtf(Dpos ? D : 1.0f);
  float sgn = beta >= 0.0f ? 1.0f : -1.0f;
  float s_ = -(beta + sgn * (Dpos ? sD : 0.0f));
  int s_ok = fabsf(s_) > O_DIVISOR_FLOOR;
  float r1 = lin ? inf : s_ / alpha;
  float r2 = s_ok ? gam / s_ : 0.0f;
  float rmin = o_min(r1, r2) + t_c;
  float rmax = o_max(r1, r2) + t_c;
  int b_small = fabsf(beta) < O_DIVISOR_FLOOR;
  float tl = t_c - gam / (b_small ? 1.0f : 2.0f * beta);
  /* _pieces */
  int lin_ent = lin && !b_small && beta < 0.0f;
  int lin_ext = lin && !b_small && beta > 0.0f;
  int lin_all = lin && b_small && gam <= 0.0f;
  int pos = !lin && alpha > 0.0f;
  int neg = !lin && alpha < 0.0f;
  *L0 = pos ? (Dpos ? rmin : inf) : (neg ? -inf : (lin_ent ? tl : ((lin_ext || lin_all) ? -inf : inf)));
  *R0 = pos ? (Dpos ? rmax : -inf)
            : (neg ? (Dpos ? rmin : inf) : (lin_ext ? tl : ((lin_ent || lin_all) ? inf : -inf)));
  *L0q = (pos && Dpos) || lin_ent;
  *R0q = (pos && Dpos) || (neg && Dpos) || lin_ext;
  int has1 = neg && Dpos;
  *L1 = has1 ? rmax : inf;
  *R1 = has1 ? inf : -inf;
}

/* a leaf's two intervals along o + t d (kind frame): csg.py:116 _planes, :138 _q_iv */
/* ------------------------------------------------------------------------------------------------ the torus */
/* leaf_kernels.py:212 torus_set on a unit ray o + s d in the torus's canonical frame: g(s) = (rho - R)^2 + z^2 - r^2
   bracketed on the padded bounding sphere, split at its (closed-form) inflection points, the extrema and then the
   roots of the six monotone pieces found by bisection; csg.py:175 the whole line's ball / slab / annulus pretests */
#define O_BISECT 40
#define O_TORUS_BRACKET_ULPS 64.0f
#define O_TORUS_AXIAL 1e-12f
#define O_TORUS_PAD_REL 1e-4f

static inline float o_torus_g(float R, float r, const float* oc, const float* d, float s) {
  const float p[3] = {oc[0] + s * d[0], oc[1] + s * d[1], oc[2] + s * d[2]};
  const float rho2 = p[0] * p[0] + p[1] * p[1];
  const float dr = (rho2 - R * R) / (sqrtf(o_max(rho2, 0.0f)) + R);
  return dr * dr + p[2] * p[2] - r * r;
}
static inline float o_torus_dg(float R, const float* oc, const float* d, float s) {
  const float p[3] = {oc[0] + s * d[0], oc[1] + s * d[1], oc[2] + s * d[2]};
  const float rho2 = p[0] * p[0] + p[1] * p[1];
  const float rho = sqrtf(o_max(rho2, O_TINY_NORMAL));
  const float dr = (rho2 - R * R) / (rho + R);
  return 2.0f * dr * ((p[0] * d[0] + p[1] * d[1]) / rho) + 2.0f * p[2] * d[2];
}
static inline int o_torus_meets(float R, float r, const float* o, const float* d) {
  const float Rb = (R + r) * (1.0f + O_TORUS_PAD_REL);
  const float bb = o[0] * d[0] + o[1] * d[1] + o[2] * d[2];
  const float disc = Rb * Rb - (o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - bb * bb);
  const float sq = sqrtf(o_max(disc, 0.0f));
  float lo = -bb - sq, hi = -bb + sq;
  int meet = disc > 0.0f && lo <= hi;
  const float pad = O_TORUS_PAD_REL * (R + r), rz = r + pad;
  const int flat = fabsf(d[2]) < O_PARALLEL;
  const float iz = 1.0f / (flat ? 1.0f : d[2]);
  if (!flat) {
    const float za = (-rz - o[2]) * iz, zb = (rz - o[2]) * iz;
    lo = o_max(lo, o_min(za, zb));
    hi = o_min(hi, o_max(za, zb));
  }
  meet = meet && lo <= hi && (!flat || fabsf(o[2]) <= rz);
  const float qa = d[0] * d[0] + d[1] * d[1], qb = o[0] * d[0] + o[1] * d[1], qc = o[0] * o[0] + o[1] * o[1];
  const float sm = o_min(o_max(-qb / (qa > O_PARALLEL ? qa : 1.0f), lo), hi);
  const float near2 = qa > O_PARALLEL ? qa * sm * sm + 2.0f * qb * sm + qc : qc;
  const float far2 = o_max(qa * lo * lo + 2.0f * qb * lo + qc, qa * hi * hi + 2.0f * qb * hi + qc);
  const float rout = R + r + pad, rin = o_max(R - r - pad, 0.0f);
  return meet && near2 <= rout * rout && far2 >= rin * rin;
}
static inline void o_torus_set(float R, float r, const float* o, const float* d, float* lo, float* hi) {
  const float tc = -((o[0] * d[0] + o[1] * d[1]) + o[2] * d[2]);
  const float oc[3] = {o[0] + tc * d[0], o[1] + tc * d[1], o[2] + tc * d[2]};
  const float q0 = (oc[0] * oc[0] + oc[1] * oc[1]) + oc[2] * oc[2];
  const float Rb = (R + r) * (1.0f + O_TORUS_BRACKET_ULPS * O_EPS32);
  const float b0 = (oc[0] * d[0] + oc[1] * d[1]) + oc[2] * d[2];
  const float disc = Rb * Rb - q0 + b0 * b0;
  const int in_ball = disc > 0.0f;
  const float sq = sqrtf(in_ball ? disc : 1.0f);
  const float s0 = -b0 - sq, s1 = -b0 + sq;
  const float a = d[0] * d[0] + d[1] * d[1];
  const float bxy = oc[0] * d[0] + oc[1] * d[1];
  const float cxy = oc[0] * oc[0] + oc[1] * oc[1];
  const int off_axis = a > O_TORUS_AXIAL;
  const float as = off_axis ? a : 1.0f;
  const float sv = off_axis ? -bxy / as : 0.0f;
  const float m2 = o_max(off_axis ? cxy - bxy * bxy / as : cxy, 0.0f);
  const float cr = o_cbrt(R * a * m2);
  const float w2 = (cr * cr - m2) / as;
  const float w = sqrtf(off_axis && w2 > 0.0f ? w2 : 0.0f);
  const float p1 = o_min(o_max(sv - w, s0), s1), p2 = o_min(o_max(sv + w, s0), s1);
  const float a0[3] = {s0, p1, p2}, a1[3] = {p1, p2, s1};
  float ex[3];
  for (int k = 0; k < 3; ++k) { /* g' rises through its minima, falls through its maximum */
    float l = a0[k], h = a1[k];
    for (int it = 0; it < O_BISECT; ++it) {
      const float m = 0.5f * (l + h);
      const float gp = o_torus_dg(R, oc, d, m);
      if (k == 1 ? gp > 0.0f : gp < 0.0f) l = m; else h = m;
    }
    ex[k] = 0.5f * (l + h);
  }
  const float kn[7] = {s0, ex[0], p1, ex[1], p2, ex[2], s1};
  float roots[6];
  for (int k = 0; k < 6; ++k) {
    const int in_l = o_torus_g(R, r, oc, d, kn[k]) <= 0.0f, in_r = o_torus_g(R, r, oc, d, kn[k + 1]) <= 0.0f;
    float l = kn[k], h = kn[k + 1];
    for (int it = 0; it < O_BISECT; ++it) {
      const float m = 0.5f * (l + h);
      if ((o_torus_g(R, r, oc, d, m) <= 0.0f) == in_l) l = m; else h = m;
    }
    roots[k] = (in_l != in_r && kn[k + 1] > kn[k] && in_ball) ? 0.5f * (l + h) + tc : O_HUGE;
  }
  std::sort(roots, roots + 6);
  const int ok0 = roots[1] < O_BIG, ok1 = roots[3] < O_BIG;
  lo[0] = ok0 ? roots[0] : O_HUGE; hi[0] = ok0 ? roots[1] : O_HUGE;
  lo[1] = ok1 ? roots[2] : O_HUGE; hi[1] = ok1 ? roots[3] : O_HUGE;
}
/* a torus leaf along o + t d (kind frame): canonical frame u = M (x - og), the unit ray, the roots scaled back
   (csg.py:207 _t_iv) */
static inline void o_torus_line(const float* lf, const float* o, const float* d, float* L0, float* R0, float* L1,
                                float* R1) {
  const float* M = lf + LUMEN_LF_A;
  const float R = lf[LUMEN_LF_B], r = lf[LUMEN_LF_B + 1];
  const float xl[3] = {o[0] - lf[0], o[1] - lf[1], o[2] - lf[2]};
  float ou[3], dl[3];
  o_Av(M, xl, ou);
  o_Av(M, d, dl);
  const float kk = sqrtf(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
  const float du[3] = {dl[0] / kk, dl[1] / kk, dl[2] / kk};
  float lo[2] = {O_HUGE, O_HUGE}, hi[2] = {O_HUGE, O_HUGE};
  if (o_torus_meets(R, r, ou, du)) o_torus_set(R, r, ou, du, lo, hi);
  *L0 = fabsf(lo[0]) < O_BIG ? lo[0] / kk : lo[0];
  *R0 = fabsf(hi[0]) < O_BIG ? hi[0] / kk : hi[0];
  *L1 = fabsf(lo[1]) < O_BIG ? lo[1] / kk : lo[1];
  *R1 = fabsf(hi[1]) < O_BIG ? hi[1] / kk : hi[1];
}

static inline OIv o_leaf_iv(const OScene* S, int g, const float* o, const float* d) {
  const float* lf = o_lf(S, g);
  const int32_t* li = o_li(S, g);
  const float inf = O_HUGE;
  float y[3] = {o[0] - lf[LUMEN_LF_OQ], o[1] - lf[LUMEN_LF_OQ + 1], o[2] - lf[LUMEN_LF_OQ + 2]};
  float ol[3] = {o[0] - lf[LUMEN_LF_OG], o[1] - lf[LUMEN_LF_OG + 1], o[2] - lf[LUMEN_LF_OG + 2]};
  float t0p = -inf, t1p = inf;
  int f0p = -1, f1p = -1, ep = 0;
  for (int k = 0; k < li[2]; ++k) {
    const float* pl = o_pl(S, li[1] + k);
    float nd = pl[0] * d[0] + pl[1] * d[1] + pl[2] * d[2];
    float rhs = pl[3] - (pl[0] * ol[0] + pl[1] * ol[1] + pl[2] * ol[2]);
    int par = fabsf(nd) < O_PARALLEL;
    float tp = rhs / (par ? 1.0f : nd);
    float ent = nd < -O_PARALLEL ? tp : -inf;
    float ext = nd > O_PARALLEL ? tp : inf;
    if (ent > t0p) { t0p = ent; f0p = k + 1; }
    if (ext < t1p) { t1p = ext; f1p = k + 1; }
    ep = ep || (par && rhs < 0.0f);
  }
  int has_q = li[0] == 1;
  float L0 = -inf, R0 = inf, L1 = inf, R1 = -inf;
  int L0q = 0, R0q = 0;
  if (has_q) o_quad_line(lf, y, d, &L0, &R0, &L0q, &R0q, &L1, &R1);
  if (li[0] == 2) {
    o_torus_line(lf, o, d, &L0, &R0, &L1, &R1);
    L0q = R0q = 1;
  }
  OIv r;
  /* clip each piece by the slab */
  {
    float lo = o_max(L0, t0p), hi = o_min(R0, t1p);
    int flo = L0 > t0p ? (L0q ? 0 : f0p) : f0p;
    int fhi = R0 < t1p ? (R0q ? 0 : f1p) : f1p;
    int ok = lo < hi && !ep;
    r.lo0 = ok ? lo : inf; r.hi0 = ok ? hi : inf; r.f_lo0 = ok ? flo : -1; r.f_hi0 = ok ? fhi : -1;
  }
  {
    float lo = o_max(L1, t0p), hi = o_min(R1, t1p);
    int flo = L1 > t0p ? 0 : f0p;
    int fhi = R1 < t1p ? 0 : f1p; /* a quadric's second piece is unbounded above; a torus's ends at a root */
    int ok = lo < hi && !ep;
    r.lo1 = ok ? lo : inf; r.hi1 = ok ? hi : inf; r.f_lo1 = ok ? flo : -1; r.f_hi1 = ok ? fhi : -1;
  }
  if (r.lo0 >= inf && r.lo1 < inf) { /* the non-empty piece first */
    OIv s = r;
    r.lo0 = s.lo1; r.hi0 = s.hi1; r.f_lo0 = s.f_lo1; r.f_hi0 = s.f_hi1;
    r.lo1 = s.lo0; r.hi1 = s.hi0; r.f_lo1 = s.f_lo0; r.f_hi1 = s.f_hi0;
  }
  return r;
}

/* whether leaf g holds the point x (kind frame; closed, no tolerance): csg.py:301 _inside_leaf */
static inline int o_inside_leaf(const OScene* S, int g, const float* x) {
  const float* lf = o_lf(S, g);
  const int32_t* li = o_li(S, g);
  float xl[3] = {x[0] - lf[LUMEN_LF_OG], x[1] - lf[LUMEN_LF_OG + 1], x[2] - lf[LUMEN_LF_OG + 2]};
  float y[3] = {x[0] - lf[LUMEN_LF_OQ], x[1] - lf[LUMEN_LF_OQ + 1], x[2] - lf[LUMEN_LF_OQ + 2]};
  int pl = 1;
  for (int k = 0; k < li[2]; ++k) {
    const float* p = o_pl(S, li[1] + k);
    pl = pl && (p[0] * xl[0] + p[1] * xl[1] + p[2] * xl[2] <= p[3]);
  }
  if (li[0] == 2) { /* the torus reads no planes: (rho - R)^2 + z^2 <= r^2 */
    float u[3];
    o_Av(lf + LUMEN_LF_A, xl, u);
    const float dr = sqrtf(u[0] * u[0] + u[1] * u[1]) - lf[LUMEN_LF_B];
    return dr * dr + u[2] * u[2] <= lf[LUMEN_LF_B + 1] * lf[LUMEN_LF_B + 1];
  }
  if (li[0] != 1) return pl;
  float Ay[3];
  o_Av(lf + LUMEN_LF_A, y, Ay);
  const float* b = lf + LUMEN_LF_B;
  float qv = (o_dot(y, Ay) + 2.0f * (b[0] * y[0] + b[1] * y[1] + b[2] * y[2])) + lf[LUMEN_LF_C];
  return pl && qv <= 0.0f;
}

/* the kind's postfix boolean (csg.py:320 _program) over member(l) in {0, 1} */
typedef int (*OMember)(void* ctx, int l);
static inline int o_program(const OScene* S, int kind, OMember member, void* ctx) {
  const int32_t* k = o_ki(S, kind);
  int32_t s = 0;
  for (int p = 0; p < k[3]; ++p) {
    const int32_t* g = S->D->prog_i + (size_t)(k[2] + p) * LUMEN_PROG_I;
    int op = g[0], arg = g[1];
    int32_t bb = s & 1, aa = (s >> 1) & 1;
    int32_t r = op == 1 ? (aa | bb) : (op == 2 ? (aa & bb) : (aa & (1 - bb)));
    if (op == 0) s = (s << 1) | (member(ctx, arg) & 1);
    else s = ((s >> 2) << 1) | r;
  }
  return (s & 1) == 1;
}

typedef struct OPtCtx { const OScene* S; int l0; const float* x; } OPtCtx;
static inline int o_member_pt(void* c, int l) {
  OPtCtx* p = (OPtCtx*)c;
  return o_inside_leaf(p->S, p->l0 + l, p->x);
}
/* whether the kind holds the point x (csg.py:341 inside) */
static inline int o_inside_kind(const OScene* S, int kind, const float* x) {
  OPtCtx c = {S, o_ki(S, kind)[0], x};
  return o_program(S, kind, o_member_pt, &c);
}

/* ------------------------------------------------------------------- first_change (csg.py:369-449), one kind */
typedef struct OScan {
  const OScene* S;
  int kind, nl;
  OIv iv[LUMEN_MAX_LEAVES]; /* every leaf's intervals along the ray (quadric leaves do not depend on the window) */
  float xa;                  /* max |o| (kind frame), the band's scale */
  float t1;
  int want;                  /* -1 any change, 1 the first entry, 0 the first exit */
  int has_init, init_known, init_inside;
  int has_skip, skip_leaf, skip_face, skip_entry; float skip_thi;
  int has_on, on_leaf, on_inside; float on_tend;
  /* the membership override in force at a probe (on_face with its running end) */
  float hend;
  float probe_t;
} OScan;

static inline float o_scan_band(const OScan* s, float t) { return o_band(s->xa + fabsf(t)); }

static inline int o_member_iv(void* c, int l) {
  OScan* s = (OScan*)c;
  const OIv* v = &s->iv[l];
  float t = s->probe_t;
  int m = (v->lo0 <= t && t < v->hi0) || (v->lo1 <= t && t < v->hi1);
  if (s->has_on && l == s->on_leaf && t < s->hend) m = s->on_inside;
  return m;
}
/* the solid's membership just after o + t d (csg.py:346 _mem_at) */
static inline int o_mem_at(OScan* s, float t, int use_on) {
  int save = s->has_on;
  s->has_on = save && use_on;
  s->probe_t = t;
  int r = o_program(s->S, s->kind, o_member_iv, s);
  s->has_on = save;
  return r;
}

static inline void o_scan_init(OScan* s, const OScene* S, int kind, const float* o, const float* d, float t1) {
  s->S = S;
  s->kind = kind;
  const int32_t* k = o_ki(S, kind);
  s->nl = k[1];
  for (int l = 0; l < s->nl; ++l) s->iv[l] = o_leaf_iv(S, k[0] + l, o, d);
  s->xa = o_max(o_max(fabsf(o[0]), fabsf(o[1])), fabsf(o[2]));
  s->t1 = t1;
  s->want = -1;
  s->has_init = s->has_skip = s->has_on = 0;
  s->hend = -O_HUGE;
}

typedef struct OFirst { int hit; float t; int inside, leaf, face; } OFirst;
typedef struct OFc { int hit; float t; int inside, leaf, face, inside0; OFirst first; } OFc;

/* the nearest leaf endpoint after t_cur (<= t1): csg.py:369 _nearest */
static inline void o_nearest(const OScan* s, float t_cur, float* e1o, int* lbo, int* fco, int* eko) {
  float e1 = O_HUGE;
  int lb = -1, fc = -1, ek = 0;
  for (int l = 0; l < s->nl; ++l) {
    const OIv* v = &s->iv[l];
    float eps_[4] = {v->lo0, v->hi0, v->lo1, v->hi1};
    int fps[4] = {v->f_lo0, v->f_hi0, v->f_lo1, v->f_hi1};
    int ens[4] = {1, 0, 1, 0};
    for (int j = 0; j < 4; ++j) {
      float ep = eps_[j];
      int ok = fabsf(ep) < O_BIG && ep <= s->t1 && ep > t_cur && ep < e1;
      if (s->has_skip)
        ok = ok && !(l == s->skip_leaf && fps[j] == s->skip_face && s->skip_entry == ens[j] && ep < s->skip_thi);
      if (ok) { e1 = ep; lb = l; fc = fps[j]; ek = ens[j]; }
    }
  }
  *e1o = e1; *lbo = lb; *fco = fc; *eko = ek;
}

/* the first change of the kind's membership in (t0, t1] (csg.py:417 first_change) */
static inline OFc o_first_change(OScan* s, float t0) {
  float t_cur = t0;
  int done = 0, now = 0, lb_h = -1, fc_h = -1, now0 = 0, it = 0;
  OFirst fs = {0, O_HUGE, 0, -1, -1};
  s->hend = s->has_on ? s->on_tend : -O_HUGE;
  while (!done && t_cur < O_HUGE && it < O_MAX_SCAN_PER_LEAF * s->nl + O_MAX_SCAN_EXTRA) {
    int first = it == 0;
    float e; int lb, fc, ek;
    if (first) { e = t0; lb = -1; fc = -1; ek = 0; }
    else o_nearest(s, t_cur, &e, &lb, &fc, &ek);
    int has = first || e < O_HUGE;
    float tp = first ? t0 : e + o_scan_band(s, e);
    if (s->has_on && !first && has && lb == s->on_leaf && ek != s->on_inside) s->hend = o_min(s->hend, e);
    int aft;
    if (!s->has_init) aft = has ? o_mem_at(s, tp, 1) : now;
    else if (has && !(first && s->init_known)) aft = o_mem_at(s, tp, 1);
    else aft = (first && s->init_known) ? s->init_inside : now;
    if (first) now0 = aft;
    int chg = !first && has && aft != now;
    int vis = s->want < 0 ? chg : (chg && aft == s->want);
    int nw = chg && !fs.hit;
    if (nw) { fs.t = e; fs.inside = aft; fs.leaf = lb; fs.face = fc; }
    fs.hit = fs.hit || chg;
    if (has) now = aft;
    float t_nx = first ? t0 : (vis ? e : (has ? tp : O_HUGE));
    if (vis) { lb_h = lb; fc_h = fc; }
    done = vis;
    t_cur = t_nx;
    it += 1;
  }
  OFc r;
  r.hit = done;
  r.t = done ? t_cur : s->t1;
  r.inside = done ? now : now0;
  r.leaf = lb_h;
  r.face = fc_h;
  r.inside0 = now0;
  r.first = fs;
  return r;
}

/* the gradient of kind-local leaf `leaf` (face 0 its quadric, >= 1 its planes) at x (kind frame): csg.py:452 */
static inline void o_leaf_grad(const OScene* S, int kind, int leaf, int face, const float* x, float* g) {
  int gi = o_ki(S, kind)[0] + (leaf > 0 ? leaf : 0);
  const float* lf = o_lf(S, gi);
  const int32_t* li = o_li(S, gi);
  if (face >= 1) {
    const float* p = o_pl(S, li[1] + face - 1);
    g[0] = p[0]; g[1] = p[1]; g[2] = p[2];
    return;
  }
  if (li[0] == 2) { /* M^T ((rho - R) / rho u_x, (rho - R) / rho u_y, u_z) */
    const float* M = lf + LUMEN_LF_A;
    const float xl[3] = {x[0] - lf[0], x[1] - lf[1], x[2] - lf[2]};
    float u[3];
    o_Av(M, xl, u);
    const float rho = sqrtf(o_max(u[0] * u[0] + u[1] * u[1], O_DIVISOR_FLOOR));
    const float k = (rho - lf[LUMEN_LF_B]) / rho;
    const float gu[3] = {k * u[0], k * u[1], u[2]};
    for (int a = 0; a < 3; ++a) g[a] = (M[a] * gu[0] + M[3 + a] * gu[1]) + M[6 + a] * gu[2];
    return;
  }
  float y[3] = {x[0] - lf[LUMEN_LF_OQ], x[1] - lf[LUMEN_LF_OQ + 1], x[2] - lf[LUMEN_LF_OQ + 2]};
  float Ay[3];
  o_Av(lf + LUMEN_LF_A, y, Ay);
  const float* b = lf + LUMEN_LF_B;
  for (int a = 0; a < 3; ++a) g[a] = 2.0f * (Ay[a] + b[a]);
}
/* |f| / |grad f| of a leaf's face at x (kind frame): csg.py:470 leaf_dist */
static inline float o_leaf_dist(const OScene* S, int kind, int leaf, int face, const float* x) {
  int gi = o_ki(S, kind)[0] + (leaf > 0 ? leaf : 0);
  const float* lf = o_lf(S, gi);
  const int32_t* li = o_li(S, gi);
  float f;
  if (face >= 1) {
    const float* p = o_pl(S, li[1] + face - 1);
    float xl[3] = {x[0] - lf[LUMEN_LF_OG], x[1] - lf[LUMEN_LF_OG + 1], x[2] - lf[LUMEN_LF_OG + 2]};
    f = p[0] * xl[0] + p[1] * xl[1] + p[2] * xl[2] - p[3];
  } else if (li[0] == 2) {
    const float xl[3] = {x[0] - lf[0], x[1] - lf[1], x[2] - lf[2]};
    float u[3];
    o_Av(lf + LUMEN_LF_A, xl, u);
    const float dr = sqrtf(u[0] * u[0] + u[1] * u[1]) - lf[LUMEN_LF_B], r = lf[LUMEN_LF_B + 1];
    f = 0.5f * (dr * dr + u[2] * u[2] - r * r);
  } else {
    float y[3] = {x[0] - lf[LUMEN_LF_OQ], x[1] - lf[LUMEN_LF_OQ + 1], x[2] - lf[LUMEN_LF_OQ + 2]};
    float Ay[3];
    o_Av(lf + LUMEN_LF_A, y, Ay);
    const float* b = lf + LUMEN_LF_B;
    f = (o_dot(y, Ay) + 2.0f * (b[0] * y[0] + b[1] * y[1] + b[2] * y[2])) + lf[LUMEN_LF_C];
  }
  float g[3];
  o_leaf_grad(S, kind, leaf, face, x, g);
  return fabsf(f) / o_safe_norm(g);
}

/* world gradient / face distance of volume i's leaf face at the world point x (surface_id.py:91 hit_grad, :100) */
static inline void o_hit_grad(const OScene* S, int item, int leaf, int face, const float* x, float* gw) {
  int i = item < 0 ? 0 : (item > S->n - 1 ? S->n - 1 : item);
  float xl[3], g[3];
  o_to_local_pt(S, i, x, xl);
  o_leaf_grad(S, o_vi(S, i)[LUMEN_VI_KIND], leaf, face, xl, g);
  o_to_world_dir(S, i, g, gw);
}
static inline float o_face_dist(const OScene* S, int item, int leaf, int face, const float* x) {
  int i = item < 0 ? 0 : (item > S->n - 1 ? S->n - 1 : item);
  float xl[3];
  o_to_local_pt(S, i, x, xl);
  return o_leaf_dist(S, o_vi(S, i)[LUMEN_VI_KIND], leaf, face, xl);
}

/* ----------------------------------------------------------------------------- surface codes (surface_id.py) */
/* srf = item (plain, < SU) or SU + (((item * LM + leaf) * FM + face) * 4 + 2 o + e) */
static inline int o_srf_pack(const OScene* S, int item, int leaf, int face, int o, int e) {
  if (item < 0 || leaf < 0 || face < 0) return item;
  return S->SU + ((item * S->LM + leaf) * S->FM + face) * 4 + 2 * o + e;
}
typedef struct OSrf { int item, leaf, face, o, known, e; } OSrf;
static inline OSrf o_srf_decode(const OScene* S, int s) {
  OSrf r;
  if (s < S->SU) { r.item = s; r.leaf = -1; r.face = -1; r.o = 0; r.known = 0; r.e = 0; return r; }
  int u = s - S->SU;
  r.e = u % 2; u /= 2;
  r.o = u % 2; u /= 2;
  r.face = u % S->FM; u /= S->FM;
  r.leaf = u % S->LM; u /= S->LM;
  r.item = u;
  r.known = 1;
  return r;
}

/* ---------------------------------------------------------------------------------- point and ray membership */
static inline int o_holds_point(const OScene* S, int i, const float* x) {
  float xl[3];
  o_to_local_pt(S, i, x, xl);
  return o_inside_kind(S, o_vi(S, i)[LUMEN_VI_KIND], xl);
}
/* whether volume i holds the ray just after t (navigate.py:163 ray_holds, csg.py:362 inside_ray) */
static inline int o_ray_holds(const OScene* S, int i, const float* od, const float* dd, float t) {
  float ol[3], dl[3];
  o_to_local_pt(S, i, od, ol);
  o_to_local_dir(S, i, dd, dl);
  OScan s;
  o_scan_init(&s, S, o_vi(S, i)[LUMEN_VI_KIND], ol, dl, O_HUGE);
  return o_mem_at(&s, t, 0);
}
/* whether x lies in volume i's world box padded by pad */
static inline int o_box_holds(const OScene* S, int i, const float* x, float pad) {
  const float* f = o_vf(S, i);
  for (int a = 0; a < 3; ++a)
    if (!(f[LUMEN_VF_LO + a] - pad <= x[a] && x[a] <= f[LUMEN_VF_HI + a] + pad)) return 0;
  return 1;
}

/* Geant4's LevelLocate: the first in the rule's order (navigation.py:150 level_locate_wins) */
static inline int o_level_wins(const OScene* S, int item, int found, int excl) {
  return (found < 0 || o_rank(S, item) > o_rank(S, found)) && item != excl && item < S->n;
}

/* the daughter of v holding the point x, or -1 (navigate.py:215 _find) */
static inline int o_find(const OScene* S, int v, const float* x) {
  const int32_t* vi = o_vi(S, v);
  int g = -1;
  for (int k = 0; k < vi[LUMEN_VI_CN]; ++k) {
    int i = S->D->cand[vi[LUMEN_VI_C0] + k];
    if (!o_box_holds(S, i, x, 0.0f)) continue;
    if (o_level_wins(S, i, g, -1) && o_holds_point(S, i, x)) g = i;
  }
  return g;
}
/* the deepest volume holding x (n: outside every volume) (navigate.py:226 locate) */
static inline int o_locate(const OScene* S, const float* x) {
  int v = S->n;
  for (;;) {
    int f = o_find(S, v, x);
    if (f < 0) return v;
    v = f;
  }
}
/* the daughter of v (other than excl) holding the ray just after t (navigate.py:243 _find_ray) */
static inline int o_find_ray(const OScene* S, int v, const float* od, const float* dd, float t, int excl, float pad) {
  const int32_t* vi = o_vi(S, v);
  float x[3] = {od[0] + t * dd[0], od[1] + t * dd[1], od[2] + t * dd[2]};
  int g = -1;
  for (int k = 0; k < vi[LUMEN_VI_CN]; ++k) {
    int i = S->D->cand[vi[LUMEN_VI_C0] + k];
    if (!o_box_holds(S, i, x, pad)) continue;
    if (o_level_wins(S, i, g, excl) && o_ray_holds(S, i, od, dd, t)) g = i;
  }
  return g;
}
/* up while v does not hold the ray just after t, then down (navigate.py:254 _settle) */
static inline int o_settle(const OScene* S, int v, const float* od, const float* dd, float t, int crossed, float pad,
                           int* moved) {
  int v_ = v, held = 0;
  for (int guard = 0; guard < 4 * S->n + 8; ++guard) {
    int vi = v_ < S->n - 1 ? v_ : S->n - 1;
    int test = !held && v_ < S->n && v_ != crossed;
    int ins = !test || o_ray_holds(S, vi, od, dd, t);
    int f = ins ? o_find_ray(S, v_, od, dd, t, crossed, pad) : -1;
    int nv = ins ? (f >= 0 ? f : v_) : o_parent(S, v_ < S->n ? v_ : S->n);
    held = ins && f >= 0;
    if (f < 0 && ins) break;
    v_ = nv;
  }
  *moved = v_ != v;
  return v_;
}

/* ------------------------------------------------------------------------------------------------ one visit */
typedef struct OSide { int known, leaf, face; float s; int entry; } OSide;
typedef struct OBest { float t; int item, leaf, face, zero, own; } OBest;
typedef struct OCtx {
  int v;
  const float *od, *dd;
  float t_lo, t_bound;
  int last;
  float band;
  OSide sd;
} OCtx;

/* the on-face rule (navigate.py:334 _on_face) */
static inline int o_on_face(const OScene* S, const OCtx* c, int i, const OFirst* fr, int kn_i) {
  float dt = fr->t - c->t_lo;
  float lim = O_K_ON * c->band;
  int far_ = 0;
  if (!kn_i && fr->hit && dt >= lim && dt < O_GRAZE * lim) {
    float x0[3] = {c->od[0] + c->t_lo * c->dd[0], c->od[1] + c->t_lo * c->dd[1], c->od[2] + c->t_lo * c->dd[2]};
    float xc[3] = {c->od[0] + fr->t * c->dd[0], c->od[1] + fr->t * c->dd[1], c->od[2] + fr->t * c->dd[2]};
    int lf = fr->leaf > 0 ? fr->leaf : 0;
    float g0[3], gc[3];
    o_hit_grad(S, i, lf, fr->face, x0, g0);
    o_hit_grad(S, i, lf, fr->face, xc, gc);
    float s0 = o_dot(g0, c->dd) / o_safe_norm(g0);
    int other_way = (s0 * o_dot(gc, c->dd) < 0.0f) && (fabsf(s0) > 1.0f / O_GRAZE);
    far_ = (o_face_dist(S, i, lf, fr->face, x0) < lim) && !other_way;
  }
  return !kn_i && fr->hit && (dt < lim || far_);
}

static inline int o_entry_wins(const OScene* S, float t, int item, const OBest* b) {
  return t < b->t || (t == b->t && (b->own || o_rank(S, item) > o_rank(S, b->item)));
}

/* the best event after volume i: own its first exit, a daughter its first entry (navigate.py:357-416) */
static inline OBest o_unit_visit(const OScene* S, const OCtx* c, int i, OBest b, int is_own) {
  const OSide* sd = &c->sd;
  float bnd = c->t_bound + c->band; /* the scan's window: the query's bound (order-independent) */
  float ol[3], dl[3];
  o_to_local_pt(S, i, c->od, ol);
  o_to_local_dir(S, i, c->dd, dl);
  int kn_i = sd->known && i == c->last;
  float t_on = c->t_lo + O_K_ON * c->band / o_max(fabsf(sd->s), 1.0f / O_GRAZE);
  int lf_on = kn_i ? sd->leaf : -2;
  OScan s;
  o_scan_init(&s, S, o_vi(S, i)[LUMEN_VI_KIND], ol, dl, bnd);
  s.want = is_own ? 0 : 1;
  s.has_init = 1; s.init_known = kn_i; s.init_inside = is_own;
  s.has_skip = 1; s.skip_leaf = lf_on; s.skip_face = sd->face; s.skip_entry = sd->entry; s.skip_thi = O_HUGE;
  s.has_on = 1; s.on_leaf = lf_on; s.on_inside = sd->entry; s.on_tend = t_on;
  OFc r = o_first_change(&s, c->t_lo);
  int h = r.hit, lf = r.leaf, f = r.face;
  float t = r.t;
  int on = o_on_face(S, c, i, &r.first, kn_i);
  int by_s = kn_i && (is_own ? sd->s > 0.0f : sd->s < 0.0f);
  int ins = kn_i ? (is_own ? (sd->s <= 0.0f && h) : sd->s < 0.0f) : (on ? r.first.inside : r.inside0);
  h = h && (is_own || !ins);
  int zero = is_own ? !ins : (ins && (i != c->last || kn_i));
  if (zero) {
    lf = by_s ? sd->leaf : (on ? r.first.leaf : -1);
    f = by_s ? sd->face : (on ? r.first.face : -1);
  }
  int by_on = zero && on && !by_s;
  int apart = 0;
  if (by_on) {
    float x0[3] = {c->od[0] + c->t_lo * c->dd[0], c->od[1] + c->t_lo * c->dd[1], c->od[2] + c->t_lo * c->dd[2]};
    apart = o_face_dist(S, i, lf > 0 ? lf : 0, f, x0) > c->band;
  }
  float te = apart ? r.first.t : (zero ? c->t_lo : (h ? t : O_HUGE));
  int wins = o_entry_wins(S, te, i, &b);
  int better = is_own || (!is_own && (zero || h) && wins);
  if (better) {
    OBest nb = {te, i, lf, f, zero && !apart, is_own};
    return nb;
  }
  return b;
}

/* the ray's slab test against volume i's padded world box (bvh.py:258 slab; navigate.py:424 _meets) */
static inline int o_meets_box(const OScene* S, const OCtx* c, int i, const float* inv) {
  const float* f = o_vf(S, i);
  float lo_t = -O_HUGE * 10.0f, hi_t = O_HUGE * 10.0f;
  for (int a = 0; a < 3; ++a) {
    float ta = (f[LUMEN_VF_LO + a] - c->od[a]) * inv[a];
    float tb = (f[LUMEN_VF_HI + a] - c->od[a]) * inv[a];
    lo_t = o_max(lo_t, o_min(ta, tb));
    hi_t = o_min(hi_t, o_max(ta, tb));
  }
  return lo_t <= hi_t && hi_t >= c->t_lo && lo_t <= c->t_bound + c->band;
}

/* the photon's next event in volume v: its own exit, then the first entry of every daughter whose box the ray meets
   (navigate.py:482 enter; the winner does not depend on the order of the daughters) */
static inline OBest o_enter(const OScene* S, const OCtx* c, int has_own, int vi) {
  OBest b = {O_HUGE, -1, -1, -1, 0, 0};
  if (has_own) b = o_unit_visit(S, c, vi, b, 1);
  float inv[3];
  for (int a = 0; a < 3; ++a) {
    float dv = c->dd[a];
    inv[a] = 1.0f / (fabsf(dv) < O_TINY_DIR ? (dv < 0.0f ? -O_TINY_DIR : O_TINY_DIR) : dv);
  }
  const int32_t* vr = o_vi(S, c->v);
  for (int k = 0; k < vr[LUMEN_VI_CN]; ++k) {
    int i = S->D->cand[vr[LUMEN_VI_C0] + k];
    if (o_meets_box(S, c, i, inv)) b = o_unit_visit(S, c, i, b, 0);
  }
  return b;
}

/* ------------------------------------------------------------------------------------------------- the query */
typedef struct OQuery {
  float t;
  int hit, cont;
  int vol_after, vol_before, vol_start, cls_before, cls_start, cls_after;
  float normal[3];
  int item, leaf, face, zero;
  float t_pass0, t_pass1;
  int n_pass, vol_at, srf, rounds;
} OQuery;

/* the first visible crossing along (o, d) before t_max for a photon in vol sitting on srf `last` (navigate.py:663
   query, with _round :557, _next_volume :515, _side :497, _finish :617) */
static inline OQuery o_query(const OScene* S, const float* o, const float* d, int vol, float t_max, int last,
                             const float* sn, float s_at) {
  const int OUT = S->n;
  float xa = o_maxabs3(o);
  int cls0 = o_cls(S, vol);
  OSrf l0 = o_srf_decode(S, last);
  int kn0 = l0.known;
  /* the round loop's carry */
  float t_lo = 0.0f;
  int v = vol, last_ = last, done = 0, it = 0;
  float rec_t = O_HUGE;
  int rec_item = -1, rec_leaf = -1, rec_face = -1, rec_zero = 0, rec_vb = vol, rec_vis = 0;
  int cur = cls0;
  float pz_tp0 = O_HUGE, pz_tp1 = O_HUGE, pz_tin = 0.0f;
  int pz_np = 0, pz_vend = vol, pz_hit = 0, pz_vat = vol, pz_zc = 0, pz_vin = vol;
  int guard = 0;
  while (!done) {
    float band = o_band(xa + fabsf(t_lo));
    int vi = v < OUT - 1 ? v : OUT - 1;
    int has_own = v < OUT;
    /* _side */
    OSrf ls = o_srf_decode(S, last_);
    OSide sd = {ls.known, ls.leaf, ls.face, 0.0f, 0};
    if (ls.known) {
      if (sn) {
        sd.s = o_dot(sn, d) * (ls.e ? 1.0f : -1.0f);
        sd.entry = sd.s * (ls.o ? 1.0f : -1.0f) < 0.0f;
      } else {
        float x0[3] = {o[0] + t_lo * d[0], o[1] + t_lo * d[1], o[2] + t_lo * d[2]};
        float g[3];
        o_hit_grad(S, ls.item, ls.leaf > 0 ? ls.leaf : 0, ls.face, x0, g);
        float gd = o_dot(g, d);
        sd.s = gd / o_safe_norm(g) * (ls.o ? 1.0f : -1.0f);
        sd.entry = gd < 0.0f;
      }
    }
    OCtx c = {v, o, d, t_lo, t_max, ls.item, band, sd};
    OBest ev = o_enter(S, &c, has_own, vi);
    float t_c = ev.t;
    int u_in = ev.item, l_in = ev.leaf, f_in = ev.face, z_in = ev.zero, is_own = ev.own;
    int hit = t_c < t_max;
    float step = o_band(xa + fabsf(hit ? t_c : t_lo));
    /* _next_volume */
    int nxt = v, moved = 0;
    {
      int go_in = !is_own;
      int uc = u_in < 0 ? 0 : (u_in > OUT - 1 ? OUT - 1 : u_in);
      int up = o_parent(S, v < OUT ? v : OUT);
      int nx0 = go_in ? u_in : up;
      int unit_x = go_in ? u_in : vi;
      int off = hit && l_in >= 0;
      float od2[3] = {o[0], o[1], o[2]};
      if (off) {
        float x[3] = {o[0] + t_c * d[0], o[1] + t_c * d[1], o[2] + t_c * d[2]};
        int itm = is_own ? vi : uc;
        int lf = l_in > 0 ? l_in : 0;
        float g[3];
        o_hit_grad(S, itm, lf, f_in, x, g);
        float gn = o_safe_norm(g);
        float n_[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
        float m = o_face_dist(S, itm, lf, f_in, x) + O_RELOCATE_BANDS * o_band(o_maxabs3(x));
        float sg = o_dot(n_, d) < 0.0f ? -1.0f : 1.0f;
        for (int a = 0; a < 3; ++a) od2[a] = o[a] + m * sg * n_[a];
      }
      float tr = off ? t_c : t_c + step;
      if (hit) nxt = o_settle(S, nx0, od2, d, tr, unit_x, step + step, &moved);
      else nxt = nx0, moved = 0;
    }
    int item = !is_own ? u_in : vi;
    int after = o_cls(S, hit ? nxt : v);
    int zl = hit && it > 0 && (z_in || t_c - pz_tin <= O_ZERO_STEP_BANDS * band);
    int touched = zl;
    if (!zl && hit && it > 0 && v < OUT && after != cur) {
      float xm[3];
      float tm = 0.5f * (pz_tin + t_c);
      for (int a = 0; a < 3; ++a) xm[a] = o[a] + tm * d[a];
      touched = !o_holds_point(S, vi, xm);
    }
    if (touched) cur = o_cls(S, pz_vin);
    int v_b = touched ? pz_vin : v;
    int vis = hit && after != cur;
    int inv = hit && !vis;
    int zc = (inv && t_c - t_lo <= O_ZERO_STEP_BANDS * band) ? pz_zc + 1 : 0;
    if (inv && pz_tp0 == O_HUGE) pz_tp0 = t_c;
    if (inv) pz_tp1 = t_c;
    pz_np += inv;
    if (inv) pz_vend = nxt;
    pz_hit = hit;
    if (inv && t_c <= s_at) pz_vat = nxt;
    pz_zc = zc;
    int n_vin = hit ? v_b : pz_vin;
    float n_tin = hit ? t_c : pz_tin;
    pz_vin = n_vin;
    pz_tin = n_tin;
    done = !hit || vis || zc >= O_ZSBP;
    if (hit) { rec_t = t_c; rec_item = item; rec_leaf = l_in; rec_face = f_in; rec_zero = z_in; rec_vb = v_b; rec_vis = vis; }
    t_lo = moved ? t_c + step : t_c;
    if (hit) v = nxt;
    last_ = item;
    it += 1;
    if (hit) cur = after;
    if (++guard > 4096) break;
  }
  /* _finish */
  OQuery q;
  float bt = rec_t;
  int bi = rec_item, bl = rec_leaf, bf = rec_face, zero = rec_zero, vb = rec_vb;
  int vis_end = rec_vis;
  int cont = !vis_end && pz_hit && pz_zc >= O_ZSBP;
  int hit = (vis_end || cont) && bt < t_max;
  float px = bt < O_HUGE ? bt : 0.0f;
  float xh[3] = {o[0] + px * d[0], o[1] + px * d[1], o[2] + px * d[2]};
  float g[3];
  o_hit_grad(S, bi, bl > 0 ? bl : 0, bf, xh, g);
  float gn = o_safe_norm(g);
  float nrm[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
  float fb[3] = {-d[0], -d[1], -d[2]};
  if (sn) {
    int sat = hit && zero && bl < 0 && kn0 && bt <= 0.0f;
    if (sat) {
      float sl = o_safe_norm(sn);
      fb[0] = sn[0] / sl; fb[1] = sn[1] / sl; fb[2] = sn[2] / sl;
    }
  }
  if (!(hit && bl >= 0)) { nrm[0] = fb[0]; nrm[1] = fb[1]; nrm[2] = fb[2]; }
  float gd = o_dot(g, d);
  int entry = bi != vb;
  q.srf = hit ? o_srf_pack(S, bi, bl, bf, entry ? gd < 0.0f : gd > 0.0f, entry) : -1;
  if (nrm[0] * d[0] + nrm[1] * d[1] + nrm[2] * d[2] > 0.0f) { nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2]; }
  vb = hit ? vb : pz_vend;
  q.t = hit ? bt : t_max;
  q.hit = hit;
  q.cont = cont;
  q.vol_after = hit ? v : vol;
  q.vol_before = vb;
  q.vol_start = vol;
  q.cls_before = o_cls(S, vb);
  q.cls_start = cls0;
  q.cls_after = hit ? cur : o_cls(S, vb);
  q.normal[0] = nrm[0]; q.normal[1] = nrm[1]; q.normal[2] = nrm[2];
  q.item = hit ? bi : -1;
  q.leaf = bl;
  q.face = bf;
  q.zero = hit && zero;
  q.t_pass0 = pz_tp0;
  q.t_pass1 = pz_tp1;
  q.n_pass = pz_np;
  q.vol_at = pz_vat;
  q.rounds = it;
  return q;
}

#endif
