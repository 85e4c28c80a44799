/*
 * ORACLE (test infrastructure): the navigator's body in the precision NF (float or double), included once per
 * precision by geom.h inside a namespace of its own (onav32, onav64) that defines NF and the O_NAV_* array selectors.
 * Every coordinate, frame, box, leaf coefficient, root, interval and band is NF (src/lumen/rules/navigation.py:96
 * Precision); constants are the NF value of the reference's own (float32 literals in float, float64 literals in
 * double, as the reference's self.F(c)). No include guard: included twice.
 */
static const NF N_HUGE = NK(1e30);
static const NF N_BIG = NK(1e29);
static const NF N_EPS = sizeof(NF) == 4 ? (NF)1.1920928955078125e-7f : (NF)2.220446049250313080847e-16;
static const NF N_BAND_ULPS_EPS = 8.0f * N_EPS; /* BAND_ULPS (8) eps of the precision (tolerances.py:76) */
static const NF N_BAND_FLOOR = NK(1e-9);
static const NF N_DIVISOR_FLOOR = NK(1e-30);
static const NF N_TINY_DIR = NK(1e-30);
static const NF N_LINEAR_REL = NK(1e-12);
static const NF N_PARALLEL = NK(1e-12);
static const NF N_TINY_NORMAL = (NF)1.17549435e-38f; /* float32's smallest normal in either precision (safe.py:52) */
static const int N_BISECT = sizeof(NF) == 4 ? 40 : 64; /* BISECT_F32, BISECT_F64 (tolerances.py:93) */
static const NF N_TORUS_AXIAL = NK(1e-12);
static const NF N_TORUS_PAD_REL = NK(1e-4);
static const NF O_TORUS_BRACKET_ULPS = 64.0f;

static inline NF o_dot(const NF* a, const NF* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline NF o_maxabs3(const NF* a) {
  NF m = n_abs(a[0]);
  if (n_abs(a[1]) > m) m = n_abs(a[1]);
  if (n_abs(a[2]) > m) m = n_abs(a[2]);
  return m;
}
static inline NF o_min(NF a, NF b) { return a < b ? a : b; }
static inline NF o_max(NF a, NF b) { return a > b ? a : b; }
/* band(scale) = BAND_ULPS eps scale + BAND_FLOOR (src/lumen/rules/navigation.py:121) */
static inline NF o_band(NF scale) { return N_BAND_ULPS_EPS * scale + N_BAND_FLOOR; }
static inline NF o_safe_norm(const NF* v) { return n_sqrt(o_max(o_dot(v, v), N_TINY_NORMAL)); }
static inline const NF* o_vfn(const OScene* S, int v) { return O_NAV_VOL(S) + (size_t)v * LUMEN_VOL_F; }
static inline const NF* o_lfn(const OScene* S, int g) { return O_NAV_LEAF(S) + (size_t)g * LUMEN_LEAF_F; }
static inline const NF* o_pln(const OScene* S, int q) { return O_NAV_PLANE(S) + (size_t)q * LUMEN_PLANE_F; }

/* the ray in volume i's frame: local = R^T (x - t) (navigate.py:151) */
static inline void o_to_local_pt(const OScene* S, int i, const NF* x, NF* xl) {
  const NF* f = o_vfn(S, i);
  const NF* R = f + LUMEN_VF_R;
  NF v0 = x[0] - f[LUMEN_VF_T], v1 = x[1] - f[LUMEN_VF_T + 1], v2 = x[2] - f[LUMEN_VF_T + 2];
  for (int a = 0; a < 3; ++a) xl[a] = R[a] * v0 + R[3 + a] * v1 + R[6 + a] * v2;
}
static inline void o_to_local_dir(const OScene* S, int i, const NF* d, NF* dl) {
  const NF* R = o_vfn(S, i) + LUMEN_VF_R;
  for (int a = 0; a < 3; ++a) dl[a] = R[a] * d[0] + R[3 + a] * d[1] + R[6 + a] * d[2];
}
static inline void o_to_world_dir(const OScene* S, int i, const NF* g, NF* gw) {
  const NF* R = o_vfn(S, i) + LUMEN_VF_R;
  for (int a = 0; a < 3; ++a) gw[a] = R[3 * a] * g[0] + R[3 * a + 1] * g[1] + R[3 * a + 2] * g[2];
}

/* ------------------------------------------------------------------------------- one leaf along a line (csg.py) */
typedef struct OIv { NF lo0, hi0; int f_lo0, f_hi0; NF lo1, hi1; int f_lo1, f_hi1; } OIv;

static inline void o_Av(const NF* A, const NF* v, NF* out) {
  for (int a = 0; a < 3; ++a) out[a] = A[3 * a] * v[0] + A[3 * a + 1] * v[1] + A[3 * a + 2] * v[2];
}

/* quadric pieces [L0, R0], [L1, inf) along y + t d (leaf_kernels.py:81 quad_line, :41 _roots, :60 _pieces) */
static inline void o_quad_line(const NF* lf, const NF* y, const NF* d, NF* L0, NF* R0, int* L0q,
                               int* R0q, NF* L1, NF* R1) {
  const NF* A = lf + LUMEN_LF_A;
  const NF* b = lf + LUMEN_LF_B;
  NF c = lf[LUMEN_LF_C], sa = lf[LUMEN_LF_SA];
  const NF inf = N_HUGE;
  NF t_o = -o_dot(y, d);
  NF y0[3] = {y[0] + t_o * d[0], y[1] + t_o * d[1], y[2] + t_o * d[2]};
  NF Ad[3];
  o_Av(A, d, Ad);
  NF alpha = o_dot(Ad, d);
  int lin = n_abs(alpha) < o_max(N_LINEAR_REL * sa, N_DIVISOR_FLOOR);
  NF bdd = o_dot(b, d);
  NF Ay0[3];
  o_Av(A, y0, Ay0);
  NF beta0 = o_dot(Ay0, d) + bdd;
  NF gam0 = (o_dot(y0, Ay0) + 2.0f * o_dot(b, y0)) + c;
  int near_ = !lin && (alpha * gam0 > 0.5f * beta0 * beta0);
  NF t_c = t_o + (near_ ? -beta0 / alpha : 0.0f);
  NF yc[3] = {y[0] + t_c * d[0], y[1] + t_c * d[1], y[2] + t_c * d[2]};
  NF Ayc[3];
  o_Av(A, yc, Ayc);
  NF beta = o_dot(Ayc, d) + bdd;
  NF gam = (o_dot(yc, Ayc) + 2.0f * o_dot(b, yc)) + c;
  /* _roots */
  NF D = beta * beta - alpha * gam;
  int Dpos = D > O_TANGENT_ULPS * N_EPS * (beta * beta + n_abs(alpha * gam));
  NF sD = n_sqrt(Dpos ? D : 1.0f);
  NF sgn = beta >= 0.0f ? 1.0f : -1.0f;
  NF s_ = -(beta + sgn * (Dpos ? sD : 0.0f));
  int s_ok = n_abs(s_) > N_DIVISOR_FLOOR;
  NF r1 = lin ? inf : s_ / alpha;
  NF r2 = s_ok ? gam / s_ : 0.0f;
  NF rmin = o_min(r1, r2) + t_c;
  NF rmax = o_max(r1, r2) + t_c;
  int b_small = n_abs(beta) < N_DIVISOR_FLOOR;
  NF tl = t_c - gam / (b_small ? 1.0f : 2.0f * beta);
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

static inline NF o_torus_g(NF R, NF r, const NF* oc, const NF* d, NF s) {
  const NF p[3] = {oc[0] + s * d[0], oc[1] + s * d[1], oc[2] + s * d[2]};
  const NF rho2 = p[0] * p[0] + p[1] * p[1];
  const NF dr = (rho2 - R * R) / (n_sqrt(o_max(rho2, 0.0f)) + R);
  return dr * dr + p[2] * p[2] - r * r;
}
static inline NF o_torus_dg(NF R, const NF* oc, const NF* d, NF s) {
  const NF p[3] = {oc[0] + s * d[0], oc[1] + s * d[1], oc[2] + s * d[2]};
  const NF rho2 = p[0] * p[0] + p[1] * p[1];
  const NF rho = n_sqrt(o_max(rho2, N_TINY_NORMAL));
  const NF dr = (rho2 - R * R) / (rho + R);
  return 2.0f * dr * ((p[0] * d[0] + p[1] * d[1]) / rho) + 2.0f * p[2] * d[2];
}
static inline int o_torus_meets(NF R, NF r, const NF* o, const NF* d) {
  const NF Rb = (R + r) * (1.0f + N_TORUS_PAD_REL);
  const NF bb = o[0] * d[0] + o[1] * d[1] + o[2] * d[2];
  const NF disc = Rb * Rb - (o[0] * o[0] + o[1] * o[1] + o[2] * o[2] - bb * bb);
  const NF sq = n_sqrt(o_max(disc, 0.0f));
  NF lo = -bb - sq, hi = -bb + sq;
  int meet = disc > 0.0f && lo <= hi;
  const NF pad = N_TORUS_PAD_REL * (R + r), rz = r + pad;
  const int flat = n_abs(d[2]) < N_PARALLEL;
  const NF iz = 1.0f / (flat ? 1.0f : d[2]);
  if (!flat) {
    const NF za = (-rz - o[2]) * iz, zb = (rz - o[2]) * iz;
    lo = o_max(lo, o_min(za, zb));
    hi = o_min(hi, o_max(za, zb));
  }
  meet = meet && lo <= hi && (!flat || n_abs(o[2]) <= rz);
  const NF qa = d[0] * d[0] + d[1] * d[1], qb = o[0] * d[0] + o[1] * d[1], qc = o[0] * o[0] + o[1] * o[1];
  const NF sm = o_min(o_max(-qb / (qa > N_PARALLEL ? qa : 1.0f), lo), hi);
  const NF near2 = qa > N_PARALLEL ? qa * sm * sm + 2.0f * qb * sm + qc : qc;
  const NF far2 = o_max(qa * lo * lo + 2.0f * qb * lo + qc, qa * hi * hi + 2.0f * qb * hi + qc);
  const NF rout = R + r + pad, rin = o_max(R - r - pad, 0.0f);
  return meet && near2 <= rout * rout && far2 >= rin * rin;
}
static inline void o_torus_set(NF R, NF r, const NF* o, const NF* d, NF* lo, NF* hi) {
  const NF tc = -((o[0] * d[0] + o[1] * d[1]) + o[2] * d[2]);
  const NF oc[3] = {o[0] + tc * d[0], o[1] + tc * d[1], o[2] + tc * d[2]};
  const NF q0 = (oc[0] * oc[0] + oc[1] * oc[1]) + oc[2] * oc[2];
  const NF Rb = (R + r) * (1.0f + O_TORUS_BRACKET_ULPS * N_EPS);
  const NF b0 = (oc[0] * d[0] + oc[1] * d[1]) + oc[2] * d[2];
  const NF disc = Rb * Rb - q0 + b0 * b0;
  const int in_ball = disc > 0.0f;
  const NF sq = n_sqrt(in_ball ? disc : 1.0f);
  const NF s0 = -b0 - sq, s1 = -b0 + sq;
  const NF a = d[0] * d[0] + d[1] * d[1];
  const NF bxy = oc[0] * d[0] + oc[1] * d[1];
  const NF cxy = oc[0] * oc[0] + oc[1] * oc[1];
  const int off_axis = a > N_TORUS_AXIAL;
  const NF as = off_axis ? a : 1.0f;
  const NF sv = off_axis ? -bxy / as : 0.0f;
  const NF m2 = o_max(off_axis ? cxy - bxy * bxy / as : cxy, 0.0f);
  const NF cr = n_cbrt(R * a * m2);
  const NF w2 = (cr * cr - m2) / as;
  const NF w = n_sqrt(off_axis && w2 > 0.0f ? w2 : 0.0f);
  const NF p1 = o_min(o_max(sv - w, s0), s1), p2 = o_min(o_max(sv + w, s0), s1);
  const NF a0[3] = {s0, p1, p2}, a1[3] = {p1, p2, s1};
  NF ex[3];
  for (int k = 0; k < 3; ++k) { /* g' rises through its minima, falls through its maximum */
    NF l = a0[k], h = a1[k];
    for (int it = 0; it < N_BISECT; ++it) {
      const NF m = 0.5f * (l + h);
      const NF gp = o_torus_dg(R, oc, d, m);
      if (k == 1 ? gp > 0.0f : gp < 0.0f) l = m; else h = m;
    }
    ex[k] = 0.5f * (l + h);
  }
  const NF kn[7] = {s0, ex[0], p1, ex[1], p2, ex[2], s1};
  NF roots[6];
  for (int k = 0; k < 6; ++k) {
    const int in_l = o_torus_g(R, r, oc, d, kn[k]) <= 0.0f, in_r = o_torus_g(R, r, oc, d, kn[k + 1]) <= 0.0f;
    NF l = kn[k], h = kn[k + 1];
    for (int it = 0; it < N_BISECT; ++it) {
      const NF m = 0.5f * (l + h);
      if ((o_torus_g(R, r, oc, d, m) <= 0.0f) == in_l) l = m; else h = m;
    }
    roots[k] = (in_l != in_r && kn[k + 1] > kn[k] && in_ball) ? 0.5f * (l + h) + tc : N_HUGE;
  }
  std::sort(roots, roots + 6);
  const int ok0 = roots[1] < N_BIG, ok1 = roots[3] < N_BIG;
  lo[0] = ok0 ? roots[0] : N_HUGE; hi[0] = ok0 ? roots[1] : N_HUGE;
  lo[1] = ok1 ? roots[2] : N_HUGE; hi[1] = ok1 ? roots[3] : N_HUGE;
}
/* a torus leaf along o + t d (kind frame): canonical frame u = M (x - og), the unit ray, the roots scaled back
   (csg.py:207 _t_iv) */
static inline void o_torus_line(const NF* lf, const NF* o, const NF* d, NF* L0, NF* R0, NF* L1,
                                NF* R1) {
  const NF* M = lf + LUMEN_LF_A;
  const NF R = lf[LUMEN_LF_B], r = lf[LUMEN_LF_B + 1];
  const NF xl[3] = {o[0] - lf[0], o[1] - lf[1], o[2] - lf[2]};
  NF ou[3], dl[3];
  o_Av(M, xl, ou);
  o_Av(M, d, dl);
  const NF kk = n_sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
  const NF du[3] = {dl[0] / kk, dl[1] / kk, dl[2] / kk};
  NF lo[2] = {N_HUGE, N_HUGE}, hi[2] = {N_HUGE, N_HUGE};
  if (o_torus_meets(R, r, ou, du)) o_torus_set(R, r, ou, du, lo, hi);
  *L0 = n_abs(lo[0]) < N_BIG ? lo[0] / kk : lo[0];
  *R0 = n_abs(hi[0]) < N_BIG ? hi[0] / kk : hi[0];
  *L1 = n_abs(lo[1]) < N_BIG ? lo[1] / kk : lo[1];
  *R1 = n_abs(hi[1]) < N_BIG ? hi[1] / kk : hi[1];
}

static inline OIv o_leaf_iv(const OScene* S, int g, const NF* o, const NF* d) {
  const NF* lf = o_lfn(S, g);
  const int32_t* li = o_li(S, g);
  const NF inf = N_HUGE;
  NF y[3] = {o[0] - lf[LUMEN_LF_OQ], o[1] - lf[LUMEN_LF_OQ + 1], o[2] - lf[LUMEN_LF_OQ + 2]};
  NF ol[3] = {o[0] - lf[LUMEN_LF_OG], o[1] - lf[LUMEN_LF_OG + 1], o[2] - lf[LUMEN_LF_OG + 2]};
  NF t0p = -inf, t1p = inf;
  int f0p = -1, f1p = -1, ep = 0;
  for (int k = 0; k < li[2]; ++k) {
    const NF* pl = o_pln(S, li[1] + k);
    NF nd = pl[0] * d[0] + pl[1] * d[1] + pl[2] * d[2];
    NF rhs = pl[3] - (pl[0] * ol[0] + pl[1] * ol[1] + pl[2] * ol[2]);
    int par = n_abs(nd) < N_PARALLEL;
    NF tp = rhs / (par ? 1.0f : nd);
    NF ent = nd < -N_PARALLEL ? tp : -inf;
    NF ext = nd > N_PARALLEL ? tp : inf;
    if (ent > t0p) { t0p = ent; f0p = k + 1; }
    if (ext < t1p) { t1p = ext; f1p = k + 1; }
    ep = ep || (par && rhs < 0.0f);
  }
  int has_q = li[0] == 1;
  NF L0 = -inf, R0 = inf, L1 = inf, R1 = -inf;
  int L0q = 0, R0q = 0;
  if (has_q) o_quad_line(lf, y, d, &L0, &R0, &L0q, &R0q, &L1, &R1);
  if (li[0] == 2) {
    o_torus_line(lf, o, d, &L0, &R0, &L1, &R1);
    L0q = R0q = 1;
  }
  OIv r;
  /* clip each piece by the slab */
  {
    NF lo = o_max(L0, t0p), hi = o_min(R0, t1p);
    int flo = L0 > t0p ? (L0q ? 0 : f0p) : f0p;
    int fhi = R0 < t1p ? (R0q ? 0 : f1p) : f1p;
    int ok = lo < hi && !ep;
    r.lo0 = ok ? lo : inf; r.hi0 = ok ? hi : inf; r.f_lo0 = ok ? flo : -1; r.f_hi0 = ok ? fhi : -1;
  }
  {
    NF lo = o_max(L1, t0p), hi = o_min(R1, t1p);
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
static inline int o_inside_leaf(const OScene* S, int g, const NF* x) {
  const NF* lf = o_lfn(S, g);
  const int32_t* li = o_li(S, g);
  NF xl[3] = {x[0] - lf[LUMEN_LF_OG], x[1] - lf[LUMEN_LF_OG + 1], x[2] - lf[LUMEN_LF_OG + 2]};
  NF y[3] = {x[0] - lf[LUMEN_LF_OQ], x[1] - lf[LUMEN_LF_OQ + 1], x[2] - lf[LUMEN_LF_OQ + 2]};
  int pl = 1;
  for (int k = 0; k < li[2]; ++k) {
    const NF* p = o_pln(S, li[1] + k);
    pl = pl && (p[0] * xl[0] + p[1] * xl[1] + p[2] * xl[2] <= p[3]);
  }
  if (li[0] == 2) { /* the torus reads no planes: (rho - R)^2 + z^2 <= r^2 */
    NF u[3];
    o_Av(lf + LUMEN_LF_A, xl, u);
    const NF dr = n_sqrt(u[0] * u[0] + u[1] * u[1]) - lf[LUMEN_LF_B];
    return dr * dr + u[2] * u[2] <= lf[LUMEN_LF_B + 1] * lf[LUMEN_LF_B + 1];
  }
  if (li[0] != 1) return pl;
  NF Ay[3];
  o_Av(lf + LUMEN_LF_A, y, Ay);
  const NF* b = lf + LUMEN_LF_B;
  NF qv = (o_dot(y, Ay) + 2.0f * (b[0] * y[0] + b[1] * y[1] + b[2] * y[2])) + lf[LUMEN_LF_C];
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

typedef struct OPtCtx { const OScene* S; int l0; const NF* x; } OPtCtx;
static inline int o_member_pt(void* c, int l) {
  OPtCtx* p = (OPtCtx*)c;
  return o_inside_leaf(p->S, p->l0 + l, p->x);
}
/* whether the kind holds the point x (csg.py:341 inside) */
static inline int o_inside_kind(const OScene* S, int kind, const NF* x) {
  OPtCtx c = {S, o_ki(S, kind)[0], x};
  return o_program(S, kind, o_member_pt, &c);
}

/* ------------------------------------------------------------------- first_change (csg.py:369-449), one kind */
typedef struct OScan {
  const OScene* S;
  int kind, nl;
  OIv iv[LUMEN_MAX_LEAVES]; /* every leaf's intervals along the ray (quadric leaves do not depend on the window) */
  NF xa;                  /* max |o| (kind frame), the band's scale */
  NF t1;
  int want;                  /* -1 any change, 1 the first entry, 0 the first exit */
  int has_init, init_known, init_inside;
  int has_skip, skip_leaf, skip_face, skip_entry; NF skip_thi;
  int has_on, on_leaf, on_inside; NF on_tend;
  /* the membership override in force at a probe (on_face with its running end) */
  NF hend;
  NF probe_t;
} OScan;

static inline NF o_scan_band(const OScan* s, NF t) { return o_band(s->xa + n_abs(t)); }

static inline int o_member_iv(void* c, int l) {
  OScan* s = (OScan*)c;
  const OIv* v = &s->iv[l];
  NF t = s->probe_t;
  int m = (v->lo0 <= t && t < v->hi0) || (v->lo1 <= t && t < v->hi1);
  if (s->has_on && l == s->on_leaf && t < s->hend) m = s->on_inside;
  return m;
}
/* the solid's membership just after o + t d (csg.py:346 _mem_at) */
static inline int o_mem_at(OScan* s, NF t, int use_on) {
  int save = s->has_on;
  s->has_on = save && use_on;
  s->probe_t = t;
  int r = o_program(s->S, s->kind, o_member_iv, s);
  s->has_on = save;
  return r;
}

static inline void o_scan_init(OScan* s, const OScene* S, int kind, const NF* o, const NF* d, NF t1) {
  s->S = S;
  s->kind = kind;
  const int32_t* k = o_ki(S, kind);
  s->nl = k[1];
  for (int l = 0; l < s->nl; ++l) s->iv[l] = o_leaf_iv(S, k[0] + l, o, d);
  s->xa = o_max(o_max(n_abs(o[0]), n_abs(o[1])), n_abs(o[2]));
  s->t1 = t1;
  s->want = -1;
  s->has_init = s->has_skip = s->has_on = 0;
  s->hend = -N_HUGE;
}

typedef struct OFirst { int hit; NF t; int inside, leaf, face; } OFirst;
typedef struct OFc { int hit; NF t; int inside, leaf, face, inside0; OFirst first; } OFc;

/* the nearest leaf endpoint after t_cur (<= t1): csg.py:369 _nearest */
static inline void o_nearest(const OScan* s, NF t_cur, NF* e1o, int* lbo, int* fco, int* eko) {
  NF e1 = N_HUGE;
  int lb = -1, fc = -1, ek = 0;
  for (int l = 0; l < s->nl; ++l) {
    const OIv* v = &s->iv[l];
    NF eps_[4] = {v->lo0, v->hi0, v->lo1, v->hi1};
    int fps[4] = {v->f_lo0, v->f_hi0, v->f_lo1, v->f_hi1};
    int ens[4] = {1, 0, 1, 0};
    for (int j = 0; j < 4; ++j) {
      NF ep = eps_[j];
      int ok = n_abs(ep) < N_BIG && ep <= s->t1 && ep > t_cur && ep < e1;
      if (s->has_skip)
        ok = ok && !(l == s->skip_leaf && fps[j] == s->skip_face && s->skip_entry == ens[j] && ep < s->skip_thi);
      if (ok) { e1 = ep; lb = l; fc = fps[j]; ek = ens[j]; }
    }
  }
  *e1o = e1; *lbo = lb; *fco = fc; *eko = ek;
}

/* the first change of the kind's membership in (t0, t1] (csg.py:417 first_change) */
static inline OFc o_first_change(OScan* s, NF t0) {
  NF t_cur = t0;
  int done = 0, now = 0, lb_h = -1, fc_h = -1, now0 = 0, it = 0;
  OFirst fs = {0, N_HUGE, 0, -1, -1};
  s->hend = s->has_on ? s->on_tend : -N_HUGE;
  while (!done && t_cur < N_HUGE && it < O_MAX_SCAN_PER_LEAF * s->nl + O_MAX_SCAN_EXTRA) {
    int first = it == 0;
    NF e; int lb, fc, ek;
    if (first) { e = t0; lb = -1; fc = -1; ek = 0; }
    else o_nearest(s, t_cur, &e, &lb, &fc, &ek);
    int has = first || e < N_HUGE;
    NF tp = first ? t0 : e + o_scan_band(s, e);
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
    NF t_nx = first ? t0 : (vis ? e : (has ? tp : N_HUGE));
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
static inline void o_leaf_grad(const OScene* S, int kind, int leaf, int face, const NF* x, NF* g) {
  int gi = o_ki(S, kind)[0] + (leaf > 0 ? leaf : 0);
  const NF* lf = o_lfn(S, gi);
  const int32_t* li = o_li(S, gi);
  if (face >= 1) {
    const NF* p = o_pln(S, li[1] + face - 1);
    g[0] = p[0]; g[1] = p[1]; g[2] = p[2];
    return;
  }
  if (li[0] == 2) { /* M^T ((rho - R) / rho u_x, (rho - R) / rho u_y, u_z) */
    const NF* M = lf + LUMEN_LF_A;
    const NF xl[3] = {x[0] - lf[0], x[1] - lf[1], x[2] - lf[2]};
    NF u[3];
    o_Av(M, xl, u);
    const NF rho = n_sqrt(o_max(u[0] * u[0] + u[1] * u[1], N_DIVISOR_FLOOR));
    const NF k = (rho - lf[LUMEN_LF_B]) / rho;
    const NF gu[3] = {k * u[0], k * u[1], u[2]};
    for (int a = 0; a < 3; ++a) g[a] = (M[a] * gu[0] + M[3 + a] * gu[1]) + M[6 + a] * gu[2];
    return;
  }
  NF y[3] = {x[0] - lf[LUMEN_LF_OQ], x[1] - lf[LUMEN_LF_OQ + 1], x[2] - lf[LUMEN_LF_OQ + 2]};
  NF Ay[3];
  o_Av(lf + LUMEN_LF_A, y, Ay);
  const NF* b = lf + LUMEN_LF_B;
  for (int a = 0; a < 3; ++a) g[a] = 2.0f * (Ay[a] + b[a]);
}
/* |f| / |grad f| of a leaf's face at x (kind frame): csg.py:470 leaf_dist */
static inline NF o_leaf_dist(const OScene* S, int kind, int leaf, int face, const NF* x) {
  int gi = o_ki(S, kind)[0] + (leaf > 0 ? leaf : 0);
  const NF* lf = o_lfn(S, gi);
  const int32_t* li = o_li(S, gi);
  NF f;
  if (face >= 1) {
    const NF* p = o_pln(S, li[1] + face - 1);
    NF xl[3] = {x[0] - lf[LUMEN_LF_OG], x[1] - lf[LUMEN_LF_OG + 1], x[2] - lf[LUMEN_LF_OG + 2]};
    f = p[0] * xl[0] + p[1] * xl[1] + p[2] * xl[2] - p[3];
  } else if (li[0] == 2) {
    const NF xl[3] = {x[0] - lf[0], x[1] - lf[1], x[2] - lf[2]};
    NF u[3];
    o_Av(lf + LUMEN_LF_A, xl, u);
    const NF dr = n_sqrt(u[0] * u[0] + u[1] * u[1]) - lf[LUMEN_LF_B], r = lf[LUMEN_LF_B + 1];
    f = 0.5f * (dr * dr + u[2] * u[2] - r * r);
  } else {
    NF y[3] = {x[0] - lf[LUMEN_LF_OQ], x[1] - lf[LUMEN_LF_OQ + 1], x[2] - lf[LUMEN_LF_OQ + 2]};
    NF Ay[3];
    o_Av(lf + LUMEN_LF_A, y, Ay);
    const NF* b = lf + LUMEN_LF_B;
    f = (o_dot(y, Ay) + 2.0f * (b[0] * y[0] + b[1] * y[1] + b[2] * y[2])) + lf[LUMEN_LF_C];
  }
  NF g[3];
  o_leaf_grad(S, kind, leaf, face, x, g);
  return n_abs(f) / o_safe_norm(g);
}

/* world gradient / face distance of volume i's leaf face at the world point x (surface_id.py:91 hit_grad, :100) */
static inline void o_hit_grad(const OScene* S, int item, int leaf, int face, const NF* x, NF* gw) {
  int i = item < 0 ? 0 : (item > S->n - 1 ? S->n - 1 : item);
  NF xl[3], g[3];
  o_to_local_pt(S, i, x, xl);
  o_leaf_grad(S, o_vi(S, i)[LUMEN_VI_KIND], leaf, face, xl, g);
  o_to_world_dir(S, i, g, gw);
}
static inline NF o_face_dist(const OScene* S, int item, int leaf, int face, const NF* x) {
  int i = item < 0 ? 0 : (item > S->n - 1 ? S->n - 1 : item);
  NF xl[3];
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
static inline int o_holds_point(const OScene* S, int i, const NF* x) {
  NF xl[3];
  o_to_local_pt(S, i, x, xl);
  return o_inside_kind(S, o_vi(S, i)[LUMEN_VI_KIND], xl);
}
/* whether volume i holds the ray just after t (navigate.py:163 ray_holds, csg.py:362 inside_ray) */
static inline int o_ray_holds(const OScene* S, int i, const NF* od, const NF* dd, NF t) {
  NF ol[3], dl[3];
  o_to_local_pt(S, i, od, ol);
  o_to_local_dir(S, i, dd, dl);
  OScan s;
  o_scan_init(&s, S, o_vi(S, i)[LUMEN_VI_KIND], ol, dl, N_HUGE);
  return o_mem_at(&s, t, 0);
}
/* whether x lies in volume i's world box padded by pad */
static inline int o_box_holds(const OScene* S, int i, const NF* x, NF pad) {
  const NF* f = o_vfn(S, i);
  for (int a = 0; a < 3; ++a)
    if (!(f[LUMEN_VF_LO + a] - pad <= x[a] && x[a] <= f[LUMEN_VF_HI + a] + pad)) return 0;
  return 1;
}

/* Geant4's LevelLocate: the first in the rule's order (navigation.py:150 level_locate_wins) */
static inline int o_level_wins(const OScene* S, int item, int found, int excl) {
  return (found < 0 || o_rank(S, item) > o_rank(S, found)) && item != excl && item < S->n;
}

/* the daughter of v holding the point x, or -1 (navigate.py:215 _find) */
static inline int o_find(const OScene* S, int v, const NF* x) {
  const int32_t* vi = o_vi(S, v);
  int g = -1;
  for (int k = 0; k < vi[LUMEN_VI_CN]; ++k) {
    int i = S->D->cand[vi[LUMEN_VI_C0] + k];
    if (!o_box_holds(S, i, x, 0.0f)) continue;
    if (o_level_wins(S, i, g, -1) && !o_is_anc(S, i, v) && o_holds_point(S, i, x)) g = i;
  }
  return g;
}
/* the deepest volume holding x (n: outside every volume) (navigate.py:226 locate) */
static inline int o_locate(const OScene* S, const NF* x) {
  int v = S->n;
  for (;;) {
    int f = o_find(S, v, x);
    if (f < 0) return v;
    v = f;
  }
}
/* the daughter of v (other than excl) holding the ray just after t (navigate.py:243 _find_ray) */
static inline int o_find_ray(const OScene* S, int v, const NF* od, const NF* dd, NF t, int excl, NF pad) {
  const int32_t* vi = o_vi(S, v);
  NF x[3] = {od[0] + t * dd[0], od[1] + t * dd[1], od[2] + t * dd[2]};
  int g = -1;
  for (int k = 0; k < vi[LUMEN_VI_CN]; ++k) {
    int i = S->D->cand[vi[LUMEN_VI_C0] + k];
    if (!o_box_holds(S, i, x, pad)) continue;
    if (o_level_wins(S, i, g, excl) && !o_is_anc(S, i, v) && o_ray_holds(S, i, od, dd, t)) g = i;
  }
  return g;
}
/* up while v does not hold the ray just after t, then down (navigate.py:254 _settle) */
static inline int o_settle(const OScene* S, int v, const NF* od, const NF* dd, NF t, int crossed, NF pad,
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
typedef struct OSide { int known, leaf, face; NF s; int entry; } OSide;
typedef struct OBest { NF t; int item, leaf, face, zero, own; } OBest;
typedef struct OCtx {
  int v;
  const NF *od, *dd;
  NF t_lo, t_bound;
  int last;
  NF band;
  OSide sd;
} OCtx;

/* the on-face rule (navigate.py:334 _on_face) */
static inline int o_on_face(const OScene* S, const OCtx* c, int i, const OFirst* fr, int kn_i) {
  NF dt = fr->t - c->t_lo;
  NF lim = O_K_ON * c->band;
  int far_ = 0;
  if (!kn_i && fr->hit && dt >= lim && dt < O_GRAZE * lim) {
    NF x0[3] = {c->od[0] + c->t_lo * c->dd[0], c->od[1] + c->t_lo * c->dd[1], c->od[2] + c->t_lo * c->dd[2]};
    NF xc[3] = {c->od[0] + fr->t * c->dd[0], c->od[1] + fr->t * c->dd[1], c->od[2] + fr->t * c->dd[2]};
    int lf = fr->leaf > 0 ? fr->leaf : 0;
    NF g0[3], gc[3];
    o_hit_grad(S, i, lf, fr->face, x0, g0);
    o_hit_grad(S, i, lf, fr->face, xc, gc);
    NF s0 = o_dot(g0, c->dd) / o_safe_norm(g0);
    int other_way = (s0 * o_dot(gc, c->dd) < 0.0f) && (n_abs(s0) > 1.0f / O_GRAZE);
    far_ = (o_face_dist(S, i, lf, fr->face, x0) < lim) && !other_way;
  }
  return !kn_i && fr->hit && (dt < lim || far_);
}

static inline int o_entry_wins(const OScene* S, NF t, int item, const OBest* b) {
  return t < b->t || (t == b->t && (b->own || o_rank(S, item) > o_rank(S, b->item)));
}

/* the best event after volume i: own its first exit, a daughter its first entry (navigate.py:357-416) */
static inline OBest o_unit_visit(const OScene* S, const OCtx* c, int i, OBest b, int is_own) {
  /* an ancestor the volume is not proved inside (a protrusion clip): its first exit from a start inside it, when
     earlier than every other event (navigate.py:376 _unit_visit) */
  const int clip = !is_own && o_is_anc(S, i, c->v);
  const int own = is_own;
  is_own = is_own || clip;
  const OSide* sd = &c->sd;
  NF bnd = c->t_bound + c->band; /* the scan's window: the query's bound (order-independent) */
  NF ol[3], dl[3];
  o_to_local_pt(S, i, c->od, ol);
  o_to_local_dir(S, i, c->dd, dl);
  int kn_i = sd->known && i == c->last;
  NF t_on = c->t_lo + O_K_ON * c->band / o_max(n_abs(sd->s), 1.0f / O_GRAZE);
  int lf_on = kn_i ? sd->leaf : -2;
  OScan s;
  o_scan_init(&s, S, o_vi(S, i)[LUMEN_VI_KIND], ol, dl, bnd);
  s.want = is_own ? 0 : 1;
  s.has_init = 1; s.init_known = kn_i; s.init_inside = is_own;
  s.has_skip = 1; s.skip_leaf = lf_on; s.skip_face = sd->face; s.skip_entry = sd->entry; s.skip_thi = N_HUGE;
  s.has_on = 1; s.on_leaf = lf_on; s.on_inside = sd->entry; s.on_tend = t_on;
  OFc r = o_first_change(&s, c->t_lo);
  int h = r.hit, lf = r.leaf, f = r.face;
  NF t = r.t;
  int on = o_on_face(S, c, i, &r.first, kn_i);
  int by_s = kn_i && (is_own ? sd->s > 0.0f : sd->s < 0.0f);
  int ins = kn_i ? (is_own ? (sd->s <= 0.0f && h) : sd->s < 0.0f) : (on ? r.first.inside : r.inside0);
  h = h && (is_own || !ins) && (!clip || ins);
  int zero = is_own ? (!ins && !clip) : (ins && (i != c->last || kn_i));
  if (zero) {
    lf = by_s ? sd->leaf : (on ? r.first.leaf : -1);
    f = by_s ? sd->face : (on ? r.first.face : -1);
  }
  int by_on = zero && on && !by_s;
  int apart = 0;
  if (by_on) {
    NF x0[3] = {c->od[0] + c->t_lo * c->dd[0], c->od[1] + c->t_lo * c->dd[1], c->od[2] + c->t_lo * c->dd[2]};
    apart = o_face_dist(S, i, lf > 0 ? lf : 0, f, x0) > c->band;
  }
  NF te = apart ? r.first.t : (zero ? c->t_lo : (h ? t : N_HUGE));
  int wins = o_entry_wins(S, te, i, &b);
  int better = own || (clip && h && te < b.t) || (!is_own && (zero || h) && wins);
  if (better) {
    OBest nb = {te, i, lf, f, zero && !apart, own};
    return nb;
  }
  return b;
}

/* the ray's slab test against volume i's padded world box (bvh.py:258 slab; navigate.py:424 _meets) */
static inline int o_meets_box(const OScene* S, const OCtx* c, int i, const NF* inv) {
  /* a volume's padded world box, or a mesh chunk's (its BVH leaf box) */
  const NF* lo = i >= S->ch0 ? O_NAV_CBOX(S) + (size_t)6 * (i - S->ch0) : o_vfn(S, i) + LUMEN_VF_LO;
  const NF* hi = i >= S->ch0 ? lo + 3 : o_vfn(S, i) + LUMEN_VF_HI;
  NF lo_t = -N_HUGE * 10.0f, hi_t = N_HUGE * 10.0f;
  for (int a = 0; a < 3; ++a) {
    NF ta = (lo[a] - c->od[a]) * inv[a];
    NF tb = (hi[a] - c->od[a]) * inv[a];
    lo_t = o_max(lo_t, o_min(ta, tb));
    hi_t = o_min(hi_t, o_max(ta, tb));
  }
  return lo_t <= hi_t && hi_t >= c->t_lo && lo_t <= c->t_bound + c->band;
}

/* ----------------------------------------------------------------------------------------------- meshes */
/* tessellated meshes (navigate.py:80 _shear, :283 _crossing, :303 _triangle, :320 _mesh_visit; surface_id.py:33,
   :56, :67, :120): the watertight ray-triangle test (Woop, Benthin and Wald, JCGT 2013) decides inside / outside,
   t comes from the triangle's plane; a facet met from either side is an entry into the mesh */
static const NF N_FACET_BEHIND_BANDS = 0.25f;
static const NF N_FACET_SHORT_ULPS = 2.0f;
static const NF N_MESH_PARALLEL = NK(1e-6);

static inline const NF* o_tri(const OScene* S, int k) { return O_NAV_TRI(S) + (size_t)k * LUMEN_TRI_F; }
static inline NF o_pick(const NF* v, int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }
/* the chunk holding triangle k (chunks are consecutive triangles, in order) */
static inline int o_tri_chunk(const OScene* S, int k) {
  int lo = 0, hi = S->n_chunk - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (S->D->mesh_chunk[4 * mid] <= k) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

typedef struct OShear { int kx, ky, kz; NF sx, sy, sz; } OShear;
static inline OShear o_shear(const NF* dd) {
  NF a0 = n_abs(dd[0]), a1 = n_abs(dd[1]), a2 = n_abs(dd[2]);
  int kz = (a0 >= a1 && a0 >= a2) ? 0 : (a1 >= a2 ? 1 : 2);
  int kx = (kz + 1) % 3, ky = (kx + 1) % 3;
  NF dz = o_pick(dd, kz);
  if (dz < 0.0f) { int s = kx; kx = ky; ky = s; }
  OShear h = {kx, ky, kz, o_pick(dd, kx) / dz, o_pick(dd, ky) / dz, (NF)1.0f / dz};
  return h;
}

static inline int o_crossing(const OScene* S, const OCtx* c, const OShear* h, int k, NF* t_k, NF* nd, NF* s0) {
  const NF* T = o_tri(S, k);
  NF A[3], B[3], C[3];
  for (int a = 0; a < 3; ++a) { A[a] = T[a] - c->od[a]; B[a] = T[3 + a] - c->od[a]; C[a] = T[6 + a] - c->od[a]; }
  NF Ax = o_pick(A, h->kx) - h->sx * o_pick(A, h->kz), Ay = o_pick(A, h->ky) - h->sy * o_pick(A, h->kz);
  NF Bx = o_pick(B, h->kx) - h->sx * o_pick(B, h->kz), By = o_pick(B, h->ky) - h->sy * o_pick(B, h->kz);
  NF Cx = o_pick(C, h->kx) - h->sx * o_pick(C, h->kz), Cy = o_pick(C, h->ky) - h->sy * o_pick(C, h->kz);
  NF U = Cx * By - Cy * Bx, V = Ax * Cy - Ay * Cx, W = Bx * Ay - By * Ax;
  int inside = (U >= 0.0f && V >= 0.0f && W >= 0.0f) || (U <= 0.0f && V <= 0.0f && W <= 0.0f);
  NF det = U + V + W;
  NF w[3];
  for (int a = 0; a < 3; ++a) w[a] = (c->od[a] + c->t_lo * c->dd[a]) - T[a];
  *s0 = o_dot(T + 9, w);
  *nd = o_dot(T + 9, c->dd);
  *t_k = c->t_lo - *s0 / (*nd != 0.0f ? *nd : (NF)-1.0f);
  return inside && det != 0.0f;
}

static inline OBest o_mesh_visit(const OScene* S, const OCtx* c, int i, OBest b) {
  const int32_t* cr = S->D->mesh_chunk + 4 * (size_t)(i - S->ch0);
  const int k0 = cr[0], kn = cr[1];
  const NF hi_t = o_min(b.t, c->t_bound);
  const OSide* sd = &c->sd;
  if (sd->known && i == c->last && sd->s < 0.0f && (c->t_lo < b.t || (c->t_lo == b.t && b.own))) {
    OBest nb = {c->t_lo, i, sd->leaf, -1, 1, 0};
    b = nb;
  }
  const OShear h = o_shear(c->dd);
  const NF tol = N_FACET_BEHIND_BANDS * c->band;
  for (int q = 0; q < kn; ++q) {
    NF t_k, nd, s0;
    int ok = o_crossing(S, c, &h, k0 + q, &t_k, &nd, &s0);
    int front = ok && nd < 0.0f && s0 > -tol && (c->t_lo - t_k <= c->band);
    int back = ok && nd > 0.0f && s0 < -tol && t_k > c->t_lo;
    NF t_c = o_max(t_k, c->t_lo);
    if ((front || back) && t_c < hi_t && (t_c < b.t || (t_c == b.t && b.own))) {
      OBest nb = {t_c, i, k0 + q, -1, t_k <= c->t_lo, 0};
      b = nb;
    }
  }
  return b;
}

static inline OSrf o_srf_decode_m(const OScene* S, int s) {
  if (s < S->sm) return o_srf_decode(S, s);
  int km = s - S->sm;
  OSrf r;
  r.e = km % 2; km /= 2;
  r.o = km % 2; km /= 2;
  r.item = S->ch0 + o_tri_chunk(S, km);
  r.leaf = km;
  r.face = -1;
  r.known = 1;
  return r;
}
static inline void o_hit_grad_m(const OScene* S, int item, int leaf, int face, const NF* x, NF* g) {
  if (item >= S->ch0) {
    const NF* T = o_tri(S, leaf > 0 ? leaf : 0);
    g[0] = T[9]; g[1] = T[10]; g[2] = T[11];
  } else {
    o_hit_grad(S, item, leaf, face, x, g);
  }
}

/* the photon's next event in volume v: its own exit, then the first entry of every daughter whose box the ray meets
   (navigate.py:482 enter; the winner does not depend on the order of the daughters) */
static inline OBest o_enter(const OScene* S, const OCtx* c, int has_own, int vi) {
  OBest b = {N_HUGE, -1, -1, -1, 0, 0};
  if (has_own) b = o_unit_visit(S, c, vi, b, 1);
  NF inv[3];
  for (int a = 0; a < 3; ++a) {
    NF dv = c->dd[a];
    inv[a] = 1.0f / (n_abs(dv) < N_TINY_DIR ? (dv < 0.0f ? -N_TINY_DIR : N_TINY_DIR) : dv);
  }
  const int32_t* vr = o_vi(S, c->v);
  for (int k = 0; k < vr[LUMEN_VI_CN]; ++k) {
    int i = S->D->cand[vr[LUMEN_VI_C0] + k];
    if (!o_meets_box(S, c, i, inv)) continue;
    b = i >= S->ch0 ? o_mesh_visit(S, c, i, b) : o_unit_visit(S, c, i, b, 0);
  }
  return b;
}

/* ------------------------------------------------------------------------------------------------- the query */
typedef OQueryT<NF> OQuery;

/* the first visible crossing along (o, d) before t_max for a photon in vol sitting on srf `last` (navigate.py:663
   query, with _round :557, _next_volume :515, _side :497, _finish :617) */
static inline OQuery o_query(const OScene* S, const NF* o, const NF* d, int vol, NF t_max, int last,
                             const float* sn_f, NF s_at) {
  /* sn: the photon's float32 normal of its last crossing, read in NF (navigate.py:684) */
  NF sn_w[3] = {0, 0, 0};
  if (sn_f) { sn_w[0] = sn_f[0]; sn_w[1] = sn_f[1]; sn_w[2] = sn_f[2]; }
  const NF* sn = sn_f ? sn_w : 0;
  const int OUT = S->n;
  NF xa = o_maxabs3(o);
  int cls0 = o_cls(S, vol);
  OSrf l0 = o_srf_decode_m(S, last);
  int kn0 = l0.known;
  /* the round loop's carry */
  NF t_lo = 0.0f;
  int v = vol, last_ = last, done = 0, it = 0;
  NF rec_t = N_HUGE;
  int rec_item = -1, rec_leaf = -1, rec_face = -1, rec_zero = 0, rec_vb = vol, rec_vis = 0;
  int cur = cls0;
  NF pz_tp0 = N_HUGE, pz_tp1 = N_HUGE, pz_tin = 0.0f;
  int pz_np = 0, pz_vend = vol, pz_hit = 0, pz_vat = vol, pz_zc = 0, pz_vin = vol;
  int guard = 0;
  while (!done) {
    NF band = o_band(xa + n_abs(t_lo));
    int vi = v < OUT - 1 ? v : OUT - 1;
    int has_own = v < OUT;
    /* _side */
    OSrf ls = o_srf_decode_m(S, last_);
    OSide sd = {ls.known, ls.leaf, ls.face, 0.0f, 0};
    if (ls.known) {
      if (sn) {
        sd.s = o_dot(sn, d) * (ls.e ? 1.0f : -1.0f);
        sd.entry = sd.s * (ls.o ? 1.0f : -1.0f) < 0.0f;
      } else {
        NF x0[3] = {o[0] + t_lo * d[0], o[1] + t_lo * d[1], o[2] + t_lo * d[2]};
        NF g[3];
        o_hit_grad_m(S, ls.item, ls.leaf > 0 ? ls.leaf : 0, ls.face, x0, g);
        NF gd = o_dot(g, d);
        sd.s = gd / o_safe_norm(g) * (ls.o ? 1.0f : -1.0f);
        sd.entry = gd < 0.0f;
      }
    }
    OCtx c = {v, o, d, t_lo, t_max, ls.item, band, sd};
    OBest ev = o_enter(S, &c, has_own, vi);
    NF t_c = ev.t;
    int u_in = ev.item, l_in = ev.leaf, f_in = ev.face, z_in = ev.zero, is_own = ev.own;
    int hit = t_c < t_max;
    NF step = o_band(xa + n_abs(hit ? t_c : t_lo));
    /* _next_volume */
    int nxt = v, moved = 0;
    {
      const int clip = !is_own && o_is_anc(S, u_in, v); /* out through an ancestor's face */
      int go_in = !is_own && !clip;
      int uc = u_in < 0 ? 0 : (u_in > OUT - 1 ? OUT - 1 : u_in);
      int up = clip ? o_parent(S, uc) : o_parent(S, v < OUT ? v : OUT);
      int nx0 = go_in ? u_in : up;
      int unit_x = go_in ? u_in : vi;
      const int is_ch = go_in && u_in >= S->ch0; /* a mesh chunk: entered, not relocated (navigate.py:531) */
      int off = hit && l_in >= 0 && !is_ch;
      NF od2[3] = {o[0], o[1], o[2]};
      if (off) {
        NF x[3] = {o[0] + t_c * d[0], o[1] + t_c * d[1], o[2] + t_c * d[2]};
        int itm = is_own ? vi : uc;
        int lf = l_in > 0 ? l_in : 0;
        NF g[3];
        o_hit_grad(S, itm, lf, f_in, x, g);
        NF gn = o_safe_norm(g);
        NF n_[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
        NF m = o_face_dist(S, itm, lf, f_in, x) + O_RELOCATE_BANDS * o_band(o_maxabs3(x));
        NF sg = o_dot(n_, d) < 0.0f ? -1.0f : 1.0f;
        for (int a = 0; a < 3; ++a) od2[a] = o[a] + m * sg * n_[a];
      }
      NF tr = off ? t_c : t_c + step;
      if (is_ch) nxt = OUT + 1 + S->D->mesh_chunk[4 * (size_t)(u_in - S->ch0) + 2], moved = 0;
      else if (hit) nxt = o_settle(S, nx0, od2, d, tr, unit_x, step + step, &moved);
      else nxt = nx0, moved = 0;
    }
    int item = !is_own ? u_in : vi;
    int after = o_cls(S, hit ? nxt : v);
    int zl = hit && it > 0 && (z_in || t_c - pz_tin <= O_ZERO_STEP_BANDS * band);
    int touched = zl;
    if (!zl && hit && it > 0 && v < OUT && after != cur) {
      NF xm[3];
      NF tm = 0.5f * (pz_tin + t_c);
      for (int a = 0; a < 3; ++a) xm[a] = o[a] + tm * d[a];
      touched = !o_holds_point(S, vi, xm);
    }
    if (touched) cur = o_cls(S, pz_vin);
    int v_b = touched ? pz_vin : v;
    int vis = hit && after != cur;
    int inv = hit && !vis;
    int zc = (inv && t_c - t_lo <= O_ZERO_STEP_BANDS * band) ? pz_zc + 1 : 0;
    if (inv && pz_tp0 == N_HUGE) pz_tp0 = t_c;
    if (inv) pz_tp1 = t_c;
    pz_np += inv;
    if (inv) pz_vend = nxt;
    pz_hit = hit;
    if (inv && t_c <= s_at) pz_vat = nxt;
    pz_zc = zc;
    int n_vin = hit ? v_b : pz_vin;
    NF n_tin = hit ? t_c : pz_tin;
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
  NF bt = rec_t;
  int bi = rec_item, bl = rec_leaf, bf = rec_face, zero = rec_zero, vb = rec_vb;
  int vis_end = rec_vis;
  int cont = !vis_end && pz_hit && pz_zc >= O_ZSBP;
  int hit = (vis_end || cont) && bt < t_max;
  if (hit && !zero && bl >= 0 && bi >= S->ch0) { /* a mesh hit's t from its plane, short of it (mesh_plane_t) */
    const NF* T = o_tri(S, bl);
    NF nd = o_dot(T + 9, d);
    if (n_abs(nd) > N_MESH_PARALLEL) {
      NF w0[3], w1[3], w2[3];
      for (int a = 0; a < 3; ++a) { w0[a] = T[a] - o[a]; w1[a] = T[3 + a] - o[a]; w2[a] = T[6 + a] - o[a]; }
      NF m0 = o_maxabs3(w0), m1 = o_maxabs3(w1), m2 = o_maxabs3(w2);
      const NF* wn = (m0 <= m1 && m0 <= m2) ? w0 : (m1 <= m2 ? w1 : w2);
      NF t_pl = o_dot(T + 9, wn) / nd;
      NF ulp = N_EPS * (xa + n_abs(bt));
      NF sh = N_FACET_SHORT_ULPS * ulp / n_abs(nd);
      bt = o_max(t_pl - sh, 0.0f);
    }
  }
  NF px = bt < N_HUGE ? bt : 0.0f;
  NF xh[3] = {o[0] + px * d[0], o[1] + px * d[1], o[2] + px * d[2]};
  NF g[3];
  o_hit_grad_m(S, bi, bl > 0 ? bl : 0, bf, xh, g);
  NF gn = o_safe_norm(g);
  NF nrm[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
  NF fb[3] = {-d[0], -d[1], -d[2]};
  if (sn) {
    int sat = hit && zero && bl < 0 && kn0 && bt <= 0.0f;
    if (sat) {
      NF sl = o_safe_norm(sn);
      fb[0] = sn[0] / sl; fb[1] = sn[1] / sl; fb[2] = sn[2] / sl;
    }
  }
  if (!(hit && bl >= 0)) { nrm[0] = fb[0]; nrm[1] = fb[1]; nrm[2] = fb[2]; }
  NF gd = o_dot(g, d);
  int entry = bi != vb && !o_is_anc(S, bi, vb); /* an ancestor's face reached out of: an exit */
  int o_ = entry ? gd < 0.0f : gd > 0.0f;
  if (bi >= S->ch0 && bl >= 0) q.srf = hit ? S->sm + 4 * bl + 2 * o_ + entry : -1; /* a mesh triangle */
  else q.srf = hit ? o_srf_pack(S, bi, bl, bf, o_, entry) : -1;
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

