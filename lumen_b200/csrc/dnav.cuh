// The navigator's body in the precision NF (float or double): included once per precision by dgeom.cuh, inside a
// namespace of its own (nav32, nav64) that defines NF, NF3, NF4, NAV_IS64 and the NAV_* array selectors. Every
// coordinate, frame, box, leaf coefficient, root, interval and band is NF (src/lumen/rules/navigation.py:96
// Precision; docs/dev/decisions.md:332); constants are the NF value of the reference's own (float32 literals in float,
// float64 literals in double, as the reference's self.F(c)). No include guard: included twice.

constexpr NF N_HUGE = NK(1e30);
constexpr NF N_BIG = NK(1e29);
constexpr NF N_EPS = sizeof(NF) == 4 ? (NF)1.1920928955078125e-7f : (NF)2.220446049250313080847e-16;
constexpr NF N_BAND_ULPS_EPS = 8.0f * N_EPS;  // BAND_ULPS eps of the precision
constexpr NF N_BAND32_EPS = (NF)9.5367431640625e-07f;  // float32's (the reach bound's look-ahead in either precision)
constexpr NF N_BAND_FLOOR = NK(1e-9);
constexpr NF N_DIVISOR_FLOOR = NK(1e-30);
constexpr NF N_TINY_DIR = NK(1e-30);
constexpr NF N_LINEAR_REL = NK(1e-12);
constexpr NF N_PARALLEL = NK(1e-12);
constexpr NF N_TINY_NORMAL = (NF)1.17549435e-38f;  // float32's smallest normal in either precision (safe.py:52)
constexpr int N_BISECT = sizeof(NF) == 4 ? 40 : 64;  // the torus bisections: the mantissa plus a margin
constexpr NF N_TORUS_AXIAL = NK(1e-12);  // a squared xy direction below this is along the axis
constexpr NF N_TORUS_PAD_REL = NK(1e-4);  // the pretests' pad, relative to R + r
constexpr NF D_TORUS_BRACKET_ULPS = 64.0f;  // the bracket's pad on the bounding sphere, in ulps

L_DEV NF d_dot(const NF* a, const NF* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
L_DEV NF d_min(NF a, NF b) { return a < b ? a : b; }
L_DEV NF d_max(NF a, NF b) { return a > b ? a : b; }
L_DEV NF d_maxabs3(const NF* a) {
  NF m = n_abs(a[0]);
  if (n_abs(a[1]) > m) m = n_abs(a[1]);
  if (n_abs(a[2]) > m) m = n_abs(a[2]);
  return m;
}
L_DEV NF d_band(NF scale) { return N_BAND_ULPS_EPS * scale + N_BAND_FLOOR; }
L_DEV NF d_band32(NF scale) { return N_BAND32_EPS * scale + N_BAND_FLOOR; }
L_DEV NF d_safe_norm(const NF* v) { return n_sqrt(d_max(d_dot(v, v), N_TINY_NORMAL)); }

L_DEV void d_to_local_pt(const DScene& S, int i, const NF* x, NF* xl) {
  const NF* f = NAV_VOL(S) + (size_t)i * LUMEN_VOL_F;
  NF v0 = x[0] - __ldg(f + 9), v1 = x[1] - __ldg(f + 10), v2 = x[2] - __ldg(f + 11);
#pragma unroll
  for (int a = 0; a < 3; ++a) xl[a] = __ldg(f + a) * v0 + __ldg(f + 3 + a) * v1 + __ldg(f + 6 + a) * v2;
}
L_DEV void d_to_local_dir(const DScene& S, int i, const NF* d, NF* dl) {
  const NF* f = NAV_VOL(S) + (size_t)i * LUMEN_VOL_F;
#pragma unroll
  for (int a = 0; a < 3; ++a) dl[a] = __ldg(f + a) * d[0] + __ldg(f + 3 + a) * d[1] + __ldg(f + 6 + a) * d[2];
}
L_DEV void d_to_world_dir(const DScene& S, int i, const NF* g, NF* gw) {
  const NF* f = NAV_VOL(S) + (size_t)i * LUMEN_VOL_F;
#pragma unroll
  for (int a = 0; a < 3; ++a) gw[a] = __ldg(f + 3 * a) * g[0] + __ldg(f + 3 * a + 1) * g[1] + __ldg(f + 3 * a + 2) * g[2];
}

// ------------------------------------------------------------------------------------------- leaf intervals
struct Iv { NF lo0, hi0; int f_lo0, f_hi0; NF lo1, hi1; int f_lo1, f_hi1; };

L_DEV void d_Av(const NF* A, const NF* v, NF* out) {
#pragma unroll
  for (int a = 0; a < 3; ++a) out[a] = __ldg(A + 3 * a) * v[0] + __ldg(A + 3 * a + 1) * v[1] + __ldg(A + 3 * a + 2) * v[2];
}
L_DEV NF d_dotg(const NF* g, const NF* v) { return __ldg(g) * v[0] + __ldg(g + 1) * v[1] + __ldg(g + 2) * v[2]; }

L_DEV void d_quad_line(const NF* lf, const NF* y, const NF* d, NF* L0, NF* R0, int* L0q, int* R0q,
                       NF* L1, NF* R1) {
  const NF* A = lf + LUMEN_LF_A;
  const NF* b = lf + LUMEN_LF_B;
  NF c = __ldg(lf + LUMEN_LF_C), sa = __ldg(lf + LUMEN_LF_SA);
  const NF inf = N_HUGE;
  NF t_o = -d_dot(y, d);
  NF y0[3] = {y[0] + t_o * d[0], y[1] + t_o * d[1], y[2] + t_o * d[2]};
  NF Ad[3];
  d_Av(A, d, Ad);
  NF alpha = d_dot(Ad, d);
  int lin = n_abs(alpha) < d_max(N_LINEAR_REL * sa, N_DIVISOR_FLOOR);
  NF bdd = d_dotg(b, d);
  NF Ay0[3];
  d_Av(A, y0, Ay0);
  NF beta0 = d_dot(Ay0, d) + bdd;
  NF gam0 = (d_dot(y0, Ay0) + 2.0f * d_dotg(b, y0)) + c;
  int near_ = !lin && (alpha * gam0 > 0.5f * beta0 * beta0);
  NF t_c = t_o + (near_ ? -beta0 / alpha : 0.0f);
  NF yc[3] = {y[0] + t_c * d[0], y[1] + t_c * d[1], y[2] + t_c * d[2]};
  NF Ayc[3];
  d_Av(A, yc, Ayc);
  NF beta = d_dot(Ayc, d) + bdd;
  NF gam = (d_dot(yc, Ayc) + 2.0f * d_dotg(b, yc)) + c;
  NF D = beta * beta - alpha * gam;
  int Dpos = D > D_TANGENT_ULPS * N_EPS * (beta * beta + n_abs(alpha * gam));
  NF sD = n_sqrt(Dpos ? D : 1.0f);
  NF sgn = beta >= 0.0f ? 1.0f : -1.0f;
  NF s_ = -(beta + sgn * (Dpos ? sD : 0.0f));
  int s_ok = n_abs(s_) > N_DIVISOR_FLOOR;
  NF r1 = lin ? inf : s_ / alpha;
  NF r2 = s_ok ? gam / s_ : 0.0f;
  NF rmin = d_min(r1, r2) + t_c;
  NF rmax = d_max(r1, r2) + t_c;
  int b_small = n_abs(beta) < N_DIVISOR_FLOOR;
  NF tl = t_c - gam / (b_small ? 1.0f : 2.0f * beta);
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

// ------------------------------------------------------------------------------------------------ the torus
// leaf_kernels.py:212 torus_set: the interval set (two slots) of a solid torus about z along a unit ray o + s d in its
// canonical frame. g(s) = (rho - R)^2 + z^2 - r^2 has at most two inflection points (closed form); they split the
// bracket on the padded bounding sphere into convex / concave / convex parts with one extremum each (bisection on g'),
// giving at most six monotone pieces with one root at most (bisection on the membership)

L_DEV NF d_torus_g(NF R, NF r, const NF* oc, const NF* d, NF s) {
  NF x = oc[0] + s * d[0], y = oc[1] + s * d[1], z = oc[2] + s * d[2];
  NF rho2 = x * x + y * y;
  NF rho = n_sqrt(d_max(rho2, 0.0f));
  NF dr = (rho2 - R * R) / (rho + R);  // rho - R without the cancellation of rho and R
  return dr * dr + z * z - r * r;
}
L_DEV NF d_torus_dg(NF R, const NF* oc, const NF* d, NF s) {
  NF x = oc[0] + s * d[0], y = oc[1] + s * d[1], z = oc[2] + s * d[2];
  NF rho2 = x * x + y * y;
  NF rho = n_sqrt(d_max(rho2, N_TINY_NORMAL));
  NF dr = (rho2 - R * R) / (rho + R);
  NF drho = (x * d[0] + y * d[1]) / rho;
  return 2.0f * dr * drho + 2.0f * z * d[2];
}

// the exact pretests of the whole line (csg.py:175 _torus_window, the window unbounded): the padded ball, the slab
// |z| <= r, the annulus R - r <= rho <= R + r. A window of the line that misses the torus holds none of its roots, so
// solving on the whole line gives every window the reference's memberships.
L_DEV int d_torus_meets(NF R, NF r, const NF* ol, const NF* du) {
  const NF Rb = (R + r) * (1.0f + N_TORUS_PAD_REL);
  NF bb = ol[0] * du[0] + ol[1] * du[1] + ol[2] * du[2];
  NF disc = Rb * Rb - (ol[0] * ol[0] + ol[1] * ol[1] + ol[2] * ol[2] - bb * bb);
  NF sq = n_sqrt(d_max(disc, 0.0f));
  NF s_lo = -bb - sq, s_hi = -bb + sq;
  int meet = disc > 0.0f && s_lo <= s_hi;
  const NF pad = N_TORUS_PAD_REL * (R + r), rz = r + pad;
  int small = n_abs(du[2]) < N_PARALLEL;
  NF iz = 1.0f / (small ? 1.0f : du[2]);
  NF za = (-rz - ol[2]) * iz, zb = (rz - ol[2]) * iz;
  if (!small) { s_lo = d_max(s_lo, d_min(za, zb)); s_hi = d_min(s_hi, d_max(za, zb)); }
  meet = meet && s_lo <= s_hi && (!small || n_abs(ol[2]) <= rz);
  NF qa = du[0] * du[0] + du[1] * du[1], qb = ol[0] * du[0] + ol[1] * du[1], qc = ol[0] * ol[0] + ol[1] * ol[1];
  NF sm = d_min(d_max(-qb / (qa > N_PARALLEL ? qa : 1.0f), s_lo), s_hi);
  NF r2_min = qa > N_PARALLEL ? (qa * sm * sm + 2.0f * qb * sm + qc) : qc;
  NF r2_max = d_max(qa * s_lo * s_lo + 2.0f * qb * s_lo + qc, qa * s_hi * s_hi + 2.0f * qb * s_hi + qc);
  NF r_out = R + r + pad, r_in = d_max(R - r - pad, 0.0f);
  return meet && r2_min <= r_out * r_out && r2_max >= r_in * r_in;
}

L_CALL void d_torus_set(NF R, NF r, const NF* od, const NF* dd, NF* lo, NF* hi) {
  const NF inf = N_HUGE;
  NF t_c = -((od[0] * dd[0] + od[1] * dd[1]) + od[2] * dd[2]);
  NF oc[3] = {od[0] + t_c * dd[0], od[1] + t_c * dd[1], od[2] + t_c * dd[2]};
  NF q0 = (oc[0] * oc[0] + oc[1] * oc[1]) + oc[2] * oc[2];
  const NF Rb = (R + r) * (1.0f + D_TORUS_BRACKET_ULPS * N_EPS);
  NF b0 = (oc[0] * dd[0] + oc[1] * dd[1]) + oc[2] * dd[2];
  NF disc = Rb * Rb - q0 + b0 * b0;
  int hit_b = disc > 0.0f;
  NF sq = n_sqrt(hit_b ? disc : 1.0f);
  NF s_lo = -b0 - sq, s_hi = -b0 + sq;
  NF a = dd[0] * dd[0] + dd[1] * dd[1];
  NF bxy = oc[0] * dd[0] + oc[1] * dd[1];
  NF cxy = oc[0] * oc[0] + oc[1] * oc[1];
  int a_ok = a > N_TORUS_AXIAL;
  NF a_s = a_ok ? a : 1.0f;
  NF s_v = a_ok ? -bxy / a_s : 0.0f;
  NF m2 = d_max(a_ok ? cxy - bxy * bxy / a_s : cxy, 0.0f);
  NF ci = n_cbrt(R * a * m2);
  NF w2 = (ci * ci - m2) / a_s;  // the inflection points s_v -+ w
  int has_w = a_ok && w2 > 0.0f;
  NF w = n_sqrt(has_w ? w2 : 0.0f);
  NF p1 = d_min(d_max(s_v - w, s_lo), s_hi), p2 = d_min(d_max(s_v + w, s_lo), s_hi);
  // the extrema: a minimum on [s_lo, p1] (g' increasing), the maximum on [p1, p2], a minimum on [p2, s_hi]
  NF el[3] = {s_lo, p1, p2}, eh[3] = {p1, p2, s_hi}, e[3];
  for (int k = 0; k < 3; ++k) {
    NF l = el[k], h = eh[k];
    for (int it = 0; it < N_BISECT; ++it) {
      NF mid = 0.5f * (l + h);
      NF gm = d_torus_dg(R, oc, dd, mid);
      int right = k == 1 ? gm > 0.0f : gm < 0.0f;
      l = right ? mid : l;
      h = right ? h : mid;
    }
    e[k] = 0.5f * (l + h);
  }
  // the roots: one per monotone piece whose ends differ in membership
  const NF knots[7] = {s_lo, e[0], p1, e[1], p2, e[2], s_hi};
  NF t[6];
  for (int k = 0; k < 6; ++k) {
    NF xl = knots[k], xr = knots[k + 1];
    int inl = d_torus_g(R, r, oc, dd, xl) <= 0.0f, inr = d_torus_g(R, r, oc, dd, xr) <= 0.0f;
    NF l = xl, h = xr;
    for (int it = 0; it < N_BISECT; ++it) {
      NF mid = 0.5f * (l + h);
      int same = (d_torus_g(R, r, oc, dd, mid) <= 0.0f) == inl;
      l = same ? mid : l;
      h = same ? h : mid;
    }
    t[k] = (inl != inr && xr > xl && hit_b) ? 0.5f * (l + h) + t_c : inf;
  }
  for (int i = 1; i < 6; ++i)  // ascending (insertion)
    for (int j = i; j > 0 && t[j] < t[j - 1]; --j) { NF x = t[j]; t[j] = t[j - 1]; t[j - 1] = x; }
  // outside at the bracket's start: the roots alternate entry and exit
  int ok0 = t[1] < N_BIG, ok1 = t[3] < N_BIG;
  lo[0] = ok0 ? t[0] : inf; hi[0] = ok0 ? t[1] : inf;
  lo[1] = ok1 ? t[2] : inf; hi[1] = ok1 ? t[3] : inf;
}

// a torus leaf's intervals along o + t d (kind frame): its canonical frame u = M (x - og), the unit ray there, the
// roots scaled back (csg.py:207 _t_iv); out of line, returned by value (the quadric-only scenes' step pays a branch)
L_DEV NF4 d_torus_line(const NF* lf, const NF* o, const NF* d) {
  const NF* M = lf + LUMEN_LF_A;
  const NF R = __ldg(lf + LUMEN_LF_B), r = __ldg(lf + LUMEN_LF_B + 1);
  NF xl[3] = {o[0] - __ldg(lf + 0), o[1] - __ldg(lf + 1), o[2] - __ldg(lf + 2)}, ol[3], dl[3];
  d_Av(M, xl, ol);
  d_Av(M, d, dl);
  NF kk = n_sqrt(dl[0] * dl[0] + dl[1] * dl[1] + dl[2] * dl[2]);
  NF du[3] = {dl[0] / kk, dl[1] / kk, dl[2] / kk};
  NF lo[2] = {N_HUGE, N_HUGE}, hi[2] = {N_HUGE, N_HUGE};
  if (d_torus_meets(R, r, ol, du)) d_torus_set(R, r, ol, du, lo, hi);
  return NF4{n_abs(lo[0]) < N_BIG ? lo[0] / kk : lo[0], n_abs(hi[0]) < N_BIG ? hi[0] / kk : hi[0],
             n_abs(lo[1]) < N_BIG ? lo[1] / kk : lo[1], n_abs(hi[1]) < N_BIG ? hi[1] / kk : hi[1]};
}

// a torus leaf's Iv (it reads no planes: each piece its own roots, face 0; the non-empty piece first); out of line,
// the ray and the result by value, so that a scan over quadric and plane leaves keeps its registers
L_CALL Iv d_torus_iv(const NF* lf, NF3 ov, NF3 dv) {
  const NF o[3] = {ov.x, ov.y, ov.z}, d[3] = {dv.x, dv.y, dv.z};
  NF4 tv = d_torus_line(lf, o, d);
  const NF inf = N_HUGE;
  Iv r;
  int ok0 = tv.x < tv.y, ok1 = tv.z < tv.w;
  r.lo0 = ok0 ? tv.x : inf; r.hi0 = ok0 ? tv.y : inf; r.f_lo0 = ok0 ? 0 : -1; r.f_hi0 = ok0 ? 0 : -1;
  r.lo1 = ok1 ? tv.z : inf; r.hi1 = ok1 ? tv.w : inf; r.f_lo1 = ok1 ? 0 : -1; r.f_hi1 = ok1 ? 0 : -1;
  if (!ok0 && ok1) {
    Iv s = r;
    r.lo0 = s.lo1; r.hi0 = s.hi1; r.f_lo0 = s.f_lo1; r.f_hi0 = s.f_hi1;
    r.lo1 = s.lo0; r.hi1 = s.hi0; r.f_lo1 = s.f_lo0; r.f_hi1 = s.f_hi0;
  }
  return r;
}

// whether the torus holds x (kind frame): (rho - R)^2 + z^2 <= r^2 in its canonical frame (csg.py:301 _inside_leaf)
L_DEV int d_torus_holds(const NF* lf, const NF* x) {
  NF xl[3] = {x[0] - __ldg(lf + 0), x[1] - __ldg(lf + 1), x[2] - __ldg(lf + 2)}, u[3];
  d_Av(lf + LUMEN_LF_A, xl, u);
  const NF R = __ldg(lf + LUMEN_LF_B), r = __ldg(lf + LUMEN_LF_B + 1);
  NF dr = n_sqrt(u[0] * u[0] + u[1] * u[1]) - R;
  return dr * dr + u[2] * u[2] <= r * r;
}

L_DEV Iv d_leaf_iv(const DScene& S, int g, const NF* o, const NF* d) {
  const NF* lf = NAV_LEAF(S) + (size_t)g * LUMEN_LEAF_F;
  const int32_t* li = S.leaf_i + (size_t)g * LUMEN_LEAF_I;
  const NF inf = N_HUGE;
  NF y[3] = {o[0] - __ldg(lf + 3), o[1] - __ldg(lf + 4), o[2] - __ldg(lf + 5)};
  NF ol[3] = {o[0] - __ldg(lf + 0), o[1] - __ldg(lf + 1), o[2] - __ldg(lf + 2)};
  NF t0p = -inf, t1p = inf;
  int f0p = -1, f1p = -1, ep = 0;
  int p0 = __ldg(li + 1), np_ = __ldg(li + 2);
  for (int k = 0; k < np_; ++k) {
    const NF* pl = NAV_PLANE(S) + (size_t)(p0 + k) * LUMEN_PLANE_F;
    NF n0 = __ldg(pl), n1 = __ldg(pl + 1), n2 = __ldg(pl + 2), h = __ldg(pl + 3);
    NF nd = n0 * d[0] + n1 * d[1] + n2 * d[2];
    NF rhs = h - (n0 * ol[0] + n1 * ol[1] + n2 * ol[2]);
    int par = n_abs(nd) < N_PARALLEL;
    NF tp = rhs / (par ? 1.0f : nd);
    NF ent = nd < -N_PARALLEL ? tp : -inf;
    NF ext = nd > N_PARALLEL ? tp : inf;
    if (ent > t0p) { t0p = ent; f0p = k + 1; }
    if (ext < t1p) { t1p = ext; f1p = k + 1; }
    ep = ep || (par && rhs < 0.0f);
  }
  int has_q = __ldg(li) == 1;
  NF L0 = -inf, R0 = inf, L1 = inf, R1 = -inf;
  int L0q = 0, R0q = 0;
  if (has_q) d_quad_line(lf, y, d, &L0, &R0, &L0q, &R0q, &L1, &R1);
  Iv r;
  {
    NF lo = d_max(L0, t0p), hi = d_min(R0, t1p);
    int flo = L0 > t0p ? (L0q ? 0 : f0p) : f0p;
    int fhi = R0 < t1p ? (R0q ? 0 : f1p) : f1p;
    int ok = lo < hi && !ep;
    r.lo0 = ok ? lo : inf; r.hi0 = ok ? hi : inf; r.f_lo0 = ok ? flo : -1; r.f_hi0 = ok ? fhi : -1;
  }
  {
    NF lo = d_max(L1, t0p), hi = d_min(R1, t1p);
    int flo = L1 > t0p ? 0 : f0p;
    int fhi = f1p;
    int ok = lo < hi && !ep;
    r.lo1 = ok ? lo : inf; r.hi1 = ok ? hi : inf; r.f_lo1 = ok ? flo : -1; r.f_hi1 = ok ? fhi : -1;
  }
  if (r.lo0 >= inf && r.lo1 < inf) {
    Iv s = r;
    r.lo0 = s.lo1; r.hi0 = s.hi1; r.f_lo0 = s.f_lo1; r.f_hi0 = s.f_hi1;
    r.lo1 = s.lo0; r.hi1 = s.hi0; r.f_lo1 = s.f_lo0; r.f_hi1 = s.f_hi0;
  }
  return r;
}

L_DEV int d_inside_leaf(const DScene& S, int g, const NF* x) {
  const NF* lf = NAV_LEAF(S) + (size_t)g * LUMEN_LEAF_F;
  const int32_t* li = S.leaf_i + (size_t)g * LUMEN_LEAF_I;
  NF xl[3] = {x[0] - __ldg(lf + 0), x[1] - __ldg(lf + 1), x[2] - __ldg(lf + 2)};
  NF y[3] = {x[0] - __ldg(lf + 3), x[1] - __ldg(lf + 4), x[2] - __ldg(lf + 5)};
  int pl = 1;
  int p0 = __ldg(li + 1), np_ = __ldg(li + 2);
  for (int k = 0; k < np_; ++k) {
    const NF* p = NAV_PLANE(S) + (size_t)(p0 + k) * LUMEN_PLANE_F;
    pl = pl && (__ldg(p) * xl[0] + __ldg(p + 1) * xl[1] + __ldg(p + 2) * xl[2] <= __ldg(p + 3));
  }
  if (__ldg(li) == 2) return d_torus_holds(lf, x);
  if (__ldg(li) != 1) return pl;
  NF Ay[3];
  d_Av(lf + LUMEN_LF_A, y, Ay);
  const NF* b = lf + LUMEN_LF_B;
  NF qv = (d_dot(y, Ay) + 2.0f * (__ldg(b) * y[0] + __ldg(b + 1) * y[1] + __ldg(b + 2) * y[2])) + __ldg(lf + LUMEN_LF_C);
  return pl && qv <= 0.0f;
}

// the kind's postfix program over a membership functor
template <class F>
L_DEV int d_program(const DScene& S, int kind, F member) {
  const int32_t* k = S.kind_i + (size_t)kind * LUMEN_KIND_I;
  int p0 = __ldg(k + 2), pl = __ldg(k + 3);
  int32_t s = 0;
  for (int p = 0; p < pl; ++p) {
    int op = __ldg(S.prog_i + (size_t)(p0 + p) * 2), arg = __ldg(S.prog_i + (size_t)(p0 + p) * 2 + 1);
    int32_t bb = s & 1, aa = (s >> 1) & 1;
    int32_t r = op == 1 ? (aa | bb) : (op == 2 ? (aa & bb) : (aa & (1 - bb)));
    if (op == 0) s = (s << 1) | (member(arg) & 1);
    else s = ((s >> 2) << 1) | r;
  }
  return (s & 1) == 1;
}

L_DEV int d_inside_kind(const DScene& S, int kind, const NF* x) {
  int l0 = __ldg(S.kind_i + (size_t)kind * LUMEN_KIND_I);
  return d_program(S, kind, [&](int l) { return d_inside_leaf(S, l0 + l, x); });
}

// ----------------------------------------------------------------------------------------- first_change
// NLMAX: the leaves a kind can have (LUMEN_MAX_LEAVES; 1 in the instantiation for scenes of single-leaf solids)
template <int NLMAX>
struct ScanT {
  int kind, nl;
  Iv iv[NLMAX];
  NF xa, t1;
  int want;
  int has_init, init_known, init_inside;
  int has_skip, skip_leaf, skip_face, skip_entry;
  NF skip_thi;
  int has_on, on_leaf, on_inside;
  NF on_tend, hend;
};

using Scan = ScanT<LUMEN_MAX_LEAVES>;

template <int NLMAX>
L_DEV NF d_scan_band(const ScanT<NLMAX>& s, NF t) { return d_band(s.xa + n_abs(t)); }

template <int NLMAX>
L_DEV int d_mem_at(const DScene& S, const ScanT<NLMAX>& s, NF t, int use_on) {
  int on = s.has_on && use_on;
  if constexpr (NLMAX == 1) {  // a single-leaf solid: its program is the leaf itself
    const Iv& v = s.iv[0];
    int m = (v.lo0 <= t && t < v.hi0) || (v.lo1 <= t && t < v.hi1);
    if (on && s.on_leaf == 0 && t < s.hend) m = s.on_inside;
    return m;
  }
  return d_program(S, s.kind, [&](int l) {
    const Iv& v = s.iv[l];
    int m = (v.lo0 <= t && t < v.hi0) || (v.lo1 <= t && t < v.hi1);
    if (on && l == s.on_leaf && t < s.hend) m = s.on_inside;
    return m;
  });
}

// TORUS: the geometry instantiation: 1 reads torus leaves, mesh chunks and protrusion clips (scenes without them run
// one without their code), 3 the same with frame groups, 2 is for scenes whose solids are single quadric / plane
// leaves, 0 the rest
template <int TORUS, int NLMAX>
L_DEV void d_scan_init(const DScene& S, ScanT<NLMAX>& s, int kind, const NF* o, const NF* d, NF t1) {
  s.kind = kind;
  const int32_t* k = S.kind_i + (size_t)kind * LUMEN_KIND_I;
  s.nl = NLMAX == 1 ? 1 : __ldg(k + 1);
  int l0 = __ldg(k);
  for (int l = 0; l < (NLMAX == 1 ? 1 : s.nl); ++l) {
    if ((TORUS & 1) && __ldg(S.leaf_i + (size_t)(l0 + l) * LUMEN_LEAF_I) == 2)
      s.iv[l] = d_torus_iv(NAV_LEAF(S) + (size_t)(l0 + l) * LUMEN_LEAF_F, NF3{o[0], o[1], o[2]},
                           NF3{d[0], d[1], d[2]});
    else
      s.iv[l] = d_leaf_iv(S, l0 + l, o, d);
  }
  s.xa = d_max(d_max(n_abs(o[0]), n_abs(o[1])), n_abs(o[2]));
  s.t1 = t1;
  s.want = -1;
  s.has_init = s.has_skip = s.has_on = 0;
  s.hend = -N_HUGE;
}

struct First { int hit; NF t; int inside, leaf, face; };
struct Fc { int hit; NF t; int inside, leaf, face, inside0; First first; };

template <int NLMAX>
L_DEV void d_nearest(const ScanT<NLMAX>& s, NF t_cur, NF* e1o, int* lbo, int* fco, int* eko) {
  NF e1 = N_HUGE;
  int lb = -1, fc = -1, ek = 0;
  for (int l = 0; l < (NLMAX == 1 ? 1 : s.nl); ++l) {
    const Iv& v = s.iv[l];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      NF ep = j == 0 ? v.lo0 : (j == 1 ? v.hi0 : (j == 2 ? v.lo1 : v.hi1));
      int fp = j == 0 ? v.f_lo0 : (j == 1 ? v.f_hi0 : (j == 2 ? v.f_lo1 : v.f_hi1));
      int en = (j & 1) == 0;
      int ok = n_abs(ep) < N_BIG && ep <= s.t1 && ep > t_cur && ep < e1;
      if (s.has_skip) ok = ok && !(l == s.skip_leaf && fp == s.skip_face && s.skip_entry == en && ep < s.skip_thi);
      if (ok) { e1 = ep; lb = l; fc = fp; ek = en; }
    }
  }
  *e1o = e1; *lbo = lb; *fco = fc; *eko = ek;
}

template <int NLMAX>
L_DEV Fc d_first_change(const DScene& S, ScanT<NLMAX>& s, NF t0) {
  NF t_cur = t0;
  int done = 0, now = 0, lb_h = -1, fc_h = -1, now0 = 0, it = 0;
  First fs = {0, N_HUGE, 0, -1, -1};
  s.hend = s.has_on ? s.on_tend : -N_HUGE;
  while (!done && t_cur < N_HUGE && it < D_MAX_SCAN_PER_LEAF * s.nl + D_MAX_SCAN_EXTRA) {
    int first = it == 0;
    NF e; int lb, fc, ek;
    if (first) { e = t0; lb = -1; fc = -1; ek = 0; }
    else d_nearest(s, t_cur, &e, &lb, &fc, &ek);
    int has = first || e < N_HUGE;
    NF tp = first ? t0 : e + d_scan_band(s, e);
    if (s.has_on && !first && has && lb == s.on_leaf && ek != s.on_inside) s.hend = d_min(s.hend, e);
    int aft;
    if (!s.has_init) aft = has ? d_mem_at(S, s, tp, 1) : now;
    else if (has && !(first && s.init_known)) aft = d_mem_at(S, s, tp, 1);
    else aft = (first && s.init_known) ? s.init_inside : now;
    if (first) now0 = aft;
    int chg = !first && has && aft != now;
    int vis = s.want < 0 ? chg : (chg && aft == s.want);
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
  Fc r;
  r.hit = done;
  r.t = done ? t_cur : s.t1;
  r.inside = done ? now : now0;
  r.leaf = lb_h;
  r.face = fc_h;
  r.inside0 = now0;
  r.first = fs;
  return r;
}

L_DEV void d_leaf_grad(const DScene& S, int kind, int leaf, int face, const NF* x, NF* g) {
  int gi = __ldg(S.kind_i + (size_t)kind * LUMEN_KIND_I) + (leaf > 0 ? leaf : 0);
  const NF* lf = NAV_LEAF(S) + (size_t)gi * LUMEN_LEAF_F;
  const int32_t* li = S.leaf_i + (size_t)gi * LUMEN_LEAF_I;
  if (face >= 1) {
    const NF* p = NAV_PLANE(S) + (size_t)(__ldg(li + 1) + face - 1) * LUMEN_PLANE_F;
    g[0] = __ldg(p); g[1] = __ldg(p + 1); g[2] = __ldg(p + 2);
    return;
  }
  if (__ldg(li) == 2) {  // M^T of the canonical gradient of ((rho - R)^2 + z^2 - r^2) / 2 (csg.py:452 leaf_grad)
    const NF* M = lf + LUMEN_LF_A;
    NF xl[3] = {x[0] - __ldg(lf + 0), x[1] - __ldg(lf + 1), x[2] - __ldg(lf + 2)}, u[3];
    d_Av(M, xl, u);
    NF rho = n_sqrt(d_max(u[0] * u[0] + u[1] * u[1], N_DIVISOR_FLOOR));
    NF k = (rho - __ldg(lf + LUMEN_LF_B)) / rho;
    NF gu[3] = {k * u[0], k * u[1], u[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] = (__ldg(M + a) * gu[0] + __ldg(M + 3 + a) * gu[1]) + __ldg(M + 6 + a) * gu[2];
    return;
  }
  NF y[3] = {x[0] - __ldg(lf + 3), x[1] - __ldg(lf + 4), x[2] - __ldg(lf + 5)};
  NF Ay[3];
  d_Av(lf + LUMEN_LF_A, y, Ay);
  const NF* b = lf + LUMEN_LF_B;
#pragma unroll
  for (int a = 0; a < 3; ++a) g[a] = 2.0f * (Ay[a] + __ldg(b + a));
}

L_DEV NF d_leaf_dist(const DScene& S, int kind, int leaf, int face, const NF* x) {
  int gi = __ldg(S.kind_i + (size_t)kind * LUMEN_KIND_I) + (leaf > 0 ? leaf : 0);
  const NF* lf = NAV_LEAF(S) + (size_t)gi * LUMEN_LEAF_F;
  const int32_t* li = S.leaf_i + (size_t)gi * LUMEN_LEAF_I;
  NF f;
  if (face >= 1) {
    const NF* p = NAV_PLANE(S) + (size_t)(__ldg(li + 1) + face - 1) * LUMEN_PLANE_F;
    NF xl[3] = {x[0] - __ldg(lf + 0), x[1] - __ldg(lf + 1), x[2] - __ldg(lf + 2)};
    f = __ldg(p) * xl[0] + __ldg(p + 1) * xl[1] + __ldg(p + 2) * xl[2] - __ldg(p + 3);
  } else if (__ldg(li) == 2) {  // ((rho - R)^2 + z^2 - r^2) / 2 (csg.py:470 leaf_dist)
    NF xl[3] = {x[0] - __ldg(lf + 0), x[1] - __ldg(lf + 1), x[2] - __ldg(lf + 2)}, u[3];
    d_Av(lf + LUMEN_LF_A, xl, u);
    NF dr = n_sqrt(u[0] * u[0] + u[1] * u[1]) - __ldg(lf + LUMEN_LF_B), rr = __ldg(lf + LUMEN_LF_B + 1);
    f = 0.5f * (dr * dr + u[2] * u[2] - rr * rr);
  } else {
    NF y[3] = {x[0] - __ldg(lf + 3), x[1] - __ldg(lf + 4), x[2] - __ldg(lf + 5)};
    NF Ay[3];
    d_Av(lf + LUMEN_LF_A, y, Ay);
    const NF* b = lf + LUMEN_LF_B;
    f = (d_dot(y, Ay) + 2.0f * (__ldg(b) * y[0] + __ldg(b + 1) * y[1] + __ldg(b + 2) * y[2])) + __ldg(lf + LUMEN_LF_C);
  }
  NF g[3];
  d_leaf_grad(S, kind, leaf, face, x, g);
  return n_abs(f) / d_safe_norm(g);
}

L_DEV int d_clampv(const DScene& S, int item) { return item < 0 ? 0 : (item > S.n - 1 ? S.n - 1 : item); }

L_DEV void d_hit_grad(const DScene& S, int item, int leaf, int face, const NF* x, NF* gw) {
  int i = d_clampv(S, item);
  NF xl[3], g[3];
  d_to_local_pt(S, i, x, xl);
  d_leaf_grad(S, vI(S, i, LUMEN_VI_KIND), leaf, face, xl, g);
  d_to_world_dir(S, i, g, gw);
}
L_DEV NF d_face_dist(const DScene& S, int item, int leaf, int face, const NF* x) {
  int i = d_clampv(S, item);
  NF xl[3];
  d_to_local_pt(S, i, x, xl);
  return d_leaf_dist(S, vI(S, i, LUMEN_VI_KIND), leaf, face, xl);
}

L_DEV int d_srf_pack(const DScene& S, int item, int leaf, int face, int o, int e) {
  if (item < 0 || leaf < 0 || face < 0) return item;
  return S.SU + ((item * S.LM + leaf) * S.FM + face) * 4 + 2 * o + e;
}
struct Srf { int item, leaf, face, o, known, e; };
L_DEV Srf d_srf_decode(const DScene& S, int s) {
  Srf r;
  if (s < S.SU) { r.item = s; r.leaf = -1; r.face = -1; r.o = 0; r.known = 0; r.e = 0; return r; }
  int u = s - S.SU;
  r.e = u % 2; u /= 2;
  r.o = u % 2; u /= 2;
  r.face = u % S.FM; u /= S.FM;
  r.leaf = u % S.LM; u /= S.LM;
  r.item = u;
  r.known = 1;
  return r;
}

L_DEV int d_holds_point(const DScene& S, int i, const NF* x) {
  NF xl[3];
  d_to_local_pt(S, i, x, xl);
  return d_inside_kind(S, vI(S, i, LUMEN_VI_KIND), xl);
}
L_DEV int d_ray_holds(const DScene& S, int i, const NF* od, const NF* dd, NF t) {
  NF ol[3], dl[3];
  d_to_local_pt(S, i, od, ol);
  d_to_local_dir(S, i, dd, dl);
  Scan s;
  d_scan_init<1>(S, s, vI(S, i, LUMEN_VI_KIND), ol, dl, N_HUGE);
  return d_mem_at(S, s, t, 0);
}
L_DEV int d_level_wins(const DScene& S, int item, int found, int excl) {
  return (found < 0 || d_rank(S, item) > d_rank(S, found)) && item != excl && item < S.n;
}

// the BVH point scan: every daughter of v whose padded box holds x, visited by `visit`
template <class F>
L_DEV void d_point_scan(const DScene& S, int v, const NF* x, NF pad, F visit) {
  int n0 = vI(S, v, LUMEN_VI_NODE0), n1 = vI(S, v, LUMEN_VI_NODE1);
  int node = n0;
  while (node < n1) {
    const NF* nf = NAV_NODE(S) + (size_t)node * LUMEN_NODE_F;
    int inside = (__ldg(nf) - pad <= x[0] && x[0] <= __ldg(nf + 3) + pad) &&
                 (__ldg(nf + 1) - pad <= x[1] && x[1] <= __ldg(nf + 4) + pad) &&
                 (__ldg(nf + 2) - pad <= x[2] && x[2] <= __ldg(nf + 5) + pad);
    const int32_t* ni = S.node_i + (size_t)node * LUMEN_NODE_I;
    int cnt = __ldg(ni + 1);
    if (inside && cnt > 0) {
      int st = __ldg(ni + 2);
      for (int k = 0; k < cnt; ++k) visit(__ldg(S.items + st + k));
    }
    node = (inside && cnt == 0) ? node + 1 : __ldg(ni);
  }
}

// the same over the extended instantiation's frame groups too: each group's nodes with the point in its frame
// (x_g = R^T x; the group tables and frames as d_enter_x reads them)
template <class F>
L_DEV void d_point_scan_x(const DScene& S, int v, const NF* x, NF pad, F visit) {
  int n0 = vI(S, v, LUMEN_VI_NODE0), n1 = vI(S, v, LUMEN_VI_NODE1);
  int g = 0, g_end = 0;
  const int* gt = (S.mesh && __ldg(S.mesh + 7) > 0) ? S.mesh + __ldg(S.mesh + 7) : nullptr;
  if (gt) {
    g = __ldg(gt + 2 * v);
    g_end = g + __ldg(gt + 2 * v + 1);
  }
  NF xs[3] = {x[0], x[1], x[2]};
  for (int guard = 0; guard <= LUMEN_MAX_GROUPS_PER_VOLUME; ++guard) {
    int node = n0;
    while (node < n1) {
      const NF* nf = NAV_NODE(S) + (size_t)node * LUMEN_NODE_F;
      int inside = (__ldg(nf) - pad <= xs[0] && xs[0] <= __ldg(nf + 3) + pad) &&
                   (__ldg(nf + 1) - pad <= xs[1] && xs[1] <= __ldg(nf + 4) + pad) &&
                   (__ldg(nf + 2) - pad <= xs[2] && xs[2] <= __ldg(nf + 5) + pad);
      const int32_t* ni = S.node_i + (size_t)node * LUMEN_NODE_I;
      int cnt = __ldg(ni + 1);
      if (inside && cnt > 0) {
        int st = __ldg(ni + 2);
        for (int k = 0; k < cnt; ++k) visit(__ldg(S.items + st + k));
      }
      node = (inside && cnt == 0) ? node + 1 : __ldg(ni);
    }
    if (g >= g_end) break;
    const int* gr = gt + 2 * (S.n + 1) + 2 * g;
    n0 = __ldg(gr);
    n1 = __ldg(gr + 1);
    const NF* R = NAV_LEAF(S) + __ldg(S.mesh + 6) + (size_t)9 * g;
#pragma unroll
    for (int a = 0; a < 3; ++a) xs[a] = (__ldg(R + a) * x[0] + __ldg(R + 3 + a) * x[1]) + __ldg(R + 6 + a) * x[2];
    g++;
  }
}

// whether volume i is an ancestor of volume v (navigate.py:199 is_ancestor: the walk is depth first, a subtree is its
// root and the LUMEN_VI_SIZE - 1 volumes after it): an ancestor among v's candidates is one v reaches out of, whose
// face is v's exit (a protrusion clip). Daughters come after v, so for them the first test ends it without a load.
L_DEV int d_is_anc(const DScene& S, int i, int v) { return i >= 0 && i < v && v < S.n && v < i + vI(S, i, LUMEN_VI_SIZE); }

L_DEV int d_find(const DScene& S, int v, const NF* x) {
  int g = -1;
  d_point_scan(S, v, x, 0.0f, [&](int i) {
    if (d_level_wins(S, i, g, -1) && d_holds_point(S, i, x)) g = i;
  });
  return g;
}
L_DEV int d_locate(const DScene& S, const NF* x) {
  int v = S.n;
  for (int guard = 0; guard < 64; ++guard) {
    int f = d_find(S, v, x);
    if (f < 0) return v;
    v = f;
  }
  return v;
}
L_DEV int d_find_ray(const DScene& S, int v, const NF* od, const NF* dd, NF t, int excl, NF pad) {
  NF x[3] = {od[0] + t * dd[0], od[1] + t * dd[1], od[2] + t * dd[2]};
  int g = -1;
  d_point_scan(S, v, x, pad, [&](int i) {
    if (d_level_wins(S, i, g, excl) && d_ray_holds(S, i, od, dd, t)) g = i;
  });
  return g;
}
L_DEV int d_settle(const DScene& S, int v, const NF* od, const NF* dd, NF t, int crossed, NF pad, int* moved) {
  int v_ = v, held = 0;
  for (int guard = 0; guard < 256; ++guard) {
    int vi = v_ < S.n - 1 ? v_ : S.n - 1;
    int test = !held && v_ < S.n && v_ != crossed;
    int ins = !test || d_ray_holds(S, vi, od, dd, t);
    int f = ins ? d_find_ray(S, v_, od, dd, t, crossed, pad) : -1;
    int nv = ins ? (f >= 0 ? f : v_) : d_parent(S, v_ < S.n ? v_ : S.n);
    held = ins && f >= 0;
    if (f < 0 && ins) break;
    v_ = nv;
  }
  *moved = v_ != v;
  return v_;
}
// the same for the extended instantiation (a scene with protrusion clips): an ancestor among the candidates is one
// the volume reaches out of, never a volume to descend into
L_DEV int d_find_x(const DScene& S, int v, const NF* x) {
  int g = -1;
  d_point_scan_x(S, v, x, 0.0f, [&](int i) {
    if (d_level_wins(S, i, g, -1) && !d_is_anc(S, i, v) && d_holds_point(S, i, x)) g = i;
  });
  return g;
}
L_DEV int d_locate_x(const DScene& S, const NF* x) {
  int v = S.n;
  for (int guard = 0; guard < 64; ++guard) {
    int f = d_find_x(S, v, x);
    if (f < 0) return v;
    v = f;
  }
  return v;
}
L_DEV int d_find_ray_x(const DScene& S, int v, const NF* od, const NF* dd, NF t, int excl, NF pad) {
  NF x[3] = {od[0] + t * dd[0], od[1] + t * dd[1], od[2] + t * dd[2]};
  int g = -1;
  d_point_scan_x(S, v, x, pad, [&](int i) {
    if (d_level_wins(S, i, g, excl) && !d_is_anc(S, i, v) && d_ray_holds(S, i, od, dd, t)) g = i;
  });
  return g;
}
L_DEV int d_settle_x(const DScene& S, int v, const NF* od, const NF* dd, NF t, int crossed, NF pad, int* moved) {
  int v_ = v, held = 0;
  for (int guard = 0; guard < 256; ++guard) {
    int vi = v_ < S.n - 1 ? v_ : S.n - 1;
    int test = !held && v_ < S.n && v_ != crossed;
    int ins = !test || d_ray_holds(S, vi, od, dd, t);
    int f = ins ? d_find_ray_x(S, v_, od, dd, t, crossed, pad) : -1;
    int nv = ins ? (f >= 0 ? f : v_) : d_parent(S, v_ < S.n ? v_ : S.n);
    held = ins && f >= 0;
    if (f < 0 && ins) break;
    v_ = nv;
  }
  *moved = v_ != v;
  return v_;
}

// --------------------------------------------------------------------------------------------- a visit
struct Side { int known, leaf, face; NF s; int entry; };
struct Best { NF t; int item, leaf, face, zero, own; };
struct Ctx {
  int v;
  NF od[3], dd[3];
  NF t_lo, t_bound;
  int last;
  NF band;
  Side sd;
};

L_DEV int d_on_face(const DScene& S, const Ctx& c, int i, const First& fr, int kn_i) {
  NF dt = fr.t - c.t_lo;
  NF lim = D_K_ON * c.band;
  int far_ = 0;
  if (!kn_i && fr.hit && dt >= lim && dt < D_GRAZE * lim) {
    NF x0[3] = {c.od[0] + c.t_lo * c.dd[0], c.od[1] + c.t_lo * c.dd[1], c.od[2] + c.t_lo * c.dd[2]};
    NF xc[3] = {c.od[0] + fr.t * c.dd[0], c.od[1] + fr.t * c.dd[1], c.od[2] + fr.t * c.dd[2]};
    int lf = fr.leaf > 0 ? fr.leaf : 0;
    NF g0[3], gc[3];
    d_hit_grad(S, i, lf, fr.face, x0, g0);
    d_hit_grad(S, i, lf, fr.face, xc, gc);
    NF s0 = d_dot(g0, c.dd) / d_safe_norm(g0);
    int other_way = (s0 * d_dot(gc, c.dd) < 0.0f) && (n_abs(s0) > 1.0f / D_GRAZE);
    far_ = (d_face_dist(S, i, lf, fr.face, x0) < lim) && !other_way;
  }
  return !kn_i && fr.hit && (dt < lim || far_);
}

L_DEV int d_entry_wins(const DScene& S, NF t, int item, const Best& b) {
  return t < b.t || (t == b.t && (b.own || d_rank(S, item) > d_rank(S, b.item)));
}

template <int TORUS>
L_DEV Best d_unit_visit(const DScene& S, const Ctx& c, int i, Best b, int is_own) {
  // an ancestor the volume is not proved inside (the extended instantiation): its first exit from a start inside it,
  // when earlier than every other event (navigate.py:376 _unit_visit, clip)
  int clip = 0;
  if constexpr ((TORUS & 1)) clip = !is_own && d_is_anc(S, i, c.v);
  const int own = is_own;
  if constexpr ((TORUS & 1)) is_own = is_own || clip;
  const Side& sd = c.sd;
  NF bnd = c.t_bound + c.band;
  NF ol[3], dl[3];
  d_to_local_pt(S, i, c.od, ol);
  d_to_local_dir(S, i, c.dd, dl);
  int kn_i = sd.known && i == c.last;
  NF t_on = c.t_lo + D_K_ON * c.band / d_max(n_abs(sd.s), 1.0f / D_GRAZE);
  int lf_on = kn_i ? sd.leaf : -2;
  ScanT<TORUS == 2 ? 1 : LUMEN_MAX_LEAVES> s;
  d_scan_init<TORUS>(S, s, vI(S, i, LUMEN_VI_KIND), ol, dl, bnd);
  s.want = is_own ? 0 : 1;
  s.has_init = 1; s.init_known = kn_i; s.init_inside = is_own;
  s.has_skip = 1; s.skip_leaf = lf_on; s.skip_face = sd.face; s.skip_entry = sd.entry; s.skip_thi = N_HUGE;
  s.has_on = 1; s.on_leaf = lf_on; s.on_inside = sd.entry; s.on_tend = t_on;
  Fc r = d_first_change(S, s, c.t_lo);
  int h = r.hit, lf = r.leaf, f = r.face;
  NF t = r.t;
  int on = d_on_face(S, c, i, r.first, kn_i);
  int by_s = kn_i && (is_own ? sd.s > 0.0f : sd.s < 0.0f);
  int ins = kn_i ? (is_own ? (sd.s <= 0.0f && h) : sd.s < 0.0f) : (on ? r.first.inside : r.inside0);
  h = h && (is_own || !ins);
  if constexpr ((TORUS & 1)) h = h && (!clip || ins);
  int zero = is_own ? !ins : (ins && (i != c.last || kn_i));
  if constexpr ((TORUS & 1)) zero = zero && !clip;
  if (zero) {
    lf = by_s ? sd.leaf : (on ? r.first.leaf : -1);
    f = by_s ? sd.face : (on ? r.first.face : -1);
  }
  int by_on = zero && on && !by_s;
  int apart = 0;
  if (by_on) {
    NF x0[3] = {c.od[0] + c.t_lo * c.dd[0], c.od[1] + c.t_lo * c.dd[1], c.od[2] + c.t_lo * c.dd[2]};
    apart = d_face_dist(S, i, lf > 0 ? lf : 0, f, x0) > c.band;
  }
  NF te = apart ? r.first.t : (zero ? c.t_lo : (h ? t : N_HUGE));
  int wins = d_entry_wins(S, te, i, b);
  int better = is_own || (!is_own && (zero || h) && wins);
  if constexpr ((TORUS & 1)) better = own || (clip && h && te < b.t) || (!is_own && (zero || h) && wins);
  if (better) {
    Best nb = {te, i, lf, f, zero && !apart, own};
    return nb;
  }
  return b;
}

// slab test of a node's box (bvh.py:258): the boxes A (the navigator's BVH: NF; the sensor reach's: float32 in either
// precision) against the ray's origin in NF and its inverse direction V (NF, or float32 from a float32 direction)
template <class A, class V>
L_DEV void d_slab(const A* __restrict__ node_f, int node, const NF* o, const V* inv, NF* tin, NF* tout) {
  const A* nf = node_f + (size_t)node * LUMEN_NODE_F;
  NF lo_t = -N_HUGE * 10.0f, hi_t = N_HUGE * 10.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    NF ta = (__ldg(nf + a) - o[a]) * inv[a];
    NF tb = (__ldg(nf + 3 + a) - o[a]) * inv[a];
    lo_t = d_max(lo_t, d_min(ta, tb));
    hi_t = d_min(hi_t, d_max(ta, tb));
  }
  *tin = lo_t;
  *tout = hi_t;
}


// ------------------------------------------------------------------------------------------------- meshes
// Tessellated meshes (navigate.py:283-332, surface_id.py:120): a mesh chunk (navigator id >= CH0) is visited by the
// watertight ray-triangle test (Woop, Benthin and Wald, JCGT 2013: the ray's axes sheared so that it runs along +z,
// each triangle's edge functions in the sheared xy plane) for inside / outside only; t comes from the triangle's
// plane. The block S.mesh: n_mesh, n_chunk, n_tri, the triangles' offset in the leaf array (elements), SM (the
// first mesh surface code), CH0, 0, 0; per chunk (first triangle, count, mesh, 0); per triangle its chunk. A triangle
// is LUMEN_TRI_F values of the navigator's precision: V0, V1, V2, the unit normal.
constexpr int MESH_HDR = 8;
constexpr NF N_FACET_BEHIND_BANDS = 0.25f;  // a start behind a facet's plane by at most this many bands is on it
constexpr NF N_FACET_SHORT_ULPS = 2.0f;     // a mesh hit's t from its plane, this many ulps short of it
constexpr NF N_MESH_PARALLEL = NK(1e-6);    // a mesh hit's plane is used where |n . d| is above this

L_DEV int m_ch0(const DScene& S) { return S.mesh ? __ldg(S.mesh + 5) : 0x7fffffff; }
L_DEV int m_sm(const DScene& S) { return S.mesh ? __ldg(S.mesh + 4) : 0x7fffffff; }
L_DEV const NF* m_tri(const DScene& S, int k) { return NAV_LEAF(S) + __ldg(S.mesh + 3) + (size_t)k * LUMEN_TRI_F; }
L_DEV NF m_pick(const NF* v, int k) { return k == 0 ? v[0] : (k == 1 ? v[1] : v[2]); }

struct Shear { int kx, ky, kz; NF sx, sy, sz; };
// the watertight test's shear of the direction (navigate.py:80 _shear)
L_DEV Shear d_shear(const NF* dd) {
  NF a0 = n_abs(dd[0]), a1 = n_abs(dd[1]), a2 = n_abs(dd[2]);
  int kz = (a0 >= a1 && a0 >= a2) ? 0 : (a1 >= a2 ? 1 : 2);
  int kx = kz == 2 ? 0 : kz + 1;
  int ky = kx == 2 ? 0 : kx + 1;
  NF dz = m_pick(dd, kz);
  if (dz < 0.0f) { int s = kx; kx = ky; ky = s; }
  Shear h = {kx, ky, kz, m_pick(dd, kx) / dz, m_pick(dd, ky) / dz, (NF)1.0f / dz};
  return h;
}

// whether the ray crosses triangle k, its t from the plane, n . d and the start's height over the plane
// (navigate.py:283 _crossing)
L_DEV int d_crossing(const DScene& S, const Ctx& c, const Shear& h, int k, NF* t_k, NF* nd, NF* s0) {
  const NF* T = m_tri(S, k);
  NF A[3], B[3], C[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    A[a] = __ldg(T + a) - c.od[a];
    B[a] = __ldg(T + 3 + a) - c.od[a];
    C[a] = __ldg(T + 6 + a) - c.od[a];
  }
  NF Ax = m_pick(A, h.kx) - h.sx * m_pick(A, h.kz), Ay = m_pick(A, h.ky) - h.sy * m_pick(A, h.kz);
  NF Bx = m_pick(B, h.kx) - h.sx * m_pick(B, h.kz), By = m_pick(B, h.ky) - h.sy * m_pick(B, h.kz);
  NF Cx = m_pick(C, h.kx) - h.sx * m_pick(C, h.kz), Cy = m_pick(C, h.ky) - h.sy * m_pick(C, h.kz);
  NF U = Cx * By - Cy * Bx;
  NF V = Ax * Cy - Ay * Cx;
  NF W = Bx * Ay - By * Ax;
  int inside = (U >= 0.0f && V >= 0.0f && W >= 0.0f) || (U <= 0.0f && V <= 0.0f && W <= 0.0f);
  NF det = U + V + W;
  NF N[3] = {__ldg(T + 9), __ldg(T + 10), __ldg(T + 11)};
  NF w[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) w[a] = (c.od[a] + c.t_lo * c.dd[a]) - __ldg(T + a);
  *s0 = d_dot(N, w);
  *nd = d_dot(N, c.dd);
  *t_k = c.t_lo - *s0 / (*nd != 0.0f ? *nd : (NF)-1.0f);
  return inside && det != 0.0f;
}

// the best event after mesh chunk i (navigate.py:320 _mesh_visit, :303 _triangle: the facet rule): the triangle the
// photon sits on, heading into it, is a zero-length re-hit; else a facet is met entering it (n . d < 0, the start
// behind its plane within the tolerance) or from clearly behind (the start inside the closed surface): both entries
L_DEV Best d_mesh_visit(const DScene& S, const Ctx& c, int ch0, int i, Best b) {
  const int* cr = S.mesh + MESH_HDR + 4 * (i - ch0);
  const int k0 = __ldg(cr), kn = __ldg(cr + 1);
  const NF hi_t = d_min(b.t, c.t_bound);
  const Side& sd = c.sd;
  int re = sd.known && i == c.last && sd.s < 0.0f && (c.t_lo < b.t || (c.t_lo == b.t && b.own));
  if (re) {
    Best nb = {c.t_lo, i, sd.leaf, -1, 1, 0};
    b = nb;
  }
  const Shear h = d_shear(c.dd);
  const NF tol = N_FACET_BEHIND_BANDS * c.band;
  for (int q = 0; q < kn; ++q) {
    NF t_k, nd, s0;
    int ok = d_crossing(S, c, h, k0 + q, &t_k, &nd, &s0);
    int front = ok && nd < 0.0f && s0 > -tol && (c.t_lo - t_k <= c.band);
    int back = ok && nd > 0.0f && s0 < -tol && t_k > c.t_lo;
    NF t_c = d_max(t_k, c.t_lo);
    if ((front || back) && t_c < hi_t && (t_c < b.t || (t_c == b.t && b.own))) {
      Best nb = {t_c, i, k0 + q, -1, t_k <= c.t_lo, 0};
      b = nb;
    }
  }
  return b;
}

// a surface code with the mesh codes (surface_id.py:33 srf_decode, :56 srf_pack: a mesh triangle k is SM + 4 k + 2 o
// + e, its item the triangle's chunk)
L_DEV Srf d_srf_decode_m(const DScene& S, int s) {
  const int sm = m_sm(S);
  if (s < sm) return d_srf_decode(S, s);
  int km = s - sm;
  Srf r;
  r.e = km % 2; km /= 2;
  r.o = km % 2; km /= 2;
  r.item = m_ch0(S) + __ldg(S.mesh + MESH_HDR + 4 * __ldg(S.mesh + 1) + km);
  r.leaf = km;
  r.face = -1;
  r.known = 1;
  return r;
}
template <int EXT>
L_DEV Srf d_decode(const DScene& S, int s) {
  if constexpr (EXT) return d_srf_decode_m(S, s);
  else return d_srf_decode(S, s);
}
// the winning surface's gradient: a mesh triangle's normal, else the volume's leaf (surface_id.py:67 hit_grad)
L_DEV void d_hit_grad_m(const DScene& S, int ch0, int item, int leaf, int face, const NF* x, NF* g) {
  if (item >= ch0) {
    const NF* T = m_tri(S, leaf > 0 ? leaf : 0);
    g[0] = __ldg(T + 9); g[1] = __ldg(T + 10); g[2] = __ldg(T + 11);
  } else {
    d_hit_grad(S, item, leaf, face, x, g);
  }
}

// the next event in volume v: its own exit, then the first entry of every daughter the BVH does not prune. One
// call site of the visit (the own solid is the first candidate, then the traversal yields one leaf item at a time).
// the extended instantiation's next event in volume v: the world-frame BVH, then each frame group's BVH with the ray
// in the group's frame (x_g = R^T x_w: the boxes there are the members' own, tight for rotated wire planes); the
// visits are the world ray's, so the winner is the same as one BVH over every candidate
L_DEV Best d_enter_x(const DScene& S, const Ctx& c, int has_own, int vi) {
  Best b = {N_HUGE, -1, -1, -1, 0, 0};
  const int ch0 = m_ch0(S);
  int n0 = vI(S, c.v, LUMEN_VI_NODE0), n1 = vI(S, c.v, LUMEN_VI_NODE1);
  int g = 0, g_end = 0;  // the volume's frame groups still to walk
  const int* gt = (S.mesh && __ldg(S.mesh + 7) > 0) ? S.mesh + __ldg(S.mesh + 7) : nullptr;
  if (gt) {
    g = __ldg(gt + 2 * c.v);
    g_end = g + __ldg(gt + 2 * c.v + 1);
  }
  NF os[3] = {c.od[0], c.od[1], c.od[2]}, ds[3] = {c.dd[0], c.dd[1], c.dd[2]};
  NF inv[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    NF dv = ds[a];
    inv[a] = 1.0f / (n_abs(dv) < N_TINY_DIR ? (dv < 0.0f ? -N_TINY_DIR : N_TINY_DIR) : dv);
  }
  int stack[D_STACK];
  NF tins[D_STACK];
  int sp = 0;
  int node = -1;
  int lp = 0, lend = 0;  // the current leaf's items still to visit: S.items[lp, lend)
  int started = 0;
  int pending = has_own;
  for (;;) {
    int item = -1, is_own = 0;
    if (pending) {
      item = vi;
      is_own = 1;
      pending = 0;
    } else {
      if (!started) {
        started = 1;
        node = -1;
        if (n0 < n1) {
          NF tin, tout;
          d_slab(NAV_NODE(S), n0, os, inv, &tin, &tout);
          node = (tin <= tout && tout >= c.t_lo && tin <= d_min(b.t, c.t_bound) + c.band) ? n0 : -1;
        }
      }
      while (item < 0) {
        if (lp < lend) {
          item = __ldg(S.items + lp++);
          break;
        }
        if (node < 0) {
          NF lim = d_min(b.t, c.t_bound) + c.band;
          while (sp > 0 && tins[sp - 1] > lim) sp--;
          if (sp == 0) break;
          sp--;
          node = stack[sp];
        }
        const int32_t* ni = S.node_i + (size_t)node * LUMEN_NODE_I;
        int cnt = __ldg(ni + 1);
        if (cnt > 0) {  // a leaf: its items in turn
          lp = __ldg(ni + 2);
          lend = lp + cnt;
          node = -1;
          continue;
        }
        int lc = node + 1;
        int rc = __ldg(S.node_i + (size_t)lc * LUMEN_NODE_I);
        NF tl, tlo, tr, tro;
        d_slab(NAV_NODE(S), lc, os, inv, &tl, &tlo);
        d_slab(NAV_NODE(S), rc, os, inv, &tr, &tro);
        NF lim = d_min(b.t, c.t_bound) + c.band;
        int hl = tl <= tlo && tlo >= c.t_lo && tl <= lim;
        int hr = tr <= tro && tro >= c.t_lo && tr <= lim;
        int first = tl <= tr;
        int near_ = first ? lc : rc, far_ = first ? rc : lc;
        int h_near = first ? hl : hr, h_far = first ? hr : hl;
        if (h_near && h_far && sp < D_STACK) {
          stack[sp] = far_;
          tins[sp] = first ? tr : tl;
          sp++;
        }
        node = h_near ? near_ : (h_far ? far_ : -1);
      }
      if (item < 0) {  // this BVH is done: the next frame group's, the ray in its frame
        if (g >= g_end) break;
        const int* gr = gt + 2 * (S.n + 1) + 2 * g;
        n0 = __ldg(gr);
        n1 = __ldg(gr + 1);
        const NF* R = NAV_LEAF(S) + __ldg(S.mesh + 6) + (size_t)9 * g;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          os[a] = (__ldg(R + a) * c.od[0] + __ldg(R + 3 + a) * c.od[1]) + __ldg(R + 6 + a) * c.od[2];
          ds[a] = (__ldg(R + a) * c.dd[0] + __ldg(R + 3 + a) * c.dd[1]) + __ldg(R + 6 + a) * c.dd[2];
        }
#pragma unroll
        for (int a = 0; a < 3; ++a) {
          NF dv = ds[a];
          inv[a] = 1.0f / (n_abs(dv) < N_TINY_DIR ? (dv < 0.0f ? -N_TINY_DIR : N_TINY_DIR) : dv);
        }
        g++;
        started = 0;
        sp = 0;
        continue;
      }
    }
    if (item >= ch0 && !is_own) b = d_mesh_visit(S, c, ch0, item, b);
    else b = d_unit_visit<1>(S, c, item, b, is_own);
  }
  return b;
}

// slab test of a box held in registers (lo[3], hi[3]): d_slab's arithmetic on a node record's child box
L_DEV void d_slab_box(const float* bx, const NF* o, const NF* inv, NF* tin, NF* tout) {
  NF lo_t = -N_HUGE * 10.0f, hi_t = N_HUGE * 10.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    NF ta = (bx[a] - o[a]) * inv[a];
    NF tb = (bx[3 + a] - o[a]) * inv[a];
    lo_t = d_max(lo_t, d_min(ta, tb));
    hi_t = d_min(hi_t, d_max(ta, tb));
  }
  *tin = lo_t;
  *tout = hi_t;
}

// The candidate entries of volume c.v along the ray (navigate.py:482 enter, :465 _group, :430 _node): the volume's own
// solid first (has_own), then its BVH depth first, the nearer child first and the farther onto the stack with its
// entry t, the stack's entries past the best event so far dropped, each leaf's items in turn (a leaf holds one or
// more). The float32 navigator walks the node records (S.node_w: per inner node both children's boxes and codes in
// 64 B, four 16-byte loads a level); the float64 one the node arrays (a child's box and its right sibling's index
// read from the node).
template <int TORUS>
L_DEV Best d_enter(const DScene& S, const Ctx& c, int has_own, int vi) {
  if constexpr (TORUS == 3) return d_enter_x(S, c, has_own, vi);
  Best b = {N_HUGE, -1, -1, -1, 0, 0};
  const int ch0 = (TORUS & 1) ? m_ch0(S) : 0x7fffffff;  // the extended instantiation: mesh chunks among the items
  int n0 = vI(S, c.v, LUMEN_VI_NODE0), n1 = vI(S, c.v, LUMEN_VI_NODE1);
  NF inv[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    NF dv = c.dd[a];
    inv[a] = 1.0f / (n_abs(dv) < N_TINY_DIR ? (dv < 0.0f ? -N_TINY_DIR : N_TINY_DIR) : dv);
  }
  int stack[D_STACK];
  NF tins[D_STACK];
  int sp = 0;
#if NAV_IS64
  int node = -1;       // the traversal's next node (-1: pop or done)
  int lp = 0, lend = 0;  // the current leaf's items still to visit: S.items[lp, lend)
#else
  int node = -1;       // the next node's code: an inner node's index, -2 - p a leaf's item list at S.witem + p, -1 none
  int lp = -1;         // the current leaf's next item in S.witem (-1: none)
#endif
  int started = 0;     // the root has been tested
  int pending = has_own;
  for (;;) {
    int item = -1, is_own = 0;
    if (pending) {
      item = vi;
      is_own = 1;
      pending = 0;
    } else {
      if (!started) {
        started = 1;
        if (n0 < n1) {
          NF tin, tout;
          d_slab(NAV_NODE(S), n0, c.od, inv, &tin, &tout);
          const int meets = tin <= tout && tout >= c.t_lo && tin <= d_min(b.t, c.t_bound) + c.band;
#if NAV_IS64
          node = meets ? n0 : -1;
#else
          node = meets ? __float_as_int(__ldg(S.node_w + (size_t)n0 * 4 + 3).z) : -1;  // the root's own code
#endif
        }
      }
      while (item < 0) {
#if NAV_IS64
        if (lp < lend) {
          item = __ldg(S.items + lp++);
          break;
        }
#else
        if (lp >= 0) {
          item = __ldg(S.witem + lp);
          lp = __ldg(S.witem + lp + 1) >= 0 ? lp + 1 : -1;
          break;
        }
#endif
        if (node == -1) {
          NF lim = d_min(b.t, c.t_bound) + c.band;
          while (sp > 0 && tins[sp - 1] > lim) sp--;
          if (sp == 0) break;
          sp--;
          node = stack[sp];
        }
#if NAV_IS64
        const int32_t* ni = S.node_i + (size_t)node * LUMEN_NODE_I;
        int cnt = __ldg(ni + 1);
        if (cnt > 0) {  // a leaf: its items in turn
          lp = __ldg(ni + 2);
          lend = lp + cnt;
          node = -1;
          continue;
        }
        int lc = node + 1;
        int rc = __ldg(S.node_i + (size_t)lc * LUMEN_NODE_I);
        NF tl, tlo, tr, tro;
        d_slab(NAV_NODE(S), lc, c.od, inv, &tl, &tlo);
        d_slab(NAV_NODE(S), rc, c.od, inv, &tr, &tro);
#else
        if (node <= -2) {  // a leaf: its items in turn
          lp = -2 - node;
          node = -1;
          continue;
        }
        const float4* nw = S.node_w + (size_t)node * 4;
        const float4 w0 = __ldg(nw), w1 = __ldg(nw + 1), w2 = __ldg(nw + 2), w3 = __ldg(nw + 3);
        const float bl[6] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y}, br[6] = {w1.z, w1.w, w2.x, w2.y, w2.z, w2.w};
        const int lc = __float_as_int(w3.x), rc = __float_as_int(w3.y);
        NF tl, tlo, tr, tro;
        d_slab_box(bl, c.od, inv, &tl, &tlo);
        d_slab_box(br, c.od, inv, &tr, &tro);
#endif
        NF lim = d_min(b.t, c.t_bound) + c.band;
        int hl = tl <= tlo && tlo >= c.t_lo && tl <= lim;
        int hr = tr <= tro && tro >= c.t_lo && tr <= lim;
        int first = tl <= tr;
        int near_ = first ? lc : rc, far_ = first ? rc : lc;
        int h_near = first ? hl : hr, h_far = first ? hr : hl;
        if (h_near && h_far && sp < D_STACK) {
          stack[sp] = far_;
          tins[sp] = first ? tr : tl;
          sp++;
        }
        node = h_near ? near_ : (h_far ? far_ : -1);
      }
      if (item < 0) break;
    }
    if ((TORUS & 1) && item >= ch0 && !is_own) b = d_mesh_visit(S, c, ch0, item, b);
    else b = d_unit_visit<TORUS>(S, c, item, b, is_own);
  }
  return b;
}

// ------------------------------------------------------------------------------------------------ the query
using Query = QueryT<NF>;

// sn: the photon's float32 normal of its last crossing, read in NF (navigate.py:684)
template <int TORUS>
L_DEV Query d_query(const DScene& S, const NF* o, const NF* d, int vol, NF t_max, int last, const float* sn_f,
                    NF s_at) {
#if NAV_IS64
  NF sn_w[3];
  if (sn_f) { sn_w[0] = sn_f[0]; sn_w[1] = sn_f[1]; sn_w[2] = sn_f[2]; }
  const NF* sn = sn_f ? sn_w : nullptr;
#else
  const NF* sn = sn_f;
#endif
  const int OUT = S.n;
  const int ch0 = (TORUS & 1) ? m_ch0(S) : 0x7fffffff;  // the extended instantiation: mesh chunks
  NF xa = d_maxabs3(o);
  int cls0 = d_cls(S, vol);
  Srf l0 = d_decode<(TORUS & 1)>(S, last);
  int kn0 = l0.known;
  NF t_lo = 0.0f;
  int v = vol, last_ = last, done = 0, it = 0;
  NF rec_t = N_HUGE;
  int rec_item = -1, rec_leaf = -1, rec_face = -1, rec_zero = 0, rec_vb = vol, rec_vis = 0;
  int cur = cls0;
  NF pz_tp0 = N_HUGE, pz_tp1 = N_HUGE, pz_tin = 0.0f;
  int pz_np = 0, pz_vend = vol, pz_hit = 0, pz_vat = vol, pz_zc = 0, pz_vin = vol;
  int guard = 0;
  while (!done) {
    NF band = d_band(xa + n_abs(t_lo));
    int vi = v < OUT - 1 ? v : OUT - 1;
    int has_own = v < OUT;
    Srf ls = d_decode<(TORUS & 1)>(S, last_);
    Side sd = {ls.known, ls.leaf, ls.face, 0.0f, 0};
    if (ls.known) {
      if (sn) {
        sd.s = d_dot(sn, d) * (ls.e ? 1.0f : -1.0f);
        sd.entry = sd.s * (ls.o ? 1.0f : -1.0f) < 0.0f;
      } else {
        NF x0[3] = {o[0] + t_lo * d[0], o[1] + t_lo * d[1], o[2] + t_lo * d[2]};
        NF g[3];
        if constexpr ((TORUS & 1)) d_hit_grad_m(S, ch0, ls.item, ls.leaf > 0 ? ls.leaf : 0, ls.face, x0, g);
        else d_hit_grad(S, ls.item, ls.leaf > 0 ? ls.leaf : 0, ls.face, x0, g);
        NF gd = d_dot(g, d);
        sd.s = gd / d_safe_norm(g) * (ls.o ? 1.0f : -1.0f);
        sd.entry = gd < 0.0f;
      }
    }
    Ctx c;
    c.v = v;
    c.od[0] = o[0]; c.od[1] = o[1]; c.od[2] = o[2];
    c.dd[0] = d[0]; c.dd[1] = d[1]; c.dd[2] = d[2];
    c.t_lo = t_lo; c.t_bound = t_max; c.last = ls.item; c.band = band; c.sd = sd;
    Best ev = d_enter<TORUS>(S, c, has_own, vi);
    NF t_c = ev.t;
    int u_in = ev.item, l_in = ev.leaf, f_in = ev.face, z_in = ev.zero, is_own = ev.own;
    int hit = t_c < t_max;
    NF step = d_band(xa + n_abs(hit ? t_c : t_lo));
    int nxt = v, moved = 0;
    {
      const int clip = (TORUS & 1) && !is_own && d_is_anc(S, u_in, v);  // out through an ancestor's face
      int go_in = !is_own && !clip;
      int uc = u_in < 0 ? 0 : (u_in > OUT - 1 ? OUT - 1 : u_in);
      int up = clip ? d_parent(S, uc) : d_parent(S, v < OUT ? v : OUT);
      int nx0 = go_in ? u_in : up;
      int unit_x = go_in ? u_in : vi;
      const int is_ch = (TORUS & 1) && go_in && u_in >= ch0;  // a mesh chunk: entered, not relocated (navigate.py:531)
      int off = hit && l_in >= 0 && !is_ch;
      NF od2[3] = {o[0], o[1], o[2]};
      if (off) {
        NF x[3] = {o[0] + t_c * d[0], o[1] + t_c * d[1], o[2] + t_c * d[2]};
        int itm = is_own ? vi : uc;
        int lf = l_in > 0 ? l_in : 0;
        NF g[3];
        d_hit_grad(S, itm, lf, f_in, x, g);
        NF gn = d_safe_norm(g);
        NF n_[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
        NF m = d_face_dist(S, itm, lf, f_in, x) + D_RELOCATE_BANDS * d_band(d_maxabs3(x));
        NF sg = d_dot(n_, d) < 0.0f ? -1.0f : 1.0f;
#pragma unroll
        for (int a = 0; a < 3; ++a) od2[a] = o[a] + m * sg * n_[a];
      }
      NF tr = off ? t_c : t_c + step;
      if (is_ch) { nxt = OUT + 1 + __ldg(S.mesh + MESH_HDR + 4 * (u_in - ch0) + 2); moved = 0; }
      else if (hit) {
        if constexpr ((TORUS & 1)) nxt = d_settle_x(S, nx0, od2, d, tr, unit_x, step + step, &moved);
        else nxt = d_settle(S, nx0, od2, d, tr, unit_x, step + step, &moved);
      }
      else { nxt = nx0; moved = 0; }
    }
    int item = !is_own ? u_in : vi;
    int after = d_cls(S, hit ? nxt : v);
    int zl = hit && it > 0 && (z_in || t_c - pz_tin <= D_ZERO_STEP_BANDS * band);
    int touched = zl;
    if (!zl && hit && it > 0 && v < OUT && after != cur) {
      NF xm[3];
      NF tm = 0.5f * (pz_tin + t_c);
#pragma unroll
      for (int a = 0; a < 3; ++a) xm[a] = o[a] + tm * d[a];
      touched = !d_holds_point(S, vi, xm);
    }
    if (touched) cur = d_cls(S, pz_vin);
    int v_b = touched ? pz_vin : v;
    int vis = hit && after != cur;
    int inv_ = hit && !vis;
    int zc = (inv_ && t_c - t_lo <= D_ZERO_STEP_BANDS * band) ? pz_zc + 1 : 0;
    if (inv_ && pz_tp0 == N_HUGE) pz_tp0 = t_c;
    if (inv_) pz_tp1 = t_c;
    pz_np += inv_;
    if (inv_) pz_vend = nxt;
    pz_hit = hit;
    if (inv_ && t_c <= s_at) pz_vat = nxt;
    pz_zc = zc;
    int n_vin = hit ? v_b : pz_vin;
    NF n_tin = hit ? t_c : pz_tin;
    pz_vin = n_vin;
    pz_tin = n_tin;
    done = !hit || vis || zc >= D_ZSBP;
    if (hit) { rec_t = t_c; rec_item = item; rec_leaf = l_in; rec_face = f_in; rec_zero = z_in; rec_vb = v_b; rec_vis = vis; }
    t_lo = moved ? t_c + step : t_c;
    if (hit) v = nxt;
    last_ = item;
    it += 1;
    if (hit) cur = after;
    if (++guard > 4096) break;
  }
  Query q;
  NF bt = rec_t;
  int bi = rec_item, bl = rec_leaf, bf = rec_face, zero = rec_zero, vb = rec_vb;
  int vis_end = rec_vis;
  int cont = !vis_end && pz_hit && pz_zc >= D_ZSBP;
  int hit = (vis_end || cont) && bt < t_max;
  if constexpr ((TORUS & 1)) {  // a mesh hit's t from its plane, short of it (surface_id.py:120 mesh_plane_t)
    if (hit && !zero && bl >= 0 && bi >= ch0) {
      const NF* T = m_tri(S, bl);
      NF nk[3] = {__ldg(T + 9), __ldg(T + 10), __ldg(T + 11)};
      NF nd = d_dot(nk, d);
      if (n_abs(nd) > N_MESH_PARALLEL) {
        NF w0[3], w1[3], w2[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) { w0[a] = __ldg(T + a) - o[a]; w1[a] = __ldg(T + 3 + a) - o[a]; w2[a] = __ldg(T + 6 + a) - o[a]; }
        NF m0 = d_maxabs3(w0), m1 = d_maxabs3(w1), m2 = d_maxabs3(w2);
        const NF* wn = (m0 <= m1 && m0 <= m2) ? w0 : (m1 <= m2 ? w1 : w2);
        NF t_pl = d_dot(nk, wn) / nd;
        NF ulp = N_EPS * (xa + n_abs(bt));
        NF sh = N_FACET_SHORT_ULPS * ulp / n_abs(nd);
        bt = d_max(t_pl - sh, 0.0f);
      }
    }
  }
  NF px = bt < N_HUGE ? bt : 0.0f;
  NF xh[3] = {o[0] + px * d[0], o[1] + px * d[1], o[2] + px * d[2]};
  NF g[3];
  if constexpr ((TORUS & 1)) d_hit_grad_m(S, ch0, bi, bl > 0 ? bl : 0, bf, xh, g);
  else d_hit_grad(S, bi, bl > 0 ? bl : 0, bf, xh, g);
  NF gn = d_safe_norm(g);
  NF nrm[3] = {g[0] / gn, g[1] / gn, g[2] / gn};
  NF fb[3] = {-d[0], -d[1], -d[2]};
  if (sn) {
    int sat = hit && zero && bl < 0 && kn0 && bt <= 0.0f;
    if (sat) {
      NF sl = d_safe_norm(sn);
      fb[0] = sn[0] / sl; fb[1] = sn[1] / sl; fb[2] = sn[2] / sl;
    }
  }
  if (!(hit && bl >= 0)) { nrm[0] = fb[0]; nrm[1] = fb[1]; nrm[2] = fb[2]; }
  NF gd = d_dot(g, d);
  int entry = bi != vb && !((TORUS & 1) && d_is_anc(S, bi, vb));  // an ancestor's face reached out of: an exit
  int o_ = entry ? gd < 0.0f : gd > 0.0f;
  if ((TORUS & 1) && bi >= ch0 && bl >= 0) q.srf = hit ? m_sm(S) + 4 * bl + 2 * o_ + entry : -1;  // a mesh triangle
  else q.srf = hit ? d_srf_pack(S, bi, bl, bf, o_, entry) : -1;
  if (nrm[0] * d[0] + nrm[1] * d[1] + nrm[2] * d[2] > 0.0f) { nrm[0] = -nrm[0]; nrm[1] = -nrm[1]; nrm[2] = -nrm[2]; }
  vb = hit ? vb : pz_vend;
  q.t = hit ? bt : t_max;
  q.hit = hit;
  q.cont = cont;
  q.vol_after = hit ? v : vol;
  q.vol_before = vb;
  q.vol_start = vol;
  q.cls_before = d_cls(S, vb);
  q.cls_start = cls0;
  q.cls_after = hit ? cur : d_cls(S, vb);
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

// ------------------------------------------------------------------------------------------------ sensor reach
// The query's bound for a bulk step (src/lumen/geometry/reach.py:201 ReachGeometry.query): where the photon, not on a
// surface, starts inside its component's box, its free path s ends before the box's exit T, and the segment [0, T]
// meets no sensor box, every crossing it can deposit at lies beyond s, so the query may stop at s plus the
// navigator's own look-ahead ((GRAZE K_ON + 2) bands): the same arithmetic for every round that starts before s
// (the boxes, the direction and s float32 in either precision: reach.py:88, :216)
L_DEV NF d_reach_bound(const DScene& S, const NF* x, const float* d, int vol, int srf, float s, NF t_max) {
  if (!S.comp || srf >= 0 || vol < 0 || vol > S.n) return t_max;
  int c = __ldg(S.comp + vol);
  if (c < 0) return t_max;
  float inv[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    float dv = d[a];
    inv[a] = 1.0f / (fabsf(dv) < D_TINY_DIR ? (dv < 0.0f ? -D_TINY_DIR : D_TINY_DIR) : dv);
  }
  const float* cb = S.comp_box + (size_t)c * 6;
  NF tin = -N_HUGE * 10.0f, tout = N_HUGE * 10.0f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    NF ta = (__ldg(cb + a) - x[a]) * inv[a];
    NF tb = (__ldg(cb + 3 + a) - x[a]) * inv[a];
    tin = d_max(tin, d_min(ta, tb));
    tout = d_min(tout, d_max(ta, tb));
  }
  if (!(tin <= 0.0f && s < tout && s < t_max)) return t_max;
  for (int node = 0, guard = 0; node < S.n_fnode && guard < S.n_fnode; ++guard) {  // any sensor box on [0, T]
    NF ti, to;
    d_slab(S.fnode_f, node, x, inv, &ti, &to);
    int hit = ti <= to && to >= 0.0f && ti <= tout;
    int leaf = __ldg(S.fnode_i + (size_t)node * LUMEN_NODE_I + 1) > 0;
    if (hit && leaf) return t_max;
    node = (hit && !leaf) ? node + 1 : __ldg(S.fnode_i + (size_t)node * LUMEN_NODE_I);
  }
  NF look = (D_GRAZE * D_K_ON + 2.0f) * d_band32(d_maxabs3(x) + s);
  return d_min(t_max, s + look);
}

