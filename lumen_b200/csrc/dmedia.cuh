// The bulk channels besides Rayleigh on the device: Geant4's Mie lobe (G4OpMieHG) with its density, the isotropic
// lobe, and G4OpWLS's re-emission (src/lumen/media/phase.py:113-191, spectra.py, emission.py:127-162); the same
// arithmetic as the CPU checker's, operation for operation.
#pragma once
#include "dphys.cuh"

namespace lb {

#define D_FOUR_PI 12.5663706143591729539f
#define D_DEFENSIVE 0.01f  // the defensive mixture's share (src/lumen/rules/choices.py:113)
// its covering weight e / (1 - e), formed in double and rounded once to float32 (estimator.py:106)
#define D_EDGE_SHARE ((float)(0.01 / (1.0 - 0.01)))
#define D_WLS_TRIES 100.0f  // G4OpWLS's redraws of an energy below the absorbed one (spectra.py:22)


// ------------------------------------------------------------------------------------------------- the Mie lobe
L_DEV void d_mie_hg_cos(float g, float r, float* cm, float* cp) {
  int up = g >= 0.0f;
  float d = up ? (1.0f - g) + 2.0f * g * r : (1.0f - g) * (1.0f - r) + (1.0f + g) * r;
  float one_gr = up ? 1.0f + g * r : (1.0f - r) + (1.0f + g) * r;
  float d2 = d * d;
  float omg = 1.0f - g, opg = 1.0f + g;
  *cm = 2.0f * (omg * omg) * (1.0f - r) * one_gr / d2;
  *cp = 2.0f * r * (opg * opg) * ((1.0f - g) + g * r) / d2;
}
L_DEV float d_hg_density(float g, float cm, float cp, float* dg) {
  float omg = 1.0f - g, opg = 1.0f + g;
  float q = g >= 0.0f ? omg * omg + 2.0f * g * cm : opg * opg - 2.0f * g * cp;
  float sq = sqrtf(q);
  float q15 = q * sq;
  float h = omg * opg / (D_FOUR_PI * q15);
  if (dg) {
    float dq = g >= 0.0f ? -2.0f * omg + 2.0f * cm : 2.0f * opg - 2.0f * cp;
    *dg = (-2.0f * g * q - 1.5f * (omg * opg) * dq) / (D_FOUR_PI * q15 * q);
  }
  return h;
}
L_DEV void d_hg_direction(float cm, float cp, float u, const float* wi, float* wo) {
  float mu = cm < cp ? 1.0f - cm : cp - 1.0f;
  float s2 = cm * cp;
  float s = s2 > 0.0f ? sqrtf(s2) : 0.0f;
  float sp, cpp;
  l_sincos2pi(u, &sp, &cpp);
  float l[3] = {s * cpp, s * sp, mu};
  d_to_world(l, wi, wo);
}
L_DEV void d_mie_sample(float gf, float gb, float ratio, const float* wi, float r0, float r1, float r2, float* wo) {
  int fwd = r0 <= ratio;
  float cm, cp;
  d_mie_hg_cos(fwd ? gf : gb, r1, &cm, &cp);
  if (!fwd) {
    float t = cm;
    cm = cp;
    cp = t;
  }
  d_hg_direction(cm, cp, r2, wi, wo);
}
L_DEV float d_mie_logpdf(float gf, float gb, float ratio, const float* wi, const float* wo, float* d) {
  float dm[3] = {wo[0] - wi[0], wo[1] - wi[1], wo[2] - wi[2]}, dp[3] = {wo[0] + wi[0], wo[1] + wi[1], wo[2] + wi[2]};
  float cm = 0.5f * d_dot(dm, dm), cp = 0.5f * d_dot(dp, dp);
  float dF, dB;
  float F = d_hg_density(gf, cm, cp, d ? &dF : nullptr);
  float B = d_hg_density(-gb, cm, cp, d ? &dB : nullptr);
  float mix = ratio * F + (1.0f - ratio) * B;
  if (d) {
    d[0] = ratio * dF / mix;
    d[1] = -((1.0f - ratio) * dB) / mix;
    d[2] = (F - B) / mix;
  }
  return l_log(mix);
}
L_DEV void d_isotropic(const float* wi, float u0, float u1, float* wo) {
  float mu = 1.0f - 2.0f * u0;
  float s2 = 1.0f - mu * mu;
  float s = s2 > 0.0f ? sqrtf(s2) : 0.0f;
  float sp, cp;
  l_sincos2pi(u1, &sp, &cp);
  float l[3] = {s * cp, s * sp, mu};
  d_to_world(l, wi, wo);
}

// ------------------------------------------------------------------------------------ the WLS spectrum sampler
// Geant4's sampler of a spectrum table (spectra.py:47 g4_arrays) read interval by interval from the pool: e the k
// knots (eV), s the intensities; with cover, the one defensive mixture over the intervals without mass
struct DSpec {
  const float* e;
  const float* s;
  int k;
  float tot, Z;
  int cover;
};
L_DEV DSpec d_spec(const float* e, const float* s, int k, int cover) {
  DSpec p;
  p.e = e; p.s = s; p.k = k; p.tot = 0.0f; p.Z = 0.0f;
  for (int j = 0; j + 1 < k; ++j) {
    float h = __ldg(e + j + 1) - __ldg(e + j);
    float m = 0.5f * (__ldg(s + j + 1) + __ldg(s + j)) * h;
    p.tot = j == 0 ? m : p.tot + m;
    if (__ldg(s + j + 1) + __ldg(s + j) <= 0.0f && h > 0.0f) p.Z = p.Z + h;
  }
  p.cover = cover && p.Z > 0.0f;
  return p;
}
L_DEV float d_spec_d(const DSpec& p, int j) {
  float sj = __ldg(p.s + j), sj1 = __ldg(p.s + j + 1);
  float d = 0.5f * (sj1 + sj) / p.tot;
  if (!p.cover) return d;
  float h = __ldg(p.e + j + 1) - __ldg(p.e + j);
  float z = (sj1 + sj <= 0.0f && h > 0.0f) ? 1.0f : 0.0f;
  return (1.0f - D_DEFENSIVE) * d + D_DEFENSIVE * z / p.Z;
}
L_DEV float d_spec_c_next(const DSpec& p, int j, float c_j, float* mass_acc) {
  float h = __ldg(p.e + j + 1) - __ldg(p.e + j);
  if (p.cover) return c_j + d_spec_d(p, j) * h;
  float m = 0.5f * (__ldg(p.s + j + 1) + __ldg(p.s + j)) * h;
  *mass_acc = j == 0 ? m : *mass_acc + m;
  return *mass_acc / p.tot;
}
L_DEV float d_spec_invert(const DSpec& p, float r) {
  int n = p.k - 1, kk = 0;
  float c = 0.0f, ck = 0.0f, acc = 0.0f;
  for (int j = 0; j < n; ++j) {
    if (c <= r) { kk = j; ck = c; }
    if (j + 1 < n) c = d_spec_c_next(p, j, c, &acc);
  }
  float d = d_spec_d(p, kk), h = __ldg(p.e + kk + 1) - __ldg(p.e + kk);
  float x = d > 0.0f ? d_max(r - ck, 0.0f) / d : 0.0f;
  x = x < 0.0f ? 0.0f : (x > h ? h : x);
  return __ldg(p.e + kk) + x;
}
L_DEV float d_spec_cumulative(const DSpec& p, float E) {
  int n = p.k - 1, kk = 0;
  float c = 0.0f, ck = 0.0f, acc = 0.0f;
  for (int j = 0; j < n; ++j) {
    if (__ldg(p.e + j) <= E) { kk = j; ck = c; }
    if (j + 1 < n) c = d_spec_c_next(p, j, c, &acc);
  }
  float h = __ldg(p.e + kk + 1) - __ldg(p.e + kk);
  float t = E - __ldg(p.e + kk);
  t = t < 0.0f ? 0.0f : (t > h ? h : t);
  float u = ck + d_spec_d(p, kk) * t;
  if (E < __ldg(p.e)) return 0.0f;
  return u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
}
L_DEV float d_spec_density(const float* e, const float* s, int k, int cover, float E) {
  if (!(E >= __ldg(e) && E <= __ldg(e + k - 1))) return 0.0f;
  float tot = 0.0f, Z = 0.0f;
  for (int j = 0; j + 1 < k; ++j) {
    float sj = __ldg(s + j), sj1 = __ldg(s + j + 1), h = __ldg(e + j + 1) - __ldg(e + j);
    float t = (sj1 + sj) * h;
    tot = j == 0 ? t : tot + t;
    if (sj1 + sj <= 0.0f && h > 0.0f) Z = Z + h;
  }
  int i = 0;
  for (int j = 0; j < k; ++j)
    if (__ldg(e + j) <= E) i = j;
  i = i > k - 2 ? k - 2 : i;
  float si = __ldg(s + i), si1 = __ldg(s + i + 1);
  float p = (si + si1) / tot;
  if (!(cover && Z > 0.0f)) return p;
  float h = __ldg(e + i + 1) - __ldg(e + i);
  float z = (si1 + si <= 0.0f && h > 0.0f) ? 1.0f : 0.0f;
  return (1.0f - D_DEFENSIVE) * p + D_DEFENSIVE * z / Z;
}
L_DEV float d_kept(float f) {
  float c = f < 0.0f ? 0.0f : (f > 1.0f - D_EPS32 ? 1.0f - D_EPS32 : f);
  return -l_expm1(D_WLS_TRIES * l_log1p(-c));
}
L_DEV float d_safe_div(float a, float b) { return b != 0.0f ? a / b : 0.0f; }

struct Emit { float lam, delay, w, w_r, dyield; };
// a G4OpWLS re-emission of a photon absorbed at lam_in (emission.py:136 EmissionRecord.sample)
L_DEV Emit d_wls_emit(const float* el, const float* sl, int kl, const float* er_, const float* sr, int kr, float yl,
                      float yr, float tau, int exponential, float lam_in, float u_lam, float u_t) {
  Emit o;
  DSpec q = d_spec(er_, sr, kr, 1);
  float E_in = D_HC / lam_in;
  float f_q = d_spec_cumulative(q, E_in);
  float energy_draw = d_spec_invert(q, u_lam * f_q);
  o.lam = D_HC / energy_draw;
  float energy = D_HC / o.lam;
  float qd = d_spec_density(er_, sr, kr, 1, energy);
  float dens_q = d_safe_div(qd, f_q);
  float dr = d_kept(f_q) * d_safe_div(qd, f_q);
  o.w_r = yr * d_safe_div(dr, dens_q);
  DSpec l = d_spec(el, sl, kl, 0);
  float f_l = d_spec_cumulative(l, E_in);
  float dl = d_kept(f_l) * d_safe_div(d_spec_density(el, sl, kl, 0, energy), f_l);
  float ratio = d_safe_div(dl, dens_q);
  o.w = yl * ratio;
  o.dyield = ratio;
  o.delay = exponential ? -tau * l_log(u_t) : tau + 0.0f * u_t;
  return o;
}

// What a bulk event of the Mie or WLS channel gives: direction, state, the lobe weight live / reference, the yield
// weights, the delay, the wavelength and the tangents of the lobe weight's log and of the yield weight
struct Bulk2 {
  float d[3], er[3], ei[3];
  float rlw, y_w, y_r, delay, lam;
  float dlob[LUMEN_MAX_GRAD], dyld[LUMEN_MAX_GRAD];
};
L_DEV void d_bulk_other(const DScene& S, const float* __restrict__ live, const float* __restrict__ ref, int shared,
                         int cs, int mi, float lam, const float* wi, const float* er0, const float* ei0, Key vkey,
                         int P, const int* gt, Bulk2& b) {
  const int32_t* m = S.med_i + (size_t)mi * LUMEN_MED_I;
  float E = D_HC / lam;
  b.rlw = 1.0f; b.y_w = 1.0f; b.y_r = 1.0f; b.delay = 0.0f; b.lam = lam;
  for (int p = 0; p < P; ++p) { b.dlob[p] = 0.0f; b.dyld[p] = 0.0f; }
  float r3 = uniform(vkey, 3), r4 = uniform(vkey, 4);
  if (cs == 1) {
    int tg[3] = {__ldg(m + LUMEN_MI_MIE_GF), __ldg(m + LUMEN_MI_MIE_GB), __ldg(m + LUMEN_MI_MIE_R)};
    float pl[3], pr[3];
    for (int k = 0; k < 3; ++k) {
      pl[k] = d_tab(S, live, tg[k], E);
      pr[k] = shared ? pl[k] : d_tab(S, ref, tg[k], E);
    }
    // a covered lobe choice (LUMEN_MI_MIE_COVER): at a forward ratio of 0 or 1 the lobe never drawn gets the
    // defensive share, the pair (r, 1 - r) renormalised (phase.py:173 _mie_cover, estimator.py:101 defensive_q)
    const float r0 = pr[2];
    if (__ldg(m + LUMEN_MI_MIE_COVER) == 1 && !(r0 > 0.0f && 1.0f - r0 > 0.0f)) {
      float q0 = r0 > 0.0f ? r0 : D_EDGE_SHARE, q1 = 1.0f - r0 > 0.0f ? 1.0f - r0 : D_EDGE_SHARE;
      pr[2] = q0 / (q0 + q1);
    }
    d_mie_sample(pr[0], pr[1], pr[2], wi, r3, r4, uniform(vkey, 5), b.d);
    float dl[3];
    float lp = d_mie_logpdf(pl[0], pl[1], pl[2], wi, b.d, dl);
    if (!shared || pr[2] != r0) b.rlw = l_exp(lp - d_mie_logpdf(pr[0], pr[1], pr[2], wi, b.d, nullptr));
    for (int p = 0; p < P; ++p)
      for (int k = 0; k < 3; ++k)
        if (tg[k] == gt[p]) b.dlob[p] = b.dlob[p] + dl[k];
    for (int a = 0; a < 3; ++a) { b.er[a] = er0[a]; b.ei[a] = ei0[a]; }
    d_project(b.er, b.ei, b.d);
  } else {
    d_isotropic(wi, r3, r4, b.d);
    for (int a = 0; a < 3; ++a) { b.er[a] = 0.0f; b.ei[a] = 0.0f; }
    int ts = __ldg(m + LUMEN_MI_WLS_SPEC), ty = __ldg(m + LUMEN_MI_WLS_YIELD), tt = __ldg(m + LUMEN_MI_WLS_TAU);
    int off = __ldg(S.tab + 2 * ts), ks = __ldg(S.tab + 2 * ts + 1);
    const float* pl_ = live + off;
    const float* pr_ = ref + off;
    float yl = d_tab(S, live, ty, E), yr = shared ? yl : d_tab(S, ref, ty, E);
    float tau = d_tab(S, live, tt, E);
    Emit em = d_wls_emit(pl_, pl_ + ks, ks, pr_, pr_ + ks, ks, yl, yr, tau, __ldg(m + LUMEN_MI_WLS_PROFILE) == 1, lam,
                         uniform(vkey, 7), uniform(vkey, 8));
    b.y_w = em.w;
    b.y_r = em.w_r;
    b.delay = em.delay;
    b.lam = em.lam;
    for (int p = 0; p < P; ++p)
      if (ty == gt[p]) b.dyld[p] = em.dyield;
  }
}

}  // namespace lb
