/* The bulk channels besides Rayleigh (test infrastructure: the CPU checker's restatement): Geant4's Mie lobe
   (G4OpMieHG) and its density, the isotropic lobe, and G4OpWLS's re-emission (the spectrum sampler, its truncation at
   the absorbed energy, the defensive cover and the weights), after src/lumen/media/phase.py:113-191,
   src/lumen/media/spectra.py and src/lumen/media/emission.py:127-162. */
#ifndef LUMEN_ORACLE_MEDIA_H
#define LUMEN_ORACLE_MEDIA_H

#include "physics.h"

#define O_FOUR_PI 12.5663706143591729539f
#define O_DEFENSIVE 0.01f      /* the defensive mixture's share (src/lumen/rules/choices.py:113) */
/* its covering weight e / (1 - e), formed in double and rounded once to float32 (estimator.py:106) */
#define O_EDGE_SHARE ((float)(0.01 / (1.0 - 0.01)))
#define O_EPS32 1.1920928955078125e-7f
#define O_WLS_TRIES 100.0f     /* G4OpWLS's redraws of an energy below the absorbed one (spectra.py:22) */


/* ----------------------------------------------------------------------------------------- the Mie lobe */
/* (1 - mu, 1 + mu) of G4OpMieHG's Henyey-Greenstein draw at asymmetry g (phase.py:113 mie_hg_cos: the inverse CDF in
   a form whose factors are sums of positive terms) */
static inline void o_mie_hg_cos(float g, float r, float* cm, float* cp) {
  int up = g >= 0.0f;
  float d = up ? (1.0f - g) + 2.0f * g * r : (1.0f - g) * (1.0f - r) + (1.0f + g) * r;
  float one_gr = up ? 1.0f + g * r : (1.0f - r) + (1.0f + g) * r;
  float d2 = d * d;
  float omg = 1.0f - g, opg = 1.0f + g;
  *cm = 2.0f * (omg * omg) * (1.0f - r) * one_gr / d2;
  *cp = 2.0f * r * (opg * opg) * ((1.0f - g) + g * r) / d2;
}
/* HG(mu; g) per steradian from 1 - mu and 1 + mu, and d/dg (phase.py:139 hg_density) */
static inline float o_hg_density(float g, float cm, float cp, float* dg) {
  float omg = 1.0f - g, opg = 1.0f + g;
  float q = g >= 0.0f ? omg * omg + 2.0f * g * cm : opg * opg - 2.0f * g * cp;
  float sq = sqrtf(q);
  float q15 = q * sq;
  float h = omg * opg / (O_FOUR_PI * q15);
  if (dg) { /* dq/dg = 2 g - 2 mu in either form */
    float dq = g >= 0.0f ? -2.0f * omg + 2.0f * cm : 2.0f * opg - 2.0f * cp;
    *dg = (-2.0f * g * q - 1.5f * (omg * opg) * dq) / (O_FOUR_PI * q15 * q);
  }
  return h;
}
/* the direction at (1 - mu, 1 + mu) about wi, azimuth 2 pi u (phase.py:170 hg_direction) */
static inline void o_hg_direction(float cm, float cp, float u, const float* wi, float* wo) {
  float mu = cm < cp ? 1.0f - cm : cp - 1.0f;
  float s2 = cm * cp;
  float s = s2 > 0.0f ? sqrtf(s2) : 0.0f;
  float sp, cpp;
  o_sincos2pi(u, &sp, &cpp);
  float l[3] = {s * cpp, s * sp, mu};
  o_to_world(l, wi, wo);
}
/* G4OpMieHG's draw about wi with 3 uniforms: lobe, cosine, azimuth (phase.py:151 mie_hg_sample) */
static inline void o_mie_sample(float gf, float gb, float ratio, const float* wi, const float* rand, float* wo) {
  int fwd = rand[0] <= ratio;
  float cm, cp;
  o_mie_hg_cos(fwd ? gf : gb, rand[1], &cm, &cp);
  if (!fwd) { float t = cm; cm = cp; cp = t; }
  o_hg_direction(cm, cp, rand[2], wi, wo);
}
/* log density per steradian of the draw, both lobes (phase.py:185 mie_hg_logpdf), and its derivatives in
   (g_forward, g_backward, forward_ratio) when d is given */
static inline float o_mie_logpdf(float gf, float gb, float ratio, const float* wi, const float* wo, float* d) {
  float dm[3] = {wo[0] - wi[0], wo[1] - wi[1], wo[2] - wi[2]}, dp[3] = {wo[0] + wi[0], wo[1] + wi[1], wo[2] + wi[2]};
  float cm = 0.5f * o_dot(dm, dm), cp = 0.5f * o_dot(dp, dp);
  float dF, dB;
  float F = o_hg_density(gf, cm, cp, d ? &dF : 0);
  float B = o_hg_density(-gb, cm, cp, d ? &dB : 0);
  float mix = ratio * F + (1.0f - ratio) * B;
  if (d) {
    d[0] = ratio * dF / mix;
    d[1] = -((1.0f - ratio) * dB) / mix;
    d[2] = (F - B) / mix;
  }
  return o_log(mix);
}
/* the isotropic lobe about wi with 2 uniforms (phase.py:78 ISOTROPIC: mu = 1 - 2 u0, azimuth 2 pi u1) */
static inline void o_isotropic(const float* wi, float u0, float u1, float* wo) {
  float mu = 1.0f - 2.0f * u0;
  float s2 = 1.0f - mu * mu;
  float s = s2 > 0.0f ? sqrtf(s2) : 0.0f;
  float sp, cp;
  o_sincos2pi(u1, &sp, &cp);
  float l[3] = {s * cp, s * sp, mu};
  o_to_world(l, wi, wo);
}

/* ------------------------------------------------------------------------------- the WLS spectrum sampler */
/* Geant4's sampler of a spectrum table (spectra.py:47 g4_arrays), read interval by interval: e (k knots, eV) and s
   (intensities); with cover, the one defensive mixture over the intervals without mass (spectra.py:110 covered) */
typedef struct OSpec { const float* e; const float* s; int k; float tot, Z; int cover; } OSpec;

static inline OSpec o_spec(const float* e, const float* s, int k, int cover) {
  OSpec p = {e, s, k, 0.0f, 0.0f, 0};
  for (int j = 0; j + 1 < k; ++j) {
    float h = e[j + 1] - e[j];
    float m = 0.5f * (s[j + 1] + s[j]) * h;
    p.tot = j == 0 ? m : p.tot + m;
    if (s[j + 1] + s[j] <= 0.0f && h > 0.0f) p.Z = p.Z + h;
  }
  p.cover = cover && p.Z > 0.0f;
  return p;
}
/* the density of interval j (g4_arrays' d, or covered's d2) */
static inline float o_spec_d(const OSpec* p, int j) {
  float d = 0.5f * (p->s[j + 1] + p->s[j]) / p->tot;
  if (!p->cover) return d;
  float h = p->e[j + 1] - p->e[j];
  float z = (p->s[j + 1] + p->s[j] <= 0.0f && h > 0.0f) ? 1.0f : 0.0f;
  return (1.0f - O_DEFENSIVE) * d + O_DEFENSIVE * z / p->Z;
}
/* the CDF at the start of interval j+1 given the CDF at the start of j (g4_arrays' c: the cumulative mass over tot;
   covered's c2: the cumulative d2 h) */
static inline float o_spec_c_next(const OSpec* p, int j, float c_j, float* mass_acc) {
  float h = p->e[j + 1] - p->e[j];
  if (p->cover) return c_j + o_spec_d(p, j) * h;
  float m = 0.5f * (p->s[j + 1] + p->s[j]) * h;
  *mass_acc = j == 0 ? m : *mass_acc + m;
  return *mass_acc / p->tot;
}
/* the energy at a uniform r (spectra.py:60 invert: the last interval whose CDF start is <= r, uniform within it) */
static inline float o_spec_invert(const OSpec* p, float r) {
  int n = p->k - 1, kk = 0;
  float c = 0.0f, ck = 0.0f, acc = 0.0f;
  for (int j = 0; j < n; ++j) {
    if (c <= r) { kk = j; ck = c; }
    if (j + 1 < n) c = o_spec_c_next(p, j, c, &acc);
  }
  float d = o_spec_d(p, kk), h = p->e[kk + 1] - p->e[kk];
  float x = d > 0.0f ? o_max(r - ck, 0.0f) / d : 0.0f;
  x = x < 0.0f ? 0.0f : (x > h ? h : x);
  return p->e[kk] + x;
}
/* the mass at energies up to E (spectra.py:76 cumulative) */
static inline float o_spec_cumulative(const OSpec* p, float E) {
  int n = p->k - 1, kk = 0;
  float c = 0.0f, ck = 0.0f, acc = 0.0f;
  for (int j = 0; j < n; ++j) {
    if (p->e[j] <= E) { kk = j; ck = c; }
    if (j + 1 < n) c = o_spec_c_next(p, j, c, &acc);
  }
  float h = p->e[kk + 1] - p->e[kk];
  float t = E - p->e[kk];
  t = t < 0.0f ? 0.0f : (t > h ? h : t);
  float u = ck + o_spec_d(p, kk) * t;
  if (E < p->e[0]) return 0.0f;
  return u < 0.0f ? 0.0f : (u > 1.0f ? 1.0f : u);
}
/* the density (1/eV) on the interval holding E, 0 outside the knots (spectra.py:96 interval_density, :103
   on_intervals; covered: spectra.py:133 covered_interval_density) */
static inline float o_spec_density(const float* e, const float* s, int k, int cover, float E) {
  if (!(E >= e[0] && E <= e[k - 1])) return 0.0f;
  float tot = 0.0f, Z = 0.0f;
  for (int j = 0; j + 1 < k; ++j) {
    float t = (s[j + 1] + s[j]) * (e[j + 1] - e[j]);
    tot = j == 0 ? t : tot + t;
    float h = e[j + 1] - e[j];
    if (s[j + 1] + s[j] <= 0.0f && h > 0.0f) Z = Z + h;
  }
  int i = 0;
  for (int j = 0; j < k; ++j)
    if (e[j] <= E) i = j;
  i = i > k - 2 ? k - 2 : i;
  float p = (s[i] + s[i + 1]) / tot;
  if (!(cover && Z > 0.0f)) return p;
  float h = e[i + 1] - e[i];
  float z = (s[i + 1] + s[i] <= 0.0f && h > 0.0f) ? 1.0f : 0.0f;
  return (1.0f - O_DEFENSIVE) * p + O_DEFENSIVE * z / Z;
}
/* the chance that one of G4OpWLS's draws finds an energy at or below the absorbed one (spectra.py:25 kept) */
static inline float o_kept(float f) {
  float c = f < 0.0f ? 0.0f : (f > 1.0f - O_EPS32 ? 1.0f - O_EPS32 : f);
  return -o_expm1(O_WLS_TRIES * o_log1p(-c));
}
static inline float o_safe_div(float a, float b) { return b != 0.0f ? a / b : 0.0f; }

/* A G4OpWLS re-emission of a photon absorbed at lam_in (emission.py:136 EmissionRecord.sample): the wavelength drawn
   at the reference spectrum under the defensive cover, truncated at the absorbed energy by its exact inverse CDF;
   the weight the yield times the chance of an energy below the absorbed one times the live density over the one
   drawn from; the reference weight the same at the reference values. The delay: the time constant (delta) or an
   exponential of it. Spectra: (e, s, k) live and reference. */
typedef struct OEmit { float lam, delay, w, w_r, dyield; } OEmit;
static inline OEmit o_wls_emit(const float* el, const float* sl, int kl, const float* er_, const float* sr, int kr,
                               float yield_l, float yield_r, float tau, int exponential, float lam_in, float u_lam,
                               float u_t) {
  OEmit o;
  OSpec q = o_spec(er_, sr, kr, 1);
  float E_in = O_HC / lam_in;
  float f_q = o_spec_cumulative(&q, E_in);
  float energy_draw = o_spec_invert(&q, u_lam * f_q);
  o.lam = O_HC / energy_draw;
  float energy = O_HC / o.lam;
  float qd = o_spec_density(er_, sr, kr, 1, energy);
  float dens_q = o_safe_div(qd, f_q);
  /* the reference weight: at the reference values, the density drawn from over itself */
  float dr = o_kept(f_q) * o_safe_div(qd, f_q);
  o.w_r = yield_r * o_safe_div(dr, dens_q);
  /* the live weight: the live spectrum's sampler and density */
  OSpec l = o_spec(el, sl, kl, 0);
  float f_l = o_spec_cumulative(&l, E_in);
  float dl = o_kept(f_l) * o_safe_div(o_spec_density(el, sl, kl, 0, energy), f_l);
  float ratio = o_safe_div(dl, dens_q);
  o.w = yield_l * ratio;
  o.dyield = ratio;
  o.delay = exponential ? -tau * o_log(u_t) : tau + 0.0f * u_t;
  return o;
}

#endif
