/*
 * ORACLE (test infrastructure; only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline load it, and only as
 * the checker or the timed CPU baseline, never as the product path).
 *
 * A scalar C++ restatement of lumen's photon loop (src/lumen/run.py:293-368 `_loop` / `item` / `body`) over one
 * photon at a time: the step (src/lumen/transport/step.py:516 `step`, with `_recover` :245, `_step_context` :318,
 * `_surface_event` :362, `_bulk` :397, `_after` :464, `_advance` :495), the deposit reduction the reference does in
 * its records + rebuild launches (src/lumen/run.py:443-557, src/lumen/readout/fill.py:216: arrival, arrival_t,
 * arrival2), and the sources (src/lumen/sources/point.py:73, _base.py:312-322). FP64 tallies; OpenMP over photons.
 *
 * Derivatives are forward-mode tangents of the live weight at the reference values, one per gradient parameter
 * (a table whose values move together): the reference's reweighting estimator (src/lumen/transport/estimator.py)
 * differentiated along the fixed path, deposits' tangents summed per sensor.
 */
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "physics.h"
#include "media.h"
#include "rng.h"
#include "readout.h"

#define O_SOURCE_STREAM 0xFFFFFFFFu
#define O_POL_STREAM 0x9017u
#define O_NORMAL_LO -0.99999994039535522461f /* nextafter(-1, 0) in float32: jax.random.normal's bound */
#define O_SQRT2 1.41421356237309504880f
#define O_MAXG LUMEN_MAX_GRAD

typedef struct ORun {
  OScene S;
  const float* live;
  const float* ref;
  int shared; /* live == ref */
  float max_distance, roulette, reach;
  int max_vertices;
  int P;
  int gt[O_MAXG];
  int jump; /* LUMEN_F_JUMP */
  int analog; /* LUMEN_F_TRUTH */
} ORun;

/* NF: the position's precision, the navigator's (state.py:120 start's `position`); every other field float32 */
template <class NF>
struct OPhotonT {
  NF x[3];
  float d[3], t, lam, w, wr;
  int alive, vertex;
  float er[3], ei[3];
  int vol, srf;
  float sn[3];
  int nz, cls;
  int gen; /* re-emissions so far (state.py Photon.gen) */
  float dw[O_MAXG];
  /* the analog photon (truth rows, state.py:30 Analog): its place x in the weight (inf: decided), its weight k, and
     at its cathode absorption the sensor, time, wavelength, 1 / A_n, crossing point and volume entered */
  float ax, ak;
  int asensor;
  float atime, alam, ascale, apos[3];
  int avol;
};

typedef struct ODep {
  int sensor;
  float q, time, lam;
  float fates[8]; /* lost, abandoned, escaped, distance_cut, absorbed_bulk, absorbed_surface, rouletted, reweighted */
  float pushed;
  float dq[O_MAXG];
  ORec rec; /* at a sensor deposit: what the readout groups read (step.py:546) */
} ODep;

static inline float o_ratio(float live, float ref) { return ref != 0.0f ? live / ref : 0.0f; }

/* ------------------------------------------------------------------------------------------ the diffusion jump */
#define O_JUMP_STREAM 0x7A11u /* the vertex key's fold for the walk's own uniforms (rng.py:25) */
typedef struct OJump { int ok, n; float y[3], d[3], er[3], L; } OJump;

/* the walk at a bulk Rayleigh event inside the proven clear ball at xs (fastpath.py:174 diffuse): free paths at the
   reference rate, the polarised Rayleigh draw and projection, until a flight leaves the ball (the photon put at the
   crossing) or the budget ceil((c mu_r)^2) of scatterings is spent; identity where it does not apply */
static OJump o_diffuse(const LumenSceneDesc* D, int mi, const float* xs, const float* d0, const float* er0,
                       const float* ei0, float mu_r, int alive, OKey vkey) {
  OJump J;
  J.ok = 0; J.n = 0; J.L = 0.0f;
  for (int a = 0; a < 3; ++a) { J.y[a] = 0.0f; J.d[a] = d0[a]; J.er[a] = er0[a]; }
  int g = -1;
  for (int k = 0; k < D->n_jump; ++k)
    if (D->jump_i[(size_t)k * LUMEN_JUMP_I] == mi) g = k;
  if (g < 0) return J;
  const float* jf = D->jump_f + (size_t)g * LUMEN_JUMP_F;
  const int32_t* ji = D->jump_i + (size_t)g * LUMEN_JUMP_I;
  float h = jf[3];
  int inside = 1, idx[3];
  float node[3];
  for (int a = 0; a < 3; ++a) {
    float fi = (xs[a] - jf[a]) / h;
    int na = ji[1 + a];
    inside = inside && fi > -0.5f && fi < (float)na - 0.5f;
    int i = (int)floorf(fi + 0.5f);
    i = i < 0 ? 0 : (i > na - 1 ? na - 1 : i);
    idx[a] = i;
    node[a] = jf[a] + h * (float)i;
  }
  float dx[3] = {xs[0] - node[0], xs[1] - node[1], xs[2] - node[2]};
  float c = D->clear[ji[4] + ((int64_t)idx[0] * ji[2] + idx[1]) * ji[3] + idx[2]] - sqrtf(o_dot(dx, dx));
  int lin = ei0[0] == 0.0f && ei0[1] == 0.0f && ei0[2] == 0.0f;
  if (!(inside && c > 0.0f && lin && alive && mu_r > 0.0f)) return J;
  J.ok = 1;
  float cm = c * mu_r;
  int budget = (int)ceilf(o_min(cm * cm, (float)LUMEN_JUMP_STEPS));
  OKey jkey = o_fold_in(vkey, O_JUMP_STREAM);
  const float zero[3] = {0.0f, 0.0f, 0.0f};
  int out = 0;
  for (int j = 0; j < budget && !out; ++j) {
    OKey kj = o_fold_in(jkey, (uint32_t)j);
    float u0 = o_uniform(kj, 0);
    float u3[3] = {o_uniform(kj, 1), o_uniform(kj, 2), o_uniform(kj, 3)};
    float s = -o_log(u0) / mu_r;
    float by = o_dot(J.y, J.d);
    float t = -by + sqrtf(o_max(by * by - (o_dot(J.y, J.y) - c * c), 0.0f));
    out = s >= t;
    float k[3];
    o_rayleigh_sample(J.er, zero, u3, k);
    float e2[3] = {J.er[0], J.er[1], J.er[2]}, z2[3] = {0.0f, 0.0f, 0.0f};
    o_project(e2, z2, k);
    float st = out ? t : s;
    for (int a = 0; a < 3; ++a) J.y[a] = J.y[a] + st * J.d[a];
    J.L = J.L + st;
    if (!out) {
      for (int a = 0; a < 3; ++a) { J.d[a] = k[a]; J.er[a] = e2[a]; }
      J.n += 1;
    }
  }
  return J;
}

/* tangents of a medium's rates in the gradient parameters: d(1/L)/dL = -1/L^2 where L's table moves; per channel
   (dch, p-major) and their sum (dmu_c) */
static inline void o_dmed(const ORun* R, int mi, float lam, const OMed* m, float* dmu_abs, float* dmu_c, float* dch) {
  const int32_t* mr = R->S.D->med_i + (size_t)mi * LUMEN_MED_I;
  float E = O_HC / lam;
  for (int p = 0; p < R->P; ++p) {
    dmu_abs[p] = 0.0f;
    if (mr[LUMEN_MI_ABS] >= 0 && mr[LUMEN_MI_ABS] == R->gt[p]) {
      float L = o_tab(R->S.D, R->live, mr[LUMEN_MI_ABS], E, 0);
      dmu_abs[p] = L >= O_FLT_TINY ? -(m->mu_abs * m->mu_abs) : 0.0f;
    }
    for (int c = 0; c < LUMEN_N_CHANNEL; ++c) {
      int t = o_channel_tab(mr, c);
      float v = 0.0f;
      if (t >= 0 && t == R->gt[p]) {
        float L = o_tab(R->S.D, R->live, t, E, 0);
        v = L >= O_FLT_TINY ? -(m->ch[c] * m->ch[c]) : 0.0f;
      }
      dch[p * LUMEN_N_CHANNEL + c] = v;
    }
    dmu_c[p] = (dch[p * LUMEN_N_CHANNEL] + dch[p * LUMEN_N_CHANNEL + 1]) + dch[p * LUMEN_N_CHANNEL + 2];
  }
}

/* lumen 0.2.0's reference weight at a covered draw (lumen_oracle_set_rule_020): checker-only, so that the published
   run of that version can be reproduced; every engine path runs the current rule */
static int g_rule_020 = 0;

/* the first step of a photon born inside a sensor that counts by volume (step.py:574 _born): it deposits what the
   sensor's entry (row_of[bp][cls]) detects, evaluated unpolarised at normal incidence with both indices 1
   (step.py:589), at its emission time, and ends: its whole weight absorbed at a surface */
template <class NF>
static void o_born(const ORun* R, OPhotonT<NF>* ph, ODep* dep, int bp, int sensor) {
  const LumenSceneDesc* D = R->S.D;
  const int P = R->P;
  int row = D->row_of[bp * D->n_cls + ph->cls];
  float nrm[3] = {-ph->d[0], -ph->d[1], -ph->d[2]};
  float dcol[O_MAXG * LUMEN_N_COL], dprobs[O_MAXG * O_N_OUT], ddet[O_MAXG];
  for (int p = 0; p < P; ++p)
    for (int c = 0; c < LUMEN_N_COL; ++c)
      dcol[p * LUMEN_N_COL + c] =
          (row >= 0 && D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_COL + c] == R->gt[p]) ? 1.0f : 0.0f;
  OEval ev;
  o_type_eval(D, R->live, row, ph->lam, ph->d, nrm, 1.0f, 1.0f, 0, 0, &ev, P, dcol, dprobs, ddet);
  const float d = ev.detect;
  float inv_an = 1.0f;
  if (row >= 0 && D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_PER_NORMAL]) {
    float an = o_normal_absorptance(D, R->live, row, ph->lam, 1.0f, nrm);
    inv_an = an > 0.0f ? 1.0f / an : 0.0f;
  }
  dep->sensor = sensor;
  dep->q = ph->w * d;
  dep->time = ph->t;
  dep->lam = ph->lam;
  for (int p = 0; p < P; ++p) dep->dq[p] = ph->dw[p] * d + ph->w * ddet[p];
  ORec* rc = &dep->rec;
  rc->sensor = sensor;
  rc->q = dep->q;
  rc->time = ph->t;
  rc->lam = ph->lam;
  rc->gen = ph->gen;
  rc->vol = ph->vol;
  for (int a = 0; a < 3; ++a) { rc->x[a] = (float)ph->x[a]; rc->d[a] = ph->d[a]; rc->n[a] = nrm[a]; }
  rc->inv_an = inv_an;
  for (int k = 0; k < 8; ++k) dep->fates[k] = 0.0f;
  dep->fates[5] = ph->w;
  dep->pushed = 0.0f;
  if (R->analog) { /* step.py:597: the analog photon absorbed with the detected share, else decided */
    const float share = ph->w * d;
    if (ph->ax < share) {
      ph->asensor = sensor;
      ph->atime = ph->t;
      ph->alam = ph->lam;
      ph->ascale = inv_an;
      for (int a = 0; a < 3; ++a) ph->apos[a] = (float)ph->x[a];
      ph->avol = ph->vol;
    }
    ph->ax = INFINITY;
  }
  ph->alive = 0;
  ph->w = 0.0f;
  ph->wr = 0.0f;
  for (int p = 0; p < P; ++p) ph->dw[p] = 0.0f;
  ph->vertex += 1;
}

/* one step (step.py:516); NF the navigator's precision */
template <class NF>
static void o_step(const ORun* R, OPhotonT<NF>* ph, OKey pkey, ODep* dep) {
  const OScene* S = &R->S;
  const LumenSceneDesc* D = S->D;
  const int P = R->P;
  if (D->cls_born && ph->vertex == 0 && ph->alive && ph->vol >= 0) {
    const int bp = D->cls_born[ph->cls];
    const int sensor = D->vol_i[(size_t)ph->vol * LUMEN_VOL_I + LUMEN_VI_SENSOR];
    if (bp >= 0 && sensor >= 0) {
      o_born(R, ph, dep, bp, sensor);
      return;
    }
  }
  /* _recover: the stuck rule's push (step.py:245) */
  NF b0 = onav_band(onav_maxabs3(ph->x));
  int stuck = ph->alive && ph->nz >= O_ZSBP;
  if (stuck) {
    NF pb = O_PUSH_BANDS * b0;
    for (int a = 0; a < 3; ++a) ph->x[a] = ph->x[a] + pb * ph->d[a];
    ph->vol = onav_locate(S, ph->x);
    ph->cls = o_cls(S, ph->vol);
    ph->srf = -1;
  }
  OKey vkey = o_fold_in(pkey, (uint32_t)ph->vertex);
  float er0[3] = {ph->er[0], ph->er[1], ph->er[2]}, ei0[3] = {ph->ei[0], ph->ei[1], ph->ei[2]};
  if (o_dot(er0, er0) + o_dot(ei0, ei0) < O_ZERO_STATE)
    o_fill(ph->d, er0, ei0, o_uniform(o_fold_in(vkey, O_POL_STREAM), 0));
  int mi = D->cls_medium[ph->cls];
  OMed ml = o_medium_at(D, R->live, ph->lam, mi);
  OMed mr = R->shared ? ml : o_medium_at(D, R->ref, ph->lam, mi);
  float dmu_abs[O_MAXG], dmu_c[O_MAXG], dch[O_MAXG * LUMEN_N_CHANNEL];
  o_dmed(R, mi, ph->lam, &ml, dmu_abs, dmu_c, dch);
  float mu_r = mr.mu_c;
  float s = -o_log(o_uniform(vkey, 0)) / o_max(mu_r, O_FLOOR32);
  /* _query (step.py:260; TrackedGeometry.query, tracked.py:86) */
  const NF dd[3] = {ph->d[0], ph->d[1], ph->d[2]}; /* the direction in the navigator's precision (navigate.py:682) */
  OQueryT<NF> q = onav_query(S, ph->x, dd, ph->vol, (NF)R->max_distance, ph->srf, ph->sn, (NF)s);
  /* the sensor the deposit credits: the one entered, or at an exit sensor's crossing the one left, whose frame the
     deposit's local fields are read in (step.py:615 _sensor_dep, :653 sensor_frame) */
  const int v_sens = (D->pair_pre && q.hit && D->pair_pre[q.cls_before * D->n_cls + q.cls_after]) ? q.vol_before
                                                                                                  : q.vol_after;
  int sensor_q = (q.hit && v_sens >= 0) ? D->vol_i[(size_t)v_sens * LUMEN_VOL_I + LUMEN_VI_SENSOR] : -1;
  float dist = q.t;
  int zero = dist <= O_ZERO_STEP_BANDS * b0;
  /* _surface (step.py:280) */
  int cb = q.cls_before, ca = q.cls_after;
  int row = D->row_of[cb * D->n_cls + ca];
  int cont = (q.cont || (zero && row < 0)) && q.hit;
  if (cont) row = row > 0 ? row : 0;
  /* _crossing at the live values and the reference (step.py:305) */
  int mi_after = D->cls_medium[ca];
  float n2l = o_index_at(D, R->live, ph->lam, mi_after);
  float dcol[O_MAXG * LUMEN_N_COL], dprobs[O_MAXG * O_N_OUT], ddet[O_MAXG];
  for (int p = 0; p < P; ++p)
    for (int c = 0; c < LUMEN_N_COL; ++c)
      dcol[p * LUMEN_N_COL + c] =
          (row >= 0 && D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_COL + c] == R->gt[p]) ? 1.0f : 0.0f;
  OEval le, re;
  o_type_eval(D, R->live, row, ph->lam, ph->d, q.normal, ml.n, n2l, er0, ei0, &le, P, dcol, dprobs, ddet);
  if (R->shared) re = le;
  else {
    float n2r = o_index_at(D, R->ref, ph->lam, mi_after);
    o_type_eval(D, R->ref, row, ph->lam, ph->d, q.normal, mr.n, n2r, er0, ei0, &re, 0, 0, 0, 0);
  }
  if (cont) { /* a continue event: a straight pass, no deposit (step.py:298 _type_eval) */
    for (int o = 0; o < O_N_OUT; ++o) { le.probs[o] = o == O_STRAIGHT; re.probs[o] = o == O_STRAIGHT; }
    le.detect = 0.0f;
    re.detect = 0.0f;
    for (int p = 0; p < P; ++p) { for (int o = 0; o < O_N_OUT; ++o) dprobs[p * O_N_OUT + o] = 0.0f; ddet[p] = 0.0f; }
  }
  float p_draw[O_N_OUT], p_prop[O_N_OUT];
  for (int o = 0; o < O_N_OUT; ++o) p_draw[o] = re.probs[o];
  /* the one defensive mixture at an edge row (estimator.py:146 edge_floor, :83 defensive): each outcome of the row's
     support whose reference probability is 0 is drawn at e / (1 - e) / n (n of them); the stand-in row of a continue
     event included, as the reference reads it */
  const int cover = row >= 0 ? D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_COVER] : 0;
  if (cover) {
    int n_fl = 0;
    for (int o = 0; o < O_N_OUT; ++o) n_fl += ((cover >> o) & 1) && p_draw[o] <= 0.0f;
    if (n_fl) {
      const float eps = O_EDGE_SHARE / (float)n_fl;
      for (int o = 0; o < O_N_OUT; ++o)
        if (((cover >> o) & 1) && p_draw[o] <= 0.0f) p_draw[o] = eps;
    }
  }
  float tot = 0.0f;
  for (int o = 0; o < O_N_OUT; ++o) tot = o == 0 ? p_draw[0] : tot + p_draw[o];
  for (int o = 0; o < O_N_OUT; ++o) p_prop[o] = tot > 0.0f ? p_draw[o] / tot : 0.0f;
  int oc_ = o_choose(p_prop, O_N_OUT, o_uniform(vkey, 2));
  int os_ = oc_ > 0 ? oc_ : 0;
  int drawn = oc_ >= 0;
  float mu = ml.mu_c;
  float reach_live = o_exp(-mu * dist), reach_ref = o_exp(-mu_r * dist);
  float att_if = o_exp(-ml.mu_abs * dist), att_r = o_exp(-mr.mu_abs * dist);
  int scatter = mu_r > 0.0f && s < dist && ph->alive;
  float v_g = O_C_VACUUM / ml.ng;
  /* tangents of the crossing's factors */
  float d_reach[O_MAXG], d_att[O_MAXG];
  for (int p = 0; p < P; ++p) {
    d_reach[p] = -(dmu_c[p] * dist) * reach_live;
    d_att[p] = -(dmu_abs[p] * dist) * att_if;
  }
  /* step.py:521-526: the deposit and the lost weight */
  int at_if = q.hit && ph->alive && row >= 0;
  float p_det = le.detect;
  float rr = o_ratio(reach_live, reach_ref);
  dep->q = at_if ? ph->w * reach_live * att_if * p_det : 0.0f;
  for (int p = 0; p < P; ++p) {
    float f = reach_live * att_if * p_det;
    float df = d_reach[p] * att_if * p_det + reach_live * d_att[p] * p_det + reach_live * att_if * ddet[p];
    dep->dq[p] = at_if ? ph->dw[p] * f + ph->w * df : 0.0f;
  }
  float lost = (q.hit && ph->alive && row < 0 && !scatter) ? ph->w * rr * att_if : 0.0f;
  /* _event: a bulk event or the drawn surface outcome (step.py:439) */
  NF nx_x[3];
  float nx_d[3], nx_w, nx_dtime, nx_sn[3], nx_er[3], nx_ei[3], nx_lam = ph->lam;
  int nx_gen = ph->gen;
  float nx_dw[O_MAXG];
  int nx_cls, nx_ok, nx_far = 0;
  float fates0, fates1, fates2, wr;
  if (scatter) { /* _bulk (step.py:397) */
    int next_cls = s < q.t_pass0 ? q.cls_start : (s > q.t_pass1 ? cb : o_cls(S, q.vol_at));
    /* the channel drawn from the reference rates (estimator.choose, uniform 1); with one channel present it is that
       channel whatever the uniform */
    int n_ch = (mr.ch[0] > 0.0f) + (mr.ch[1] > 0.0f) + (mr.ch[2] > 0.0f);
    int cs = n_ch > 1 ? o_choose(mr.ch, LUMEN_N_CHANNEL, o_uniform(vkey, 1)) : (mr.ch[0] > 0.0f ? 0 : (mr.ch[1] > 0.0f ? 1 : 2));
    cs = cs < 0 ? 0 : cs;
    float mu_c_r = mr.ch[cs];
    float e_r = o_exp(-mu_r * s), e_l = o_exp(-mu * s);
    float path_r = mu_c_r * e_r;
    float w_path = o_ratio(ml.ch[cs] * e_l, path_r);
    float att = o_exp(-ml.mu_abs * s);
    float w = w_path * att;
    float w_r = o_ratio(path_r, path_r) * o_exp(-mr.mu_abs * s);
    for (int a = 0; a < 3; ++a) nx_x[a] = ph->x[a] + s * ph->d[a];
    float rl3[3] = {o_uniform(vkey, 3), o_uniform(vkey, 4), o_uniform(vkey, 5)};
    float rlw = 1.0f, y_w = 1.0f, y_r = 1.0f, delay = 0.0f;
    float dlob[O_MAXG], dyld[O_MAXG];
    for (int p = 0; p < P; ++p) { dlob[p] = 0.0f; dyld[p] = 0.0f; }
    const int32_t* mrec = D->med_i + (size_t)mi * LUMEN_MED_I;
    float Eph = O_HC / ph->lam;
    OJump J;
    J.ok = 0;
    if (cs == 0) { /* Rayleigh: the polarised dipole draw, the state projected (phase.py:57) */
      o_rayleigh_sample(er0, ei0, rl3, nx_d);
      for (int a = 0; a < 3; ++a) { nx_er[a] = er0[a]; nx_ei[a] = ei0[a]; }
      o_project(nx_er, nx_ei, nx_d);
      if (R->jump) { /* the diffusion jump (step.py:421): the walk's factor on the weight, its time on the clock */
        const float xs[3] = {(float)nx_x[0], (float)nx_x[1], (float)nx_x[2]}; /* the grids are float32 (fastpath.py:177) */
        J = o_diffuse(D, mi, xs, nx_d, nx_er, nx_ei, mu_r, ph->alive, vkey);
        if (J.ok) {
          for (int a = 0; a < 3; ++a) { nx_x[a] = nx_x[a] + J.y[a]; nx_d[a] = J.d[a]; nx_er[a] = J.er[a]; }
        }
      }
    } else if (cs == 1) { /* Mie (G4OpMieHG): drawn at the reference constants, weighted live / reference */
      int tg[3] = {mrec[LUMEN_MI_MIE_GF], mrec[LUMEN_MI_MIE_GB], mrec[LUMEN_MI_MIE_R]};
      float pl[3], pr[3];
      for (int k = 0; k < 3; ++k) {
        pl[k] = o_tab(D, R->live, tg[k], Eph, 0);
        pr[k] = R->shared ? pl[k] : o_tab(D, R->ref, tg[k], Eph, 0);
      }
      /* a covered lobe choice (medium.py:96 channel_draw): drawn at the forward ratio's defensive cover
         (phase.py:173 _mie_cover: estimator.py:101 defensive_q over (r, 1 - r), both covered), weighted live / cover */
      const float r0 = pr[2];
      if (mrec[LUMEN_MI_MIE_COVER] == 1 && !(r0 > 0.0f && 1.0f - r0 > 0.0f)) {
        float q0 = r0 > 0.0f ? r0 : O_EDGE_SHARE, q1 = 1.0f - r0 > 0.0f ? 1.0f - r0 : O_EDGE_SHARE;
        pr[2] = q0 / (q0 + q1);
      }
      o_mie_sample(pr[0], pr[1], pr[2], ph->d, rl3, nx_d);
      float dl[3];
      float lp = o_mie_logpdf(pl[0], pl[1], pl[2], ph->d, nx_d, dl);
      if (!R->shared || pr[2] != r0) rlw = o_exp(lp - o_mie_logpdf(pr[0], pr[1], pr[2], ph->d, nx_d, 0));
      for (int p = 0; p < P; ++p)
        for (int k = 0; k < 3; ++k)
          if (tg[k] == R->gt[p]) dlob[p] = dlob[p] + dl[k];
      for (int a = 0; a < 3; ++a) { nx_er[a] = er0[a]; nx_ei[a] = ei0[a]; }
      o_project(nx_er, nx_ei, nx_d);
    } else { /* WLS (G4OpWLS): isotropic, unpolarised, re-emitted at the record's wavelength after its delay */
      o_isotropic(ph->d, rl3[0], rl3[1], nx_d);
      for (int a = 0; a < 3; ++a) { nx_er[a] = 0.0f; nx_ei[a] = 0.0f; }
      int ts = mrec[LUMEN_MI_WLS_SPEC], ty = mrec[LUMEN_MI_WLS_YIELD], tt = mrec[LUMEN_MI_WLS_TAU];
      const float* pl_ = R->live + D->tab[2 * ts];
      const float* pr_ = R->ref + D->tab[2 * ts];
      int ks = D->tab[2 * ts + 1];
      float yl = o_tab(D, R->live, ty, Eph, 0), yr = R->shared ? yl : o_tab(D, R->ref, ty, Eph, 0);
      float tau = o_tab(D, R->live, tt, Eph, 0);
      OEmit em = o_wls_emit(pl_, pl_ + ks, ks, pr_, pr_ + ks, ks, yl, yr, tau, mrec[LUMEN_MI_WLS_PROFILE] == 1, ph->lam,
                            o_uniform(vkey, 7), o_uniform(vkey, 8));
      y_w = em.w;
      y_r = em.w_r;
      delay = em.delay;
      nx_lam = em.lam;
      nx_gen = ph->gen + 1; /* medium.py:126: the WLS channel re-emits */
      for (int p = 0; p < P; ++p)
        if (ty == R->gt[p]) dyld[p] = em.dyield;
    }
    float w_at = ph->w * w_path;
    fates0 = w_at * att * y_w;
    fates1 = w_at * (1.0f - att * y_w);
    fates2 = 0.0f;
    nx_w = ph->w * w * rlw * y_w;
    float wj = 1.0f;
    if (J.ok) { /* the walk's likelihood ratio (fastpath.py:212): its absorption and its path, live over reference */
      float lr = o_log(o_max(mu, O_FLOOR32) / o_max(mu_r, O_FLOOR32));
      wj = o_exp(-ml.mu_abs * J.L) * o_exp((float)J.n * lr - (mu - mu_r) * J.L);
      fates1 = fates1 + fates0 * (1.0f - wj);
      fates0 = fates0 * wj;
      nx_w = nx_w * wj;
    }
    for (int p = 0; p < P; ++p) {
      float dwp = (dch[p * LUMEN_N_CHANNEL + cs] * e_l + ml.ch[cs] * (-(dmu_c[p] * s) * e_l)) / path_r;
      if (!(path_r != 0.0f)) dwp = 0.0f;
      float datt = -(dmu_abs[p] * s) * att;
      float dwf = dwp * att + w_path * datt;
      if (cs == 0) nx_dw[p] = ph->dw[p] * w + ph->w * dwf;
      else nx_dw[p] = (ph->dw[p] * w + ph->w * dwf) * rlw * y_w + ph->w * w * rlw * (dlob[p] * y_w + dyld[p]);
      if (J.ok) {
        float dlr = mu > O_FLOOR32 ? dmu_c[p] / mu : 0.0f;
        float dwj = wj * (-(dmu_abs[p] * J.L) + (float)J.n * dlr - dmu_c[p] * J.L);
        nx_dw[p] = nx_dw[p] * wj + ph->w * w * dwj;
      }
    }
    nx_cls = next_cls;
    nx_ok = 1;
    nx_dtime = s / v_g + delay;
    if (J.ok) nx_dtime = nx_dtime + J.L / v_g;
    for (int a = 0; a < 3; ++a) nx_sn[a] = q.normal[a];
    wr = ph->wr * w_r * y_r;
    if (J.ok) wr = wr * o_exp(-mr.mu_abs * J.L);
  } else { /* _surface_event (step.py:362) */
    float pl = le.probs[os_], pp = p_prop[os_];
    float r_live = drawn ? (pp != 0.0f ? pl / pp : 0.0f) : 0.0f;
    float w_if = ph->w * rr * att_if * r_live;
    float dirn[3], wi[3] = {ph->d[0], ph->d[1], ph->d[2]};
    const float* nrm = q.normal;
    float eta = ml.n / n2l;
    float out_w = 1.0f, out_wd = 1.0f, lobe_dls = 0.0f, lobe_sign = 1.0f; /* GLISUR: r = 1 - polish */
    int out_far = 0;
    float s_ax[3];
    o_s_axis(wi, nrm, s_ax);
    Oc es, ep;
    o_components(er0, ei0, wi, s_ax, &es, &ep);
    for (int a = 0; a < 3; ++a) { nx_er[a] = er0[a]; nx_ei[a] = ei0[a]; }
    switch (os_) {
      case O_REFRACT: {
        float cos_i = -o_dot(wi, nrm);
        float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
        int tir = sin2_t >= 1.0f;
        float ct2 = 1.0f - sin2_t;
        float cos_t = ct2 > 0.0f ? sqrtf(ct2) : 0.0f;
        if (tir) {
          for (int a = 0; a < 3; ++a) dirn[a] = wi[a] + 2.0f * cos_i * nrm[a];
        } else {
          float k = eta * cos_i - cos_t;
          for (int a = 0; a < 3; ++a) dirn[a] = eta * wi[a] + k * nrm[a];
          o_unit(dirn);
        }
        float du[3] = {dirn[0], dirn[1], dirn[2]};
        o_unit(du);
        o_recombine(es, ep, le.amps[2], le.amps[3], s_ax, du, nx_er, nx_ei);
        break;
      }
      case O_SPECULAR: {
        float wn = o_dot(wi, nrm);
        for (int a = 0; a < 3; ++a) dirn[a] = wi[a] - 2.0f * wn * nrm[a];
        float du[3] = {dirn[0], dirn[1], dirn[2]};
        o_unit(du);
        o_recombine(es, ep, le.amps[0], le.amps[1], s_ax, du, nx_er, nx_ei);
        break;
      }
      case O_BACKSCATTER:
        for (int a = 0; a < 3; ++a) { dirn[a] = -wi[a]; nx_er[a] = -er0[a]; nx_ei[a] = -ei0[a]; }
        break;
      case O_DIFFUSE: {
        o_lambert(nrm, o_uniform(vkey, 3), o_uniform(vkey, 4), dirn);
        float h[3] = {dirn[0] - wi[0], dirn[1] - wi[1], dirn[2] - wi[2]};
        o_unit(h);
        o_mirror(nx_er, nx_ei, h);
        break;
      }
      case O_GLOSSY: {
        float rl3[3] = {o_uniform(vkey, 3), o_uniform(vkey, 4), o_uniform(vkey, 5)};
        int capped = 0;
        int gl = D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_GLISUR];
        if (gl == 0) { /* the unified facet path drawn at the reference width, weighted by its path density live over
                          reference (surface_event.py:106 _facet_path_branch): 1 without a reference, whose
                          derivative is the path's score in sigma */
          float lp = 0.0f, lr = 0.0f;
          int dens = !R->shared || P > 0;
          o_facet_path(re.sigma, wi, nrm, rl3, dirn, nx_er, nx_ei, &capped, dens ? D->unified : 0, le.sigma,
                       !R->shared, &lp, &lr, P > 0 ? &lobe_dls : 0);
          if (!R->shared) out_w = o_exp(lp - lr);
        } else if (gl == 1) { /* GLISUR metal: drawn from the cover at the reference width (1 - polish), weighted by
                                 the exact path density over the cover's; the drawn weight is the cover's support */
          out_w = o_glisur_metal_path(re.sigma, le.sigma, wi, nrm, rl3, O_GLISUR_COVER, dirn, nx_er, nx_ei, &capped,
                                      &out_wd, &lobe_dls);
          lobe_sign = -1.0f;
        } else { /* GLISUR dielectric: each facet reflects or refracts at the live indices, possibly ending beyond */
          out_w = o_glisur_dielectric_path(re.sigma, le.sigma, ml.n, n2l, wi, nrm, rl3, O_GLISUR_COVER, dirn, nx_er,
                                           nx_ei, &out_far, &capped, &out_wd, &lobe_dls);
          lobe_sign = -1.0f;
        }
        break;
      }
      default:
        for (int a = 0; a < 3; ++a) dirn[a] = wi[a];
        break;
    }
    for (int a = 0; a < 3; ++a) nx_d[a] = dirn[a];
    o_unit(nx_d);
    int far_side = (os_ == O_STRAIGHT || os_ == O_REFRACT);
    int far_ = (far_side || out_far) && drawn;
    int ok = q.hit && drawn && row >= 0;
    for (int a = 0; a < 3; ++a) nx_x[a] = ph->x[a] + q.t * ph->d[a];
    float r_o = drawn ? (p_prop[os_] != 0.0f ? p_draw[os_] / p_prop[os_] : 0.0f) : 0.0f;
    if (g_rule_020 && drawn && cover) { /* lumen 0.2.0: a covered draw at a surface absorbing every photon at the
                                           reference left the reference weight as it was (CHANGELOG.md, 0.2.1) */
      float s0 = 0.0f;
      for (int o = 0; o < O_N_OUT; ++o) s0 += re.probs[o];
      if (s0 <= 0.0f) r_o = 1.0f;
    }
    wr = ph->wr * (reach_ref != 0.0f ? 1.0f : 0.0f) * att_r * r_o * out_wd;
    float w_at = ph->w * rr;
    float s_cont = 0.0f;
    for (int o = 0; o < O_N_OUT; ++o) s_cont = o == 0 ? le.probs[0] : s_cont + le.probs[o];
    fates0 = ok ? w_at * att_if * s_cont : 0.0f;
    fates1 = q.hit ? w_at * (1.0f - att_if) : 0.0f;
    fates2 = (q.hit && row >= 0) ? w_at * att_if * (1.0f - s_cont) : 0.0f;
    nx_w = w_if * out_w;
    for (int p = 0; p < P; ++p) {
      float dpl = dprobs[p * O_N_OUT + os_];
      float dr_live = drawn ? (pp != 0.0f ? dpl / pp : 0.0f) : 0.0f;
      float drr = reach_ref != 0.0f ? d_reach[p] / reach_ref : 0.0f;
      float X = rr * att_if * r_live;
      float dX = drr * att_if * r_live + rr * d_att[p] * r_live + rr * att_if * dr_live;
      float dwid = lobe_sign > 0.0f ? dcol[p * LUMEN_N_COL + LUMEN_COL_SIGMA] : -dcol[p * LUMEN_N_COL + LUMEN_COL_POLISH];
      nx_dw[p] = (ph->dw[p] * X + ph->w * dX) * out_w + w_if * out_w * (lobe_dls * dwid);
    }
    nx_cls = far_ ? ca : cb;
    nx_ok = ok;
    nx_dtime = dist / v_g;
    for (int a = 0; a < 3; ++a) nx_sn[a] = q.normal[a];
    nx_far = far_;
  }
  /* step.py:529-542: the weights that end here */
  float a_surf = ph->alive ? fates2 : 0.0f;
  int far_end = ph->alive && !q.hit && !scatter;
  float d_end = o_min(dist, R->max_distance);
  float w_far = ph->w * o_ratio(o_exp(-mu * d_end), o_exp(-mu_r * d_end));
  float att_far = o_exp(-ml.mu_abs * d_end);
  int cut = R->max_distance < R->reach;
  float escaped = (far_end && !cut) ? w_far * att_far : 0.0f;
  float distance_cut = (far_end && cut) ? w_far * att_far : 0.0f;
  float a_bulk = (ph->alive ? fates1 : 0.0f) + (far_end ? w_far * (1.0f - att_far) : 0.0f);
  float reweighted = (ph->alive && nx_ok) ? fates0 - nx_w : 0.0f;
  float time = ph->t + dist / v_g;
  /* _after: the roulette and the stuck rule (step.py:464) */
  float w_new = nx_w;
  int low = wr < R->roulette;
  float p_s = wr / R->roulette;
  int keep = 0;
  if (R->analog) {
    /* step.py:625 _analog_crossing: the analog photon is absorbed where x falls in the crossing's reached share;
       past the weight the event leaves its fate was another loss (decided) */
    const float share = (at_if && !scatter) ? ph->w * att_if * p_det : 0.0f;
    if (ph->ax < share) {
      ph->asensor = at_if ? sensor_q : -1;
      ph->atime = time;
      ph->alam = ph->lam;
      ph->ascale = 1.0f;
      if (row >= 0 && D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_PER_NORMAL]) {
        const float an = o_normal_absorptance(D, R->live, row, ph->lam, ml.n, q.normal);
        ph->ascale = an > 0.0f ? 1.0f / an : 0.0f;
      }
      for (int a = 0; a < 3; ++a) ph->apos[a] = (float)(ph->x[a] + q.t * ph->d[a]);
      ph->avol = v_sens;
      ph->ax = INFINITY;
    } else {
      const float left = ph->ax - share;
      ph->ax = left < nx_w ? left : INFINITY;
    }
    /* step.py:649 _analog_roulette: kept while the analog fate is open, so that the keep's total is p_s */
    const float pi = wr * ph->ak;
    const float extra = (p_s - pi) / (pi < 1.0f ? 1.0f - pi : 1.0f);
    if (low) keep = std::isfinite(ph->ax) || o_uniform(vkey, 6) < extra;
  } else if (low) {
    keep = o_uniform(vkey, 6) < p_s;
  }
  int kept = low && keep, lostr = low && !keep;
  float p_kept = kept ? p_s : 1.0f;
  if (R->analog && kept && std::isfinite(ph->ax)) ph->ax = ph->ax / p_kept;
  float w_in = w_new;
  w_new = kept ? w_new / p_kept : (lostr ? 0.0f : w_new);
  float rouletted = (ph->alive && nx_ok) ? w_in - w_new : 0.0f;
  float wr_new = kept ? wr / p_kept : (lostr ? 0.0f : wr);
  int alive = ph->alive && nx_ok && !lostr;
  int nz_new = (q.hit && !scatter && dist <= O_ZERO_STEP_BANDS * b0) ? ph->nz + 1 : 0;
  int abandon = alive && nz_new >= O_ZSBK;
  float abandoned = abandon ? w_new : 0.0f;
  alive = alive && !abandon;
  float dw_new[O_MAXG];
  for (int p = 0; p < P; ++p) dw_new[p] = kept ? nx_dw[p] / p_kept : (lostr ? 0.0f : nx_dw[p]);
  /* _advance (step.py:495) */
  int vol_b = s < q.t_pass0 ? q.vol_start : (s > q.t_pass1 ? q.vol_before : q.vol_at);
  int vol = scatter ? vol_b : (nx_far ? q.vol_after : q.vol_before);
  int held = scatter && s <= O_ZERO_STEP_BANDS * b0 && ph->srf >= 0;
  int srf = held ? ph->srf : ((scatter || !q.hit) ? -1 : q.srf);
  float pushed = (ph->alive && ph->nz == O_ZSBP) ? ph->w : 0.0f;
  /* the deposit */
  dep->sensor = at_if ? sensor_q : -1;
  dep->time = time;
  dep->lam = ph->lam;
  if (dep->sensor >= 0) { /* step.py:687 _local: the crossing point, direction and normal; the sensor's volume */
    ORec* rc = &dep->rec;
    rc->sensor = dep->sensor;
    rc->q = dep->q;
    rc->time = time;
    rc->lam = ph->lam;
    rc->gen = ph->gen;
    rc->vol = v_sens;
    for (int a = 0; a < 3; ++a) { rc->x[a] = (float)(ph->x[a] + q.t * ph->d[a]); rc->d[a] = ph->d[a]; rc->n[a] = q.normal[a]; }
    rc->inv_an = 1.0f;
    if (row >= 0 && D->row_i[(size_t)row * LUMEN_ROW_I + LUMEN_RI_PER_NORMAL]) {
      float an = o_normal_absorptance(D, R->live, row, ph->lam, ml.n, q.normal);
      rc->inv_an = an > 0.0f ? 1.0f / an : 0.0f;
    }
  }
  dep->fates[0] = lost;
  dep->fates[1] = abandoned;
  dep->fates[2] = escaped;
  dep->fates[3] = distance_cut;
  dep->fates[4] = a_bulk;
  dep->fates[5] = a_surf;
  dep->fates[6] = rouletted;
  dep->fates[7] = reweighted;
  dep->pushed = pushed;
  /* the photon after the step */
  for (int a = 0; a < 3; ++a) { ph->x[a] = nx_x[a]; ph->d[a] = nx_d[a]; ph->er[a] = nx_er[a]; ph->ei[a] = nx_ei[a]; }
  ph->t = ph->t + nx_dtime;
  ph->lam = nx_lam;
  ph->gen = nx_gen;
  ph->w = alive ? w_new : 0.0f;
  ph->wr = alive ? wr_new : 0.0f;
  for (int p = 0; p < P; ++p) ph->dw[p] = alive ? dw_new[p] : 0.0f;
  ph->alive = alive;
  ph->vertex += 1;
  ph->vol = vol;
  ph->srf = srf;
  if (!held) for (int a = 0; a < 3; ++a) ph->sn[a] = nx_sn[a];
  ph->nz = nz_new;
  ph->cls = nx_cls;
}

/* ------------------------------------------------------------------------------------------------ sources */
typedef struct ORow { float x[3], d[3], t, lam, w0, er[3], ei[3]; int event; } ORow;

/* gaussian from a uniform (sources/_base.py:318): jax.random.normal's map of the same bits */
static inline float o_gaussian(float u) {
  float f = u - 5.9604644775390625e-8f;
  float v = f * (1.0f - O_NORMAL_LO) + O_NORMAL_LO;
  v = v > O_NORMAL_LO ? v : O_NORMAL_LO;
  return O_SQRT2 * o_erfinv(v);
}

static int o_event_of(const int64_t* first, int n_ev, int64_t gid) {
  int lo = 0, hi = n_ev - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (first[mid] <= gid) lo = mid; else hi = mid - 1;
  }
  return lo;
}

/* photon gid of a procedural source (uniforms of vertex 0 of its own key under the source stream) */
/* 2 pi alpha for Frank-Tamm (units.py:16 FINE_STRUCTURE): the product in double, rounded once */
static const float O_TWO_PI_ALPHA = (float)(6.283185307179586 * (1.0 / 137.035999084));

/* a material's scintillation photon (scintillation.py:69 flash; shares :48; the component's defensive draw,
   estimator.py:101, and _base.py:298 lit; the wavelength _base.py:337; the delays emission.py:48) */
static void o_scint_shares(const LumenSceneDesc* D, const float* pool, const int32_t* m, float* f) {
  float y[3];
  for (int i = 0; i < 3; ++i) {
    int t = m[LUMEN_SM_SHARE + i];
    y[i] = t >= 0 ? o_tab(D, pool, t, 1.0f, 0) : (i == 0 ? 1.0f : 0.0f);
  }
  const float s = (y[0] + y[1]) + y[2];
  f[0] = 1.0f; f[1] = 0.0f; f[2] = 0.0f;
  if (m[LUMEN_SM_N] == 2) { f[0] = y[0] / s; f[1] = 1.0f - y[0] / s; }
  if (m[LUMEN_SM_N] == 3) for (int i = 0; i < 3; ++i) f[i] = y[i] / s;
}

static void o_scint_row(const LumenSceneDesc* D, const float* live, const float* ref, const LumenSource* src,
                        const float* f, OKey rk, ORow* r) {
  const int32_t* m = src->mat;
  const int nc = m[LUMEN_SM_N], seg = m[LUMEN_SM_SEGMENT];
  float fl[3], q[3];
  o_scint_shares(D, live, m, fl);
  o_scint_shares(D, ref, m, q);
  int zeros = 0;
  for (int i = 0; i < nc; ++i) zeros += q[i] <= 0.0f ? 1 : 0;
  if (zeros) {
    const float eps = (float)(0.01 / 0.99) / (float)zeros;
    float tot = 0.0f;
    for (int i = 0; i < nc; ++i) {
      if (q[i] <= 0.0f) q[i] = eps;
      tot = i == 0 ? q[i] : tot + q[i];
    }
    for (int i = 0; i < nc; ++i) q[i] = q[i] / tot;
  }
  float u_lam = o_uniform(rk, 0), u_z = o_uniform(rk, 1), u_phi = o_uniform(rk, 2), u_comp = o_uniform(rk, 3);
  float u_time = o_uniform(rk, 4);
  int c = 0;
  float cum = 0.0f;
  for (int i = 0; i < nc - 1; ++i) {
    cum = i == 0 ? q[0] : cum + q[i];
    if (u_comp >= cum) ++c;
  }
  int first_lit = nc, last_lit = 0;
  for (int i = 0; i < nc; ++i) {
    if (q[i] > 0.0f) last_lit = i;
    if (q[i] > 0.0f && i >= c && first_lit == nc) first_lit = i;
  }
  c = first_lit < last_lit ? first_lit : last_lit;
  const int ts = m[LUMEN_SM_SPEC + c];
  const float* kr = ref + D->tab[2 * ts];
  const float* kl = live + D->tab[2 * ts];
  const int k = D->tab[2 * ts + 1];
  OSpec qs = o_spec(kr, kr + k, k, 1);
  r->lam = O_HC / o_spec_invert(&qs, u_lam);
  const float energy = O_HC / r->lam;
  const float wt = o_safe_div(o_spec_density(kl, kl + k, k, 0, energy), o_spec_density(kr, kr + k, k, 1, energy));
  const float z = 1.0f - 2.0f * u_z;
  const float sz = 1.0f - z * z;
  const float rho = sz > 0.0f ? sqrtf(sz) : 0.0f;
  float sp, cp;
  o_sincos2pi(u_phi, &sp, &cp);
  r->d[0] = rho * cp; r->d[1] = rho * sp; r->d[2] = z;
  const float tau = o_tab(D, live, m[LUMEN_SM_TAU + c], 1.0f, 0);
  float delay = -tau * o_log(u_time);
  if (m[LUMEN_SM_RISES]) {
    const float rise = o_tab(D, live, m[LUMEN_SM_RISE + c], 1.0f, 0);
    const float s = tau + rise;
    delay = delay + -(tau * rise / (s > 0.0f ? s : 1.0f)) * o_log(o_uniform(rk, 5 + seg));
  }
  const float yl = o_tab(D, live, m[LUMEN_SM_YIELD], 1.0f, 0);
  const float edep = f[8], birks = f[9];
  float n_ph = yl * edep;
  if (seg) { /* Birks' law along the segment (scintillation.py:42 visible_energy) */
    float v[3] = {f[4] - f[0], f[5] - f[1], f[6] - f[2]};
    float len = sqrtf((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
    float quench = 1.0f + birks * edep / (len > 0.0f ? len : 1.0f);
    n_ph = yl * ((len > 0.0f && edep > 0.0f) ? edep / quench : (edep > 0.0f ? edep : 0.0f));
  }
  r->w0 = n_ph / f[10] * o_safe_div(fl[c], q[c]) * wt;
  if (seg) {
    const float u = o_uniform(rk, 5);
    for (int a = 0; a < 3; ++a) r->x[a] = f[a] + u * (f[4 + a] - f[a]);
    r->t = f[3] + u * (f[7] - f[3]) + delay;
  } else {
    for (int a = 0; a < 3; ++a) r->x[a] = f[a];
    r->t = f[3] + delay;
  }
}

static void o_source_row(const LumenSceneDesc* D, const float* pool, const float* ref, const LumenSource* src,
                         OKey key, int64_t gid, ORow* r) {
  OKey sk = o_fold_in(key, O_SOURCE_STREAM);
  OKey rk = o_fold_in(o_fold_in(sk, (uint32_t)gid), 0u);
  int e = o_event_of(src->ev_first, src->n_events, gid);
  const float* f = src->ev_f + (size_t)e * LUMEN_EV_F;
  r->event = e;
  r->w0 = src->ev_w[e];
  for (int a = 0; a < 3; ++a) { r->er[a] = 0.0f; r->ei[a] = 0.0f; }
  if (src->kind == LUMEN_SRC_TRACK) {
    float u0 = o_uniform(rk, 0), u1 = o_uniform(rk, 1), u2 = o_uniform(rk, 2);
    const float* ax = f + 3;
    float along = u0 * f[6];
    for (int a = 0; a < 3; ++a) r->x[a] = f[a] + along * ax[a];
    float c = src->cone_cos;
    float sn = sqrtf(1.0f - c * c);
    float sp, cp;
    o_sincos2pi(u1, &sp, &cp);
    float l[3] = {sn * cp, sn * sp, c};
    o_to_world(l, ax, r->d);
    r->t = f[7] + along / O_C_VACUUM;
    r->lam = src->lam1 > src->lam0 ? src->lam0 + (src->lam1 - src->lam0) * u2 : src->lam0;
    /* Cherenkov polarisation: in the plane of the axis and d, perpendicular to d (polar.py:89 cherenkov) */
    float ad = o_dot(ax, r->d);
    for (int a = 0; a < 3; ++a) r->er[a] = ad * r->d[a] - ax[a];
    o_unit(r->er);
    return;
  }
  if (src->kind == LUMEN_SRC_SCINT_MATERIAL) {
    o_scint_row(D, pool, ref, src, f, rk, r);
    return;
  }
  if (src->kind == LUMEN_SRC_CHERENKOV) { /* cherenkov.py:33 cone: a Frank-Tamm photon of the segment */
    float u_lam = o_uniform(rk, 0), u_pos = o_uniform(rk, 1), u_phi = o_uniform(rk, 2);
    const float* ax = f + 3;
    const float len = f[6], beta = f[8], charge = f[9], samples = f[10];
    const float zq = 1.0f / src->lam0 - 1.0f / src->lam1;
    const float lam = 1.0f / (1.0f / src->lam0 - u_lam * zq);
    const float n = o_tab(D, pool, src->rindex_tab, O_HC / lam, 0);
    const float bn2 = beta * beta * n * n;
    const int emits = 1.0f - 1.0f / bn2 > 0.0f;
    const float s = emits ? 1.0f - 1.0f / bn2 : 0.0f;
    r->w0 = O_TWO_PI_ALPHA * (charge * charge) * len * s * zq / samples * 1e9f;
    const float cos_c = emits ? 1.0f / (beta * n) : 1.0f;
    const float sq = 1.0f - cos_c * cos_c;
    const float sin_c = sq > 0.0f ? sqrtf(sq) : 0.0f;
    float sp, cp;
    o_sincos2pi(u_phi, &sp, &cp);
    float l[3] = {sin_c * cp, sin_c * sp, cos_c};
    o_to_world(l, ax, r->d);
    const float xs = u_pos * len;
    for (int a = 0; a < 3; ++a) r->x[a] = f[a] + xs * ax[a];
    r->t = f[7] + xs / (beta * O_C_VACUUM);
    r->lam = lam;
    float ad = o_dot(ax, r->d);
    for (int a = 0; a < 3; ++a) r->er[a] = ad * r->d[a] - ax[a];
    o_unit(r->er);
    return;
  }
  float g[3] = {o_gaussian(o_uniform(rk, 0)), o_gaussian(o_uniform(rk, 1)), o_gaussian(o_uniform(rk, 2))};
  o_unit(g);
  for (int a = 0; a < 3; ++a) { r->x[a] = f[a]; r->d[a] = g[a]; }
  float u3 = o_uniform(rk, 3);
  r->lam = src->lam1 > src->lam0 ? src->lam0 + (src->lam1 - src->lam0) * u3 : src->lam0;
  r->t = f[3];
  if (src->kind == LUMEN_SRC_SCINT) {
    float u4 = o_uniform(rk, 4), u5 = o_uniform(rk, 5);
    float tau = u4 < src->frac1 ? src->tau1 : src->tau2;
    r->t = f[3] + -o_log(u5) * tau;
  }
}

/* -------------------------------------------------------------------------------------------- the photon loop */
typedef struct OTally {
  int S_, E, nb, P;
  float bin0, bin_w;
  std::vector<double> arrival, arrival_t, arrival2, hist, jac, health;
  std::vector<long long> counts;
} OTally;

static inline int s_out_of(const OTally* T, int s) { return s < 0 || s >= T->S_; }

/* a photon's per-sensor sums, in the order its sensors first took light: the second moment adds the square of each at
   the photon's end (run.py:483 _moment_adds: the photon's own cell total squared, exact over any number of sensors) */
typedef std::vector<std::pair<int, double>> OPhotonSums;

/* a thread's readout groups: the cells, and the photons' records when the caller asks for them (photon id, record,
   the photon's row weight and event) */
typedef struct OGroupCtx {
  const LumenTallies* out;
  OGroupT T;
  int keep;
  std::vector<int64_t> photon;
  std::vector<ORec> recs;
  std::vector<std::pair<float, int>> w0_ev;
} OGroupCtx;

/* one photon's loop (run.py:307 item): begin, steps until it ends or reaches the vertex guard */
template <class NF>
static void o_photon(const ORun* R, const ORow* row, OKey key, int64_t gid, OTally* T, int32_t* rec_i,
                     float* rec_f, OGroupCtx* gc, float* truth) {
  const OScene* S = &R->S;
  OPhotonT<NF> ph;
  memset(&ph, 0, sizeof(ph));
  for (int a = 0; a < 3; ++a) { ph.x[a] = row->x[a]; ph.d[a] = row->d[a]; ph.er[a] = row->er[a]; ph.ei[a] = row->ei[a]; }
  ph.t = row->t;
  ph.lam = row->lam;
  ph.w = 1.0f;
  ph.wr = 1.0f;
  ph.alive = 1;
  ph.vertex = 0;
  ph.vol = onav_locate(S, ph.x);
  ph.cls = o_cls(S, ph.vol);
  ph.srf = -1;
  ph.nz = 0;
  OKey pkey = o_fold_in(key, (uint32_t)gid);
  const double w0 = row->w0;
  const int e = row->event;
  if (R->analog) { /* run.py:319: one uniform of the photon's analog stream; open with probability k (state.py:58) */
    const float u = o_uniform(o_fold_in(pkey, 0x7A4A1061u), 0);
    ph.ak = row->w0;
    ph.ax = u < ph.ak ? u / (ph.ak > 0.0f ? ph.ak : 1.0f) : INFINITY;
    ph.asensor = -1;
    ph.ascale = 1.0f;
    ph.avol = -1;
  }
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  double pushed = 0.0;
  OPhotonSums ps;
  int n_dep = 0, first_sensor = -1;
  double sum_q = 0.0, sum_qt = 0.0;
  long long steps = 0;
  std::vector<ORec> recs;
  while (ph.alive && ph.vertex < R->max_vertices) {
    ODep dep;
    o_step(R, &ph, pkey, &dep);
    steps++;
    for (int k = 0; k < 8; ++k) acc[k] += (double)dep.fates[k];
    pushed += (double)dep.pushed * w0;
    if (dep.sensor >= 0 && (e < 0 || e >= T->E || s_out_of(T, dep.sensor))) { /* an event or sensor out of range:
                                                                                  counted, not tallied (the engine's rule) */
      n_dep++;
      T->counts[LUMEN_C_DEPOSITS] += 1;
      if (gc) recs.push_back(dep.rec);
      if (first_sensor < 0) first_sensor = dep.sensor;
      sum_q += (double)dep.q;
      sum_qt += (double)dep.q * (double)dep.time;
    } else if (dep.sensor >= 0) {
      int s = dep.sensor;
      double v = (double)dep.q * w0;
      size_t ix = (size_t)e * T->S_ + s;
      T->arrival[ix] += v;
      T->arrival_t[ix] += v * (double)dep.time;
      if (T->nb > 0) {
        float b = floorf((dep.time - T->bin0) / T->bin_w);
        if (b >= 0.0f && b < (float)T->nb) T->hist[ix * T->nb + (size_t)b] += v;
      }
      for (int p = 0; p < R->P; ++p) T->jac[ix * R->P + p] += (double)dep.dq[p] * w0;
      if (v != 0.0) { /* a deposit of 0 (a photon of weight 0) adds nothing to any sum */
        size_t j = 0;
        while (j < ps.size() && ps[j].first != s) ++j;
        if (j == ps.size()) ps.push_back({s, 0.0});
        ps[j].second += v;
      }
      n_dep++;
      if (gc) recs.push_back(dep.rec);
      if (first_sensor < 0) first_sensor = s;
      sum_q += (double)dep.q;
      sum_qt += (double)dep.q * (double)dep.time;
      T->counts[LUMEN_C_DEPOSITS] += 1;
    }
  }
  if (ps.size() > 4) T->counts[LUMEN_C_MULTI] += (long long)ps.size() - 4; /* the sums past the photon's first four */
  for (const auto& sv : ps) T->arrival2[(size_t)e * T->S_ + sv.first] += sv.second * sv.second;
  if (gc && !recs.empty()) {
    if (e >= 0 && e < T->E) o_bin_photon(R->S.D, gc->out, recs, w0, e, T->S_, &gc->T);
    if (gc->keep)
      for (const ORec& rc : recs) {
        gc->photon.push_back(gid);
        gc->recs.push_back(rc);
        gc->w0_ev.push_back({(float)w0, e});
      }
  }
  for (int k = 0; k < 8; ++k) T->health[k] += acc[k] * w0;
  double trunc = ph.alive ? (double)ph.w * w0 : 0.0;
  T->health[LUMEN_H_TRUNCATED] += trunc;
  T->health[LUMEN_H_PUSHED] += pushed;
  T->health[LUMEN_H_START] += w0;
  T->counts[LUMEN_C_PHOTONS] += 1;
  T->counts[LUMEN_C_STEPS] += steps;
  if (ph.alive) T->counts[LUMEN_C_TRUNCATED] += 1;
  if (truth) { /* the photon's analog record (run.py:350) */
    memcpy(truth + LUMEN_TR_SENSOR, &ph.asensor, 4);
    truth[LUMEN_TR_TIME] = ph.atime;
    truth[LUMEN_TR_LAM] = ph.alam;
    truth[LUMEN_TR_SCALE] = ph.ascale;
    for (int a = 0; a < 3; ++a) truth[LUMEN_TR_POS + a] = ph.apos[a];
    memcpy(truth + LUMEN_TR_VOL, &ph.avol, 4);
  }
  if (rec_i) {
    rec_i[0] = ph.vertex;
    rec_i[1] = n_dep;
    rec_i[2] = ph.alive ? 0 : 1;
    rec_i[3] = first_sensor;
    rec_i[4] = ph.vol;
    rec_f[0] = (float)sum_q;
    rec_f[1] = ph.w;
    rec_f[2] = ph.t;
    rec_f[3] = (float)sum_qt;
  }
}

static int o_scene(const LumenSceneDesc* D, OScene* S) {
  S->D = D;
  S->n = D->n_vol;
  S->LM = 1;
  S->FM = 1;
  for (int k = 0; k < D->n_kind; ++k) {
    const int32_t* ki = D->kind_i + (size_t)k * LUMEN_KIND_I;
    if (ki[1] > S->LM) S->LM = ki[1];
    if (ki[1] > LUMEN_MAX_LEAVES) return LUMEN_ERR_SCENE;
    for (int l = 0; l < ki[1]; ++l) {
      int np = D->leaf_i[(size_t)(ki[0] + l) * LUMEN_LEAF_I + 2];
      if (np + 1 > S->FM) S->FM = np + 1;
    }
  }
  S->n_chunk = D->n_mesh > 0 ? D->n_chunk : 0;
  S->ch0 = D->n_mesh > 0 ? D->n_vol + 1 + D->n_mesh : 0x7fffffff;
  S->SU = D->n_vol + 1 + (D->n_mesh > 0 ? D->n_mesh + D->n_chunk : 0);
  S->sm = D->n_mesh > 0 ? S->SU + D->n_vol * S->LM * S->FM * 4 : 0x7fffffff;
  S->nav64 = D->precision == LUMEN_PREC_FLOAT64;
  if (S->nav64 && (!D->vol_f64 || !D->leaf_f64 || (D->n_plane > 0 && !D->plane_f64))) return LUMEN_ERR_ARG;
  return LUMEN_OK;
}

static void o_run_init(ORun* R, const LumenSceneDesc* D, const float* live, const float* ref,
                       const LumenControls* c) {
  o_scene(D, &R->S);
  R->live = live ? live : D->pool;
  R->ref = ref ? ref : R->live;
  R->shared = R->ref == R->live;
  R->reach = D->reach;
  R->max_distance = c->max_distance > 0.0f ? c->max_distance : D->reach;
  R->roulette = c->roulette;
  R->max_vertices = c->max_vertices;
  R->P = c->n_grad;
  R->jump = (c->flags & LUMEN_F_JUMP) && D->n_jump > 0;
  R->analog = (c->flags & LUMEN_F_TRUTH) != 0;
  for (int p = 0; p < R->P; ++p) R->gt[p] = c->grad_tab[p];
}

/* host rows in the layout of LumenRows (every pointer a host array) */
static void o_row_of(const ORun* R, const LumenRows* rows, const LumenSource* src, OKey key, int64_t first_id,
                     int64_t i, ORow* r) {
  if (rows) {
    r->x[0] = rows->x[i]; r->x[1] = rows->y[i]; r->x[2] = rows->z[i];
    r->d[0] = rows->dx[i]; r->d[1] = rows->dy[i]; r->d[2] = rows->dz[i];
    r->t = rows->t[i]; r->lam = rows->lam[i]; r->w0 = rows->w[i];
    for (int a = 0; a < 3; ++a) {
      r->er[a] = rows->pol ? rows->pol[6 * i + a] : 0.0f;
      r->ei[a] = rows->pol ? rows->pol[6 * i + 3 + a] : 0.0f;
    }
    r->event = rows->event ? rows->event[i] : 0;
  } else {
    o_source_row(R->S.D, R->live, R->ref, src, key, first_id + i, r);
  }
}

extern "C" {

int32_t lumen_oracle_threefry(uint32_t k0, uint32_t k1, uint32_t x0, uint32_t x1, uint32_t* out) {
  o_threefry(k0, k1, x0, x1, out, out + 1);
  return 0;
}

/* uniforms(vertex_key(photon_key(key, id), vertex), n) for ids[i] (rng.py:81 uniforms) */
int32_t lumen_oracle_uniforms(uint32_t k0, uint32_t k1, const int64_t* ids, int64_t n_ids, int32_t vertex,
                              int32_t n, float* out) {
  OKey key = {k0, k1};
  for (int64_t i = 0; i < n_ids; ++i) {
    OKey vk = o_fold_in(o_fold_in(key, (uint32_t)ids[i]), (uint32_t)vertex);
    for (int j = 0; j < n; ++j) out[i * n + j] = o_uniform(vk, (uint32_t)j);
  }
  return 0;
}

/* elementwise math for the golden checks: fn 0 exp, 1 log, 2 sin 2 pi x, 3 cos 2 pi x, 4 acos, 5 cbrt, 6 erfinv,
   7 sin, 8 cos, 9 dipole_cos, 10 gaussian */
/* 1: run lumen 0.2.0's rule for the reference weight after a covered draw at a surface whose reference probabilities
   are all 0 (the weight kept; 0.2.1 multiplies it by e / (1 - e) / n, src/lumen/transport/estimator.py:83); 0: the
   current rule. Returns the previous setting. Not thread-safe: set it before a trace. */
int32_t lumen_oracle_set_rule_020(int32_t on) {
  int32_t was = g_rule_020;
  g_rule_020 = on != 0;
  return was;
}

int32_t lumen_oracle_math(int32_t fn, const float* x, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) {
    float s, c;
    switch (fn) {
      case 0: out[i] = o_exp(x[i]); break;
      case 1: out[i] = o_log(x[i]); break;
      case 2: o_sincos2pi(x[i], &s, &c); out[i] = s; break;
      case 3: o_sincos2pi(x[i], &s, &c); out[i] = c; break;
      case 4: out[i] = o_acos(x[i]); break;
      case 5: out[i] = o_cbrt(x[i]); break;
      case 6: out[i] = o_erfinv(x[i]); break;
      case 7: o_sincos(x[i], &s, &c); out[i] = s; break;
      case 8: o_sincos(x[i], &s, &c); out[i] = c; break;
      case 9: out[i] = o_dipole_cos(x[i]); break;
      case 10: out[i] = o_gaussian(x[i]); break;
      default: return LUMEN_ERR_ARG;
    }
  }
  return 0;
}

/* Fresnel amplitudes (fresnel.py:25) for n rows of (cos_i, n1, n2re, n2im): out 8 floats per row */
int32_t lumen_oracle_fresnel(const float* in, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) {
    Oc a[4];
    o_amplitudes(in[4 * i], in[4 * i + 1], oc(in[4 * i + 2], in[4 * i + 3]), a);
    for (int j = 0; j < 4; ++j) { out[8 * i + 2 * j] = a[j].re; out[8 * i + 2 * j + 1] = a[j].im; }
  }
  return 0;
}

/* Geant4's GROUPVEL group index of an index table (energies e, values n, k knots) at wavelengths lam (laws.py:170) */
int32_t lumen_oracle_group_index(const float* e, const float* n, int32_t k, const float* lam, int64_t m, float* out) {
  if (k < 1 || k > LUMEN_MAX_KNOTS) return LUMEN_ERR_ARG;
  std::vector<float> pool(2 * k);
  for (int j = 0; j < k; ++j) { pool[j] = e[j]; pool[k + j] = n[j]; }
  int32_t tab[2] = {0, k};
  LumenSceneDesc D;
  memset(&D, 0, sizeof(D));
  D.tab = tab;
  for (int64_t i = 0; i < m; ++i) out[i] = o_group_index(&D, pool.data(), 0, O_HC / lam[i]);
  return 0;
}

/* n unified facet paths off a flat surface (normal +z) for the incoming direction wi, each from three uniforms of
   its own key (the lobe's rand); out: the last directions (n * 3), capped: paths that hit a loop bound. With the
   tables U (else null), dens (n * 3) gets each path's log density at sig_live, at sigma, and the former's derivative
   in sig_live. With one set, each draw is a single facet reflection (its direction may point into the surface). */
int32_t lumen_oracle_facet_path(float sigma, const float* wi, uint32_t k0, uint32_t k1, int64_t n, float* out,
                                int64_t* capped, const float* U, float sig_live, float* dens, int32_t one) {
  const float up[3] = {0.0f, 0.0f, 1.0f};
  OKey key = {k0, k1};
  int64_t nc = 0;
#pragma omp parallel for reduction(+ : nc)
  for (int64_t i = 0; i < n; ++i) {
    OKey k = o_fold_in(key, (uint32_t)i);
    float r[3] = {o_uniform(k, 0), o_uniform(k, 1), o_uniform(k, 2)};
    float er[3] = {0.0f, 1.0f, 0.0f}, ei[3] = {0.0f, 0.0f, 0.0f};
    int c = 0;
    float lp = 0.0f, lr = 0.0f, dls = 0.0f;
    if (one) { /* the path's first facet alone */
      float mwi[3] = {-wi[0], -wi[1], -wi[2]}, V[3], m[3];
      o_to_local(mwi, up, V);
      o_unified_facet(sigma, V, o_fold_in(o_seed_key(r[0], r[1], r[2]), 0), m, &c);
      float vm = o_dot(V, m);
      float L[3] = {2.0f * vm * m[0] - V[0], 2.0f * vm * m[1] - V[1], 2.0f * vm * m[2] - V[2]};
      o_to_world(L, up, out + 3 * i);
      if (U) {
        lp = o_unified_logpdf(U, sig_live, wi, up, out + 3 * i, &dls);
        lr = o_unified_logpdf(U, sigma, wi, up, out + 3 * i, 0);
      }
    } else {
      o_facet_path(sigma, wi, up, r, out + 3 * i, er, ei, &c, U, sig_live, 1, &lp, &lr, &dls);
    }
    if (U) { dens[3 * i] = lp; dens[3 * i + 1] = lr; dens[3 * i + 2] = dls; }
    nc += c;
  }
  *capped = nc;
  return 0;
}

/* n Mie draws (G4OpMieHG) about wi at constants (gf, gb, ratio), each from three uniforms of its own key: out the
   directions (n * 3), lp their log densities (n) */
int32_t lumen_oracle_mie(float gf, float gb, float ratio, const float* wi, uint32_t k0, uint32_t k1, int64_t n,
                         float* out, float* lp) {
  OKey key = {k0, k1};
#pragma omp parallel for
  for (int64_t i = 0; i < n; ++i) {
    OKey k = o_fold_in(key, (uint32_t)i);
    float r[3] = {o_uniform(k, 0), o_uniform(k, 1), o_uniform(k, 2)};
    o_mie_sample(gf, gb, ratio, wi, r, out + 3 * i);
    lp[i] = o_mie_logpdf(gf, gb, ratio, wi, out + 3 * i, 0);
  }
  return 0;
}
/* The Mie log density at n given directions (n * 3) about wi, with its derivatives in (gf, gb, ratio): out n * 4 */
int32_t lumen_oracle_mie_logpdf(float gf, float gb, float ratio, const float* wi, const float* wo, int64_t n,
                                float* out) {
  for (int64_t i = 0; i < n; ++i) out[4 * i] = o_mie_logpdf(gf, gb, ratio, wi, wo + 3 * i, out + 4 * i + 1);
  return 0;
}
/* n G4OpWLS emissions of photons absorbed at lam_in from the spectra (live e, s; reference er, sr: k knots each),
   each from two uniforms of its own key: out n * 4 (wavelength, delay, weight, reference weight) */
int32_t lumen_oracle_wls(const float* e, const float* sl, const float* sr, int32_t k, float yield_l, float yield_r,
                         float tau, int32_t exponential, float lam_in, uint32_t k0, uint32_t k1, int64_t n,
                         float* out) {
  OKey key = {k0, k1};
#pragma omp parallel for
  for (int64_t i = 0; i < n; ++i) {
    OKey kk = o_fold_in(key, (uint32_t)i);
    OEmit em = o_wls_emit(e, sl, k, e, sr, k, yield_l, yield_r, tau, exponential, lam_in, o_uniform(kk, 0),
                          o_uniform(kk, 1));
    out[4 * i] = em.lam; out[4 * i + 1] = em.delay; out[4 * i + 2] = em.w; out[4 * i + 3] = em.w_r;
  }
  return 0;
}

/* n GLISUR facet paths off a flat surface (normal +z): kind 1 metal, 2 dielectric (indices n1 incident, n2 far), at
   r = 1 - polish, each from three uniforms of its own key, with the photon's Jones vector er (n * 3, real linear
   states); e the cover's share (0: Geant4's draw). out n * 6: the last direction, the far flag, the path weight,
   d/dr of the log weight */
int32_t lumen_oracle_glisur(int32_t kind, float polish, float n1, float n2, const float* wi, const float* er_in,
                            float e, uint32_t k0, uint32_t k1, int64_t n, float* out, int64_t* capped) {
  const float up[3] = {0.0f, 0.0f, 1.0f};
  OKey key = {k0, k1};
  int64_t nc = 0;
  float r = 1.0f - polish;
#pragma omp parallel for reduction(+ : nc)
  for (int64_t i = 0; i < n; ++i) {
    OKey k = o_fold_in(key, (uint32_t)i);
    float rr[3] = {o_uniform(k, 0), o_uniform(k, 1), o_uniform(k, 2)};
    float er[3] = {er_in[3 * i], er_in[3 * i + 1], er_in[3 * i + 2]}, ei[3] = {0.0f, 0.0f, 0.0f};
    int c = 0, far = 0;
    float on = 0.0f, dl = 0.0f, w;
    if (kind == 1) w = o_glisur_metal_path(r, r, wi, up, rr, e, out + 6 * i, er, ei, &c, &on, &dl);
    else w = o_glisur_dielectric_path(r, r, n1, n2, wi, up, rr, e, out + 6 * i, er, ei, &far, &c, &on, &dl);
    out[6 * i + 3] = (float)far;
    out[6 * i + 4] = w;
    out[6 * i + 5] = dl;
    nc += c;
  }
  *capped = nc;
  return 0;
}

/* The unified tables and density on n inputs (in, out per fn): 0 log zeta at y = log sigma (y -> lz, dlz/dy);
   1 F at (x, y) (-> F, dF/dx, dF/dy); 2 one facet reflection's log density at (sigma, w0 (3), normal (3), w1 (3))
   (-> log p1, d log p1 / d sigma) */
int32_t lumen_oracle_unified(const float* U, int32_t fn, const float* in, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) {
    if (fn == 0) {
      out[2 * i] = o_table_lz(U, in[i], out + 2 * i + 1);
    } else if (fn == 1) {
      out[3 * i] = o_table_front(U, in[2 * i], in[2 * i + 1], out + 3 * i + 1, out + 3 * i + 2);
    } else if (fn == 2) {
      const float* a = in + 10 * i;
      out[2 * i] = o_unified_logpdf(U, a[0], a + 1, a + 4, a + 7, out + 2 * i + 1);
    } else {
      return 1;
    }
  }
  return 0;
}

/* basis(n) for n unit vectors: out t1, t2 (frames.py:14) */
int32_t lumen_oracle_basis(const float* nv, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i) o_basis(nv + 3 * i, out + 6 * i, out + 6 * i + 3);
  return 0;
}

int32_t lumen_oracle_locate(const LumenSceneDesc* D, const float* pts, int64_t n, int32_t* vol) {
  OScene S;
  int st = o_scene(D, &S);
  if (st) return st;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) vol[i] = onav32::o_locate(&S, pts + 3 * i);
  return 0;
}

/* locate and query in float64 (a float64 scene: LUMEN_PREC_FLOAT64), the layout of lumen_b200_locate64 / query64 */
int32_t lumen_oracle_locate64(const LumenSceneDesc* D, const double* pts, int64_t n, int32_t* vol) {
  OScene S;
  int st = o_scene(D, &S);
  if (st) return st;
  if (!S.nav64) return LUMEN_ERR_ARG;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) vol[i] = onav64::o_locate(&S, pts + 3 * i);
  return 0;
}

int32_t lumen_oracle_query64(const LumenSceneDesc* D, const double* ray, const int32_t* vol, const int32_t* srf,
                             double t_max, int64_t n, int32_t* out_i, double* out_f) {
  OScene S;
  int st = o_scene(D, &S);
  if (st) return st;
  if (!S.nav64) return LUMEN_ERR_ARG;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    const double* o = ray + 6 * i;
    const double* d = ray + 6 * i + 3;
    int v = vol[i] >= 0 ? vol[i] : onav64::o_locate(&S, o);
    int last = vol[i] >= 0 ? srf[i] : -1;
    OQueryT<double> q = onav64::o_query(&S, o, d, v, t_max, last, 0, 1e30);
    int32_t* oi = out_i + 8 * i;
    oi[0] = q.hit; oi[1] = q.vol_before; oi[2] = q.vol_after; oi[3] = q.cls_before; oi[4] = q.cls_after;
    oi[5] = q.srf; oi[6] = q.zero;
    oi[7] = q.hit ? D->vol_i[(size_t)q.vol_after * LUMEN_VOL_I + LUMEN_VI_SENSOR] : -1;
    double* of = out_f + 4 * i;
    of[0] = q.t; of[1] = q.normal[0]; of[2] = q.normal[1]; of[3] = q.normal[2];
  }
  return 0;
}

/* the navigator query on a fixed ray set, the layout of lumen_b200_query (host arrays) */
int32_t lumen_oracle_query(const LumenSceneDesc* D, const float* ray, const int32_t* vol, const int32_t* srf,
                           float t_max, int64_t n, int32_t* out_i, float* out_f) {
  OScene S;
  int st = o_scene(D, &S);
  if (st) return st;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < n; ++i) {
    const float* o = ray + 6 * i;
    const float* d = ray + 6 * i + 3;
    int v = vol[i] >= 0 ? vol[i] : onav32::o_locate(&S, o);
    int last = vol[i] >= 0 ? srf[i] : -1;
    OQuery q = onav32::o_query(&S, o, d, v, t_max, last, 0, O_HUGE);
    int32_t* oi = out_i + 8 * i;
    oi[0] = q.hit; oi[1] = q.vol_before; oi[2] = q.vol_after; oi[3] = q.cls_before; oi[4] = q.cls_after;
    oi[5] = q.srf; oi[6] = q.zero;
    oi[7] = q.hit ? D->vol_i[(size_t)q.vol_after * LUMEN_VOL_I + LUMEN_VI_SENSOR] : -1;
    float* of = out_f + 4 * i;
    of[0] = q.t; of[1] = q.normal[0]; of[2] = q.normal[1]; of[3] = q.normal[2];
  }
  return 0;
}

/* Trace photons first_id .. first_id + n - 1 (host arrays throughout; rows or src, one of them). Tallies are ADDED
   to the host arrays of `out` (LumenTallies layout); rec_i / rec_f (optional) get the per-photon record of
   lumen_b200_trace_photons. threads <= 0: OpenMP's default. */
int32_t lumen_oracle_trace(const LumenSceneDesc* D, const float* pool_live, const float* pool_ref,
                           const LumenRows* rows, const LumenSource* src, uint32_t key0, uint32_t key1,
                           int64_t first_id, int64_t n, const LumenControls* c, LumenTallies* out, int32_t* rec_i,
                           float* rec_f, int32_t threads) {
  if (!D || !c || !out || (!rows && !src) || n < 0) return LUMEN_ERR_ARG;
  if (c->n_grad < 0 || c->n_grad > LUMEN_MAX_GRAD) return LUMEN_ERR_NOT_SUPPORTED;
  ORun R;
  o_run_init(&R, D, pool_live, pool_ref, c);
  if (o_scene(D, &R.S)) return LUMEN_ERR_SCENE;
  OKey key = {key0, key1};
  const int Sn = D->n_sensor > 0 ? D->n_sensor : 1, E = out->n_events > 0 ? out->n_events : 1;
  int nth = threads > 0 ? threads : omp_get_max_threads();
  std::vector<OTally> parts(nth);
  const int groups = out->n_groups > 0;
  if (groups && (out->n_groups > LUMEN_MAX_GROUPS || !out->groups)) return LUMEN_ERR_ARG;
  std::vector<OGroupCtx> gparts(groups ? nth : 0);
  for (auto& G : gparts) {
    G.out = out;
    G.keep = out->records != 0;
    o_groups_init(&G.T, out, E, Sn);
  }
  for (auto& T : parts) {
    T.S_ = Sn; T.E = E; T.nb = out->hist ? out->n_bins : 0; T.P = c->n_grad;
    T.bin0 = out->bin0; T.bin_w = out->bin_w;
    T.arrival.assign((size_t)E * Sn, 0.0); T.arrival_t.assign((size_t)E * Sn, 0.0);
    T.arrival2.assign((size_t)E * Sn, 0.0);
    T.hist.assign((size_t)E * Sn * T.nb, 0.0);
    T.jac.assign((size_t)E * Sn * (c->n_grad > 0 ? c->n_grad : 0), 0.0);
    T.health.assign(LUMEN_N_HEALTH, 0.0);
    T.counts.assign(LUMEN_N_COUNT, 0);
  }
#pragma omp parallel for schedule(dynamic, 16) num_threads(nth)
  for (int64_t i = 0; i < n; ++i) {
    ORow r;
    o_row_of(&R, rows, src, key, first_id, i, &r);
    OTally* Tp = &parts[omp_get_thread_num()];
    OGroupCtx* gp = groups ? &gparts[omp_get_thread_num()] : 0;
    float* tr = (R.analog && out->truth) ? out->truth + (size_t)LUMEN_TRUTH_WORDS * i : 0;
    if (R.S.nav64)
      o_photon<double>(&R, &r, key, first_id + i, Tp, rec_i ? rec_i + 5 * i : 0, rec_f ? rec_f + 4 * i : 0, gp, tr);
    else
      o_photon<float>(&R, &r, key, first_id + i, Tp, rec_i ? rec_i + 5 * i : 0, rec_f ? rec_f + 4 * i : 0, gp, tr);
  }
  if (groups) { /* the threads' cells, and the records in photon order (the engine's layout, LUMEN_REC_WORDS each) */
    for (auto& G : gparts) {
      for (int g = 0; g < out->n_groups; ++g) {
        const LumenGroup& LG = out->groups[g];
        for (size_t k = 0; k < G.T.charge[g].size(); ++k) { LG.charge[k] += G.T.charge[g][k]; LG.charge2[k] += G.T.charge2[g][k]; }
        for (size_t k = 0; k < G.T.time[g].size(); ++k) LG.time[k] += G.T.time[g][k];
        for (size_t k = 0; k < G.T.over_q[g].size(); ++k) { LG.over_q[k] += G.T.over_q[g][k]; LG.over_qt[k] += G.T.over_qt[g][k]; }
      }
      if (out->pe2) for (size_t k = 0; k < G.T.pe2.size(); ++k) out->pe2[k] += G.T.pe2[k];
    }
    std::vector<std::pair<int64_t, std::pair<int, size_t>>> order; /* (photon, (thread, index)) */
    for (int t = 0; t < (int)gparts.size(); ++t)
      for (size_t k = 0; k < gparts[t].recs.size(); ++k) order.push_back({gparts[t].photon[k], {t, k}});
    std::stable_sort(order.begin(), order.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    if (out->counts) out->counts[LUMEN_C_RECORDS] += (unsigned long long)order.size();
    if (out->records) {
      uint32_t* w = (uint32_t*)out->records;
      int64_t n_out = (int64_t)order.size() < out->rec_capacity ? (int64_t)order.size() : out->rec_capacity;
      for (int64_t k = 0; k < n_out; ++k) {
        const OGroupCtx& G = gparts[order[k].second.first];
        const size_t j = order[k].second.second;
        const ORec& rc = G.recs[j];
        uint32_t* o = w + k * LUMEN_REC_WORDS;
        float f[LUMEN_REC_WORDS];
        memset(f, 0, sizeof(f));
        memcpy(o, f, sizeof(f));
        const int first = k == 0 || order[k - 1].first != order[k].first;
        const int last = k + 1 == (int64_t)order.size() || order[k + 1].first != order[k].first;
        int32_t iv[4] = {first ? -1 : (int32_t)(k - 1), rc.sensor, rc.gen, rc.vol};
        memcpy(o + 0, &iv[0], 4); memcpy(o + 1, &iv[1], 4); memcpy(o + 6, &iv[2], 4); memcpy(o + 7, &iv[3], 4);
        memcpy(o + 2, &rc.q, 4); memcpy(o + 3, &rc.time, 4); memcpy(o + 4, &rc.lam, 4); memcpy(o + 5, &rc.inv_an, 4);
        memcpy(o + 8, rc.x, 12); memcpy(o + 11, rc.d, 12); memcpy(o + 14, rc.n, 12);
        if (last) {
          o[17] = 1u;
          memcpy(o + 18, &G.w0_ev[j].first, 4);
          memcpy(o + 19, &G.w0_ev[j].second, 4);
        }
      }
    }
  }
  for (auto& T : parts) {
    for (size_t k = 0; k < T.arrival.size(); ++k) {
      out->arrival[k] += T.arrival[k];
      out->arrival_t[k] += T.arrival_t[k];
      out->arrival2[k] += T.arrival2[k];
    }
    if (out->hist) for (size_t k = 0; k < T.hist.size(); ++k) out->hist[k] += T.hist[k];
    if (out->jac) for (size_t k = 0; k < T.jac.size(); ++k) out->jac[k] += T.jac[k];
    if (out->health) for (int k = 0; k < LUMEN_N_HEALTH; ++k) out->health[k] += T.health[k];
    if (out->counts) for (int k = 0; k < LUMEN_N_COUNT; ++k) out->counts[k] += (unsigned long long)T.counts[k];
  }
  return 0;
}

/* emission rows of a procedural source (host): x, d, t, lam, w0, er, ei, event per photon; D, pool (the live values)
   and ref (the reference's; null: the live) are read by the Cherenkov and the material scintillation sources */
int32_t lumen_oracle_source_rows(const LumenSceneDesc* D, const float* pool, const float* ref, const LumenSource* src,
                                 uint32_t key0, uint32_t key1, int64_t first_id, int64_t n, float* out_f,
                                 int32_t* out_event) {
  OKey key = {key0, key1};
  if ((src->kind == LUMEN_SRC_CHERENKOV || src->kind == LUMEN_SRC_SCINT_MATERIAL) && !D) return LUMEN_ERR_ARG;
  const float* pl = pool ? pool : (D ? D->pool : 0);
  const float* rf = ref ? ref : pl;
  for (int64_t i = 0; i < n; ++i) {
    ORow r;
    o_source_row(D, pl, rf, src, key, first_id + i, &r);
    float* f = out_f + 15 * i;
    for (int a = 0; a < 3; ++a) { f[a] = r.x[a]; f[3 + a] = r.d[a]; f[9 + a] = r.er[a]; f[12 + a] = r.ei[a]; }
    f[6] = r.t; f[7] = r.lam; f[8] = r.w0;
    out_event[i] = r.event;
  }
  return 0;
}

}  /* extern "C" */
