// One photon step on the device (src/lumen/transport/step.py:516 `step`, with `_recover` :245, `_step_context` :318,
// `_surface_event` :362, `_bulk` :397, `_after` :464, `_advance` :495), with forward-mode tangents of the live
// weight in up to G gradient parameters (the reference's reweighting estimator differentiated along the fixed path).
// Arithmetic operation for operation the CPU checker's; uniforms are drawn lazily (each is a pure function of the
// vertex key and its index, so skipping an unused one changes nothing).
#pragma once
#include "dmedia.cuh"

namespace lb {

#define D_POL_STREAM 0x9017u
#define D_SOURCE_STREAM 0xFFFFFFFFu
#define D_NORMAL_LO -0.99999994039535522461f
#define D_SQRT2 1.41421356237309504880f

struct Run {
  DScene S;
  const float* __restrict__ live;
  const float* __restrict__ ref;
  int shared;
  float max_distance, roulette, reach;
  int max_vertices;
  int P;
  int gt[LUMEN_MAX_GRAD];
  int reach_on;  // LUMEN_F_REACH: bulk steps' queries bounded by the sensor reach
  int jump_on;   // LUMEN_F_JUMP: the diffusion jump at bulk Rayleigh events
  uint32_t* rec;                // the deposit records of the readout groups (LUMEN_REC_WORDS each), or null
  long long rec_cap;            // records the scratch holds
  unsigned long long* rec_n;    // the call's record counter
};

// ------------------------------------------------------------------------------------------ the diffusion jump
#define D_JUMP_STREAM 0x7A11u  // the vertex key's fold for the walk's own uniforms (rng.py:25)
struct Jmp {
  int ok, n;
  float y[3], d[3], er[3], L;
};
// the walk at a bulk Rayleigh event inside the proven clear ball at xs (fastpath.py:174 diffuse): free paths at the
// reference rate, the polarised Rayleigh draw and projection, until a flight leaves the ball (the photon put at the
// crossing) or the budget ceil((c mu_r)^2) of scatterings (at most LUMEN_JUMP_STEPS) is spent
L_DEV void d_diffuse(const DScene& S, int mi, const float* xs, const float* d0, const float* er0, const float* ei0,
                      float mu_r, int alive, Key vkey, Jmp& J) {
  J.ok = 0; J.n = 0; J.L = 0.0f;
  for (int a = 0; a < 3; ++a) { J.y[a] = 0.0f; J.d[a] = d0[a]; J.er[a] = er0[a]; }
  int g = __ldg(S.med_jump + mi);
  if (g < 0) return;
  const float* jf = S.jump_f + (size_t)g * LUMEN_JUMP_F;
  const int32_t* ji = S.jump_i + (size_t)g * LUMEN_JUMP_I;
  float h = __ldg(jf + 3);
  int inside = 1, idx[3];
  float node[3];
  for (int a = 0; a < 3; ++a) {
    float fi = (xs[a] - __ldg(jf + a)) / h;
    int na = __ldg(ji + 1 + a);
    inside = inside && fi > -0.5f && fi < (float)na - 0.5f;
    int i = (int)floorf(fi + 0.5f);
    i = i < 0 ? 0 : (i > na - 1 ? na - 1 : i);
    idx[a] = i;
    node[a] = __ldg(jf + a) + h * (float)i;
  }
  float dx[3] = {xs[0] - node[0], xs[1] - node[1], xs[2] - node[2]};
  float c = __ldg(S.clear + __ldg(ji + 4) + ((int64_t)idx[0] * __ldg(ji + 2) + idx[1]) * __ldg(ji + 3) + idx[2]) -
            sqrtf(d_dot(dx, dx));
  int lin = ei0[0] == 0.0f && ei0[1] == 0.0f && ei0[2] == 0.0f;
  if (!(inside && c > 0.0f && lin && alive && mu_r > 0.0f)) return;
  J.ok = 1;
  float cm = c * mu_r;
  int budget = (int)ceilf(d_min(cm * cm, (float)LUMEN_JUMP_STEPS));
  Key jkey = fold_in(vkey, D_JUMP_STREAM);
  const float zero[3] = {0.0f, 0.0f, 0.0f};
  int out = 0;
  for (int j = 0; j < budget && !out; ++j) {
    Key kj = fold_in(jkey, (uint32_t)j);
    float u0 = uniform(kj, 0);
    float s = -l_log(u0) / mu_r;
    float by = d_dot(J.y, J.d);
    float t = -by + sqrtf(d_max(by * by - (d_dot(J.y, J.y) - c * c), 0.0f));
    out = s >= t;
    float k[3];
    d_rayleigh_sample(J.er, zero, uniform(kj, 1), uniform(kj, 2), uniform(kj, 3), k);
    float e2[3] = {J.er[0], J.er[1], J.er[2]}, z2[3] = {0.0f, 0.0f, 0.0f};
    d_project(e2, z2, k);
    float st = out ? t : s;
    for (int a = 0; a < 3; ++a) J.y[a] = J.y[a] + st * J.d[a];
    J.L = J.L + st;
    if (!out) {
      for (int a = 0; a < 3; ++a) { J.d[a] = k[a]; J.er[a] = e2[a]; }
      J.n += 1;
    }
  }
}

// NF: the position's precision, the navigator's (float32, or float64 with the float64 navigator: state.py:120 start's
// `position`); every other field float32
template <class NF>
struct PhotonT {
  NF x[3];
  float d[3], t, lam, w, wr;
  int alive, vertex;
  float er[3], ei[3];
  int vol, srf;
  float sn[3];
  int nz, cls;
  int gen;   // re-emissions so far (state.py Photon.gen: a WLS channel event adds one)
  int last;  // the photon's last deposit record (-1: none; the readout groups only)
};
using Photon = PhotonT<float>;

// ----------------------------------------------------------------------------------- the deposit records
// A_n: the share of a row absorbed and detected at normal incidence with eff 1, at the photon's wavelength and the
// crossing's incoming index, unpolarised (types.py:397 normal_absorptance, :391 _normal_incidence): the chain's
// absorbed rest of the cut reflectance (the R column; for a complex index the unpolarised Fresnel reflectance
// 0.5 (|r_s|^2 + |r_p|^2), fresnel.py:53) and T
L_DEV float d_normal_absorptance(const DScene& S, const float* __restrict__ pool, int row, float lam, float n1,
                                 const float* nrm) {
  const int32_t* ri = S.row_i + (size_t)row * LUMEN_ROW_I;
  float E = D_HC / lam;
  float Rc = d_tab(S, pool, __ldg(ri + LUMEN_RI_COL + LUMEN_COL_R), E);
  if (__ldg(ri + LUMEN_RI_MODEL) == 2) {
    float cos_i = d_clip01(-((-nrm[0] * nrm[0] + -nrm[1] * nrm[1]) + -nrm[2] * nrm[2]));
    Cf amps[4];
    d_amplitudes(cos_i, n1, cf(d_tab(S, pool, __ldg(ri + LUMEN_RI_COL + LUMEN_COL_NR), E),
                               d_tab(S, pool, __ldg(ri + LUMEN_RI_COL + LUMEN_COL_NK), E)), amps);
    Rc = d_clip01(0.5f * (c_abs2(amps[0]) + c_abs2(amps[1])));
  }
  float cut[2] = {Rc, d_tab(S, pool, __ldg(ri + LUMEN_RI_COL + LUMEN_COL_T), E)}, zc[2] = {0.0f, 0.0f}, rta[3], drta[3];
  d_chained<2>(cut, zc, rta, drta);
  return rta[2];
}

// appends one deposit record (step.py:546 the deposit's local fields, before the sensor frame: the crossing point,
// the direction and the normal in world coordinates, the volume entered, the re-emission count, 1 / A_n on a row
// flagged per_normal) and returns its index (-1 past the scratch's capacity); prev links the photon's records
L_DEV int d_record(const Run& R, int prev, int sensor, float q, float time, float lam, int gen, int row, float n1,
                    int vol, const float* x, const float* d, const float* nrm) {
  const DScene& S = R.S;
  float inv_an = 1.0f;
  if (row >= 0 && __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_PER_NORMAL)) {
    float an = d_normal_absorptance(S, R.live, row, lam, n1, nrm);
    inv_an = an > 0.0f ? 1.0f / an : 0.0f;
  }
  unsigned long long k = atomicAdd(R.rec_n, 1ull);
  if (k >= (unsigned long long)R.rec_cap) return -1;
  float4* r = reinterpret_cast<float4*>(R.rec + k * LUMEN_REC_WORDS);
  r[0] = make_float4(__int_as_float(prev), __int_as_float(sensor), q, time);
  r[1] = make_float4(lam, inv_an, __int_as_float(gen), __int_as_float(vol));
  r[2] = make_float4(x[0], x[1], x[2], d[0]);
  r[3] = make_float4(d[1], d[2], nrm[0], nrm[1]);
  r[4] = make_float4(nrm[2], __int_as_float(0), 0.0f, __int_as_float(0));
  return (int)k;
}

// marks a photon's last record as the head of its chain, with the photon's row weight and event
L_DEV void d_record_head(const Run& R, int last, float w0, int ev) {
  uint32_t* r = R.rec + (size_t)last * LUMEN_REC_WORDS;
  r[17] = 1u;
  r[18] = __float_as_uint(w0);
  r[19] = (uint32_t)ev;
}

struct Dep {
  int sensor;
  float q, time;
  float fates[8];
  float pushed;
};

L_DEV float d_ratio(float live, float ref) { return ref != 0.0f ? live / ref : 0.0f; }

// What a step computes before its query and uses after it: the vertex key, the band at the step's start (before a
// stuck push), the free path drawn at the reference, the medium at the live and reference values. The polarisation
// state after the fill is written back into the photon.
template <class NF>
struct PreT {
  Key vkey;
  NF b0;  // the band at the start, in the navigator's precision (step.py:252)
  float s;
  Med ml, mr;
};
using Pre = PreT<float>;

// the step up to its query: the stuck push, the vertex key, the polarisation fill, the media, the free path
// (step.py:318 _step_context, :245 _recover)
template <int EXT = 0, class NF>
L_DEV void d_pre(const Run& R, PhotonT<NF>& ph, Key pkey, PreT<NF>& pr) {
  const DScene& S = R.S;
  pr.b0 = nav_band(nav_maxabs3(ph.x));
  int stuck = ph.alive && ph.nz >= D_ZSBP;
  if (stuck) {
    NF pb = D_PUSH_BANDS * pr.b0;
#pragma unroll
    for (int a = 0; a < 3; ++a) ph.x[a] = ph.x[a] + pb * ph.d[a];
    ph.vol = nav_locate<EXT>(S, ph.x);
    ph.cls = d_cls(S, ph.vol);
    ph.srf = -1;
  }
  pr.vkey = fold_in(pkey, (uint32_t)ph.vertex);
  if (d_dot(ph.er, ph.er) + d_dot(ph.ei, ph.ei) < D_ZERO_STATE)
    d_fill(ph.d, ph.er, ph.ei, uniform(fold_in(pr.vkey, D_POL_STREAM), 0));
  int mi = __ldg(S.cls_medium + ph.cls);
  pr.ml = d_medium_at(S, R.live, ph.lam, mi);
  pr.mr = R.shared ? pr.ml : d_medium_at(S, R.ref, ph.lam, mi);
  pr.s = -l_log(uniform(pr.vkey, 0)) / d_max(pr.mr.mu_c, D_FLOOR32);
}

// the step's query, bounded just past the free path where no sensor can be met (step.py:260 _query with
// reach.py's bound; the same result as the unbounded query on everything the step reads)
template <int TORUS, class NF>
L_DEV QueryT<NF> d_step_query(const Run& R, const PhotonT<NF>& ph, const PreT<NF>& pr) {
  NF tm = R.reach_on ? nav_reach_bound(R.S, ph.x, ph.d, ph.vol, ph.srf, pr.s, (NF)R.max_distance) : (NF)R.max_distance;
  if constexpr (sizeof(NF) == 8) {  // the direction read in the navigator's precision (navigate.py:682)
    const NF dd[3] = {ph.d[0], ph.d[1], ph.d[2]};
    return nav_query<TORUS>(R.S, ph.x, dd, ph.vol, tm, ph.srf, ph.sn, (NF)pr.s);
  } else {
    return nav_query<TORUS>(R.S, ph.x, ph.d, ph.vol, tm, ph.srf, ph.sn, pr.s);
  }
}

// The GLOSSY outcome's facet path by the row's lobe (surface_event.py:106 _facet_path_branch, :137
// _dielectric_path_branch): the unified path drawn at the reference width and weighted live over reference, or GLISUR's
// metal or dielectric path drawn from the cover at the reference width (1 - polish) and weighted exact over cover.
// Behind the outcome's branch: a detector without glossy rows never runs it.
struct Glossy {
  float d[3];
  float w, wd, dls, sign;
  int far;
};
L_DEV void d_glossy(const Run& R, int row, float sig_r, float sig_l, float n1, float n2, const float* wi,
                     const float* nrm, Key vkey, int want_d, float* er, float* ei, Glossy& g) {
  const DScene& S = R.S;
  int capped = 0;
  int gl = __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_GLISUR);
  float u3 = uniform(vkey, 3), u4 = uniform(vkey, 4), u5 = uniform(vkey, 5);
  g.w = 1.0f; g.wd = 1.0f; g.dls = 0.0f; g.sign = 1.0f; g.far = 0;
  if (gl == 0) {
    float lp = 0.0f, lr = 0.0f;
    int dens = !R.shared || want_d;
    d_facet_path(sig_r, wi, nrm, u3, u4, u5, g.d, er, ei, &capped, dens ? S.uni : nullptr, sig_l, !R.shared, want_d,
                 &lp, &lr, &g.dls);
    if (!R.shared) g.w = l_exp(lp - lr);
  } else if (gl == 1) {
    g.w = d_glisur_metal_path(sig_r, sig_l, wi, nrm, u3, u4, u5, D_GLISUR_COVER, g.d, er, ei, &capped, &g.wd, &g.dls);
    g.sign = -1.0f;
  } else {
    g.w = d_glisur_dielectric_path(sig_r, sig_l, n1, n2, wi, nrm, u3, u4, u5, D_GLISUR_COVER, g.d, er, ei, &g.far,
                                   &capped, &g.wd, &g.dls);
    g.sign = -1.0f;
  }
}

// the step after its query (step.py:516 step: the crossing, the event, the deposit, the roulette)
// the analog photon riding on a tracked one (truth rows; state.py:30 Analog): x uniform on [0, w) while its fate is
// open (inf once decided), k its row's analog weight (<= 1), and at its cathode absorption the sensor (-1 none), time,
// wavelength, the row's 1 / A_n, the crossing point and the volume entered
#define D_ANALOG_STREAM 0x7A4A1061u  // the photon key's fold of its analog uniform (rng.py:23)
struct Ana {
  float x, k;
  int sensor;
  float time, lam, scale, pos[3];
  int vol;
};

template <int G, int ANALOG = 0, class NF = float>
L_DEV void d_post(const Run& R, PhotonT<NF>& ph, float* dw, const PreT<NF>& pr, const QueryT<NF>& q, Dep& dep,
                  float* dq, Ana& an) {
  const DScene& S = R.S;
  const int P = G > 0 ? R.P : 0;
  const NF b0 = pr.b0;
  const float s = pr.s;
  const Key vkey = pr.vkey;
  const Med& ml = pr.ml;
  const Med& mr = pr.mr;
  float er0[3] = {ph.er[0], ph.er[1], ph.er[2]}, ei0[3] = {ph.ei[0], ph.ei[1], ph.ei[2]};
  const int mi = __ldg(S.cls_medium + ph.cls);
  float dmu_abs[G > 0 ? G : 1], dmu_c[G > 0 ? G : 1], dch[G > 0 ? G : 1][LUMEN_N_CHANNEL];
  if (G > 0) {
    const int32_t* m = S.med_i + (size_t)mi * LUMEN_MED_I;
    int ta = __ldg(m + LUMEN_MI_ABS);
    float E = D_HC / ph.lam;
    for (int p = 0; p < P; ++p) {
      dmu_abs[p] = 0.0f;
      if (ta >= 0 && ta == R.gt[p]) dmu_abs[p] = d_tab(S, R.live, ta, E) >= D_FLT_TINY ? -(ml.mu_abs * ml.mu_abs) : 0.0f;
#pragma unroll
      for (int c = 0; c < LUMEN_N_CHANNEL; ++c) {
        int t = d_channel_tab(m, c);
        float L = (t >= 0 && t == R.gt[p]) ? d_tab(S, R.live, t, E) : 0.0f;
        float rc = d_rate(L);
        dch[p][c] = (t >= 0 && t == R.gt[p] && L >= D_FLT_TINY) ? -(rc * rc) : 0.0f;
      }
      dmu_c[p] = (dch[p][0] + dch[p][1]) + dch[p][2];
    }
  }
  float mu_r = mr.mu_c;
  // the sensor a crossing's deposit credits: the one entered, or at an exit sensor's crossing the one left, whose
  // frame the deposit's local fields are read in (step.py:615 _sensor_dep, :653 sensor_frame)
  const int v_sens = (S.pair_pre && q.hit && __ldg(S.pair_pre + q.cls_before * S.n_cls + q.cls_after)) ? q.vol_before
                                                                                                       : q.vol_after;
  int sensor_q = (q.hit && v_sens >= 0) ? vI(S, v_sens, LUMEN_VI_SENSOR) : -1;
  float dist = q.t;
  int zero = dist <= D_ZERO_STEP_BANDS * b0;
  int cb = q.cls_before, ca = q.cls_after;
  int row = __ldg(S.row_of + cb * S.n_cls + ca);
  int cont = (q.cont || (zero && row < 0)) && q.hit;
  if (cont) row = row > 0 ? row : 0;
  int mi_after = __ldg(S.cls_medium + ca);
  int scatter = mu_r > 0.0f && s < dist && ph.alive;
  // A bulk step reads of the crossing's surface row only its detected share (the expected deposit at the crossing),
  // and that share is a * eff: where eff is 0 at this wavelength and moves with no gradient parameter, the row's
  // evaluation is not needed (its outcome probabilities are read by a surface event only)
  int need_eval = !scatter;
  if (scatter && q.hit && ph.alive && row >= 0 && !cont) {
    int te = __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_COL + LUMEN_COL_EFF);
    need_eval = d_tab(S, R.live, te, D_HC / ph.lam) != 0.0f;
    if (G > 0)
      for (int p = 0; p < P; ++p) need_eval = need_eval || te == R.gt[p];
  }
  float dprobs[G > 0 ? G : 1][N_OUT], ddet[G > 0 ? G : 1];
  Eval le, re;
  float n2l = 1.0f;  // the far side's live index (a surface event always evaluates the row)
  if (need_eval) {
    n2l = d_index_at(S, R.live, ph.lam, mi_after);
    d_type_eval<G>(S, R.live, row, ph.lam, ph.d, q.normal, ml.n, n2l, er0, ei0, le, P, R.gt, dprobs, ddet);
    if (R.shared || scatter) re = le;  // a bulk step reads no reference probability
    else {
      float n2r = d_index_at(S, R.ref, ph.lam, mi_after);
      d_type_eval<0>(S, R.ref, row, ph.lam, ph.d, q.normal, mr.n, n2r, er0, ei0, re, 0, R.gt, dprobs, ddet);
    }
  } else {
#pragma unroll
    for (int o = 0; o < N_OUT; ++o) le.probs[o] = 0.0f;
    le.detect = 0.0f;
    le.sigma = 0.1f;
    re = le;
    if (G > 0)
      for (int p = 0; p < P; ++p) {
#pragma unroll
        for (int o = 0; o < N_OUT; ++o) dprobs[p][o] = 0.0f;
        ddet[p] = 0.0f;
      }
  }
  if (cont) {
#pragma unroll
    for (int o = 0; o < N_OUT; ++o) { le.probs[o] = o == STRAIGHT; re.probs[o] = o == STRAIGHT; }
    le.detect = 0.0f;
    re.detect = 0.0f;
    if (G > 0)
      for (int p = 0; p < P; ++p) {
#pragma unroll
        for (int o = 0; o < N_OUT; ++o) dprobs[p][o] = 0.0f;
        ddet[p] = 0.0f;
      }
  }
  // the one defensive mixture at an edge row (estimator.py:146 edge_floor, :83 defensive): each outcome of the row's
  // support whose reference probability is 0 is drawn at e / (1 - e) / n (n of them), the stand-in row of a continue
  // event included; re.probs holds the draw's probabilities from here on (a bulk step draws no outcome)
  if (!scatter && row >= 0) {
    const int cover = __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_COVER);
    if (cover) {
      int n_fl = 0;
#pragma unroll
      for (int o = 0; o < N_OUT; ++o) n_fl += ((cover >> o) & 1) && re.probs[o] <= 0.0f;
      if (n_fl) {
        const float eps = D_EDGE_SHARE / (float)n_fl;
#pragma unroll
        for (int o = 0; o < N_OUT; ++o)
          if (((cover >> o) & 1) && re.probs[o] <= 0.0f) re.probs[o] = eps;
      }
    }
  }
  float p_prop[N_OUT];
  float tot = 0.0f;
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) tot = o == 0 ? re.probs[0] : tot + re.probs[o];
#pragma unroll
  for (int o = 0; o < N_OUT; ++o) p_prop[o] = tot > 0.0f ? re.probs[o] / tot : 0.0f;
  float mu = ml.mu_c;
  int oc_ = scatter ? 0 : d_choose6(p_prop, uniform(vkey, 2));
  int os_ = oc_ > 0 ? oc_ : 0;
  int drawn = oc_ >= 0;
  float reach_live = l_exp(-mu * dist), reach_ref = l_exp(-mu_r * dist);
  float att_if = l_exp(-ml.mu_abs * dist), att_r = l_exp(-mr.mu_abs * dist);
  float v_g = D_C_VACUUM / ml.ng;
  int at_if = q.hit && ph.alive && row >= 0;
  float p_det = le.detect;
  float rr = d_ratio(reach_live, reach_ref);
  dep.q = at_if ? ph.w * reach_live * att_if * p_det : 0.0f;
  float d_reach[G > 0 ? G : 1], d_att[G > 0 ? G : 1];
  if (G > 0)
    for (int p = 0; p < P; ++p) {
      d_reach[p] = -(dmu_c[p] * dist) * reach_live;
      d_att[p] = -(dmu_abs[p] * dist) * att_if;
      float f = reach_live * att_if * p_det;
      float df = d_reach[p] * att_if * p_det + reach_live * d_att[p] * p_det + reach_live * att_if * ddet[p];
      dq[p] = at_if ? dw[p] * f + ph.w * df : 0.0f;
    }
  float lost = (q.hit && ph.alive && row < 0 && !scatter) ? ph.w * rr * att_if : 0.0f;
  NF nx_x[3];
  float nx_d[3], nx_w, nx_dtime, nx_er[3], nx_ei[3], nx_lam = ph.lam;
  int nx_gen = ph.gen;
  float nx_dw[G > 0 ? G : 1];
  int nx_cls, nx_ok, nx_far = 0;
  float fates0, fates1, fates2, wr;
  if (scatter) {
    int next_cls = s < q.t_pass0 ? q.cls_start : (s > q.t_pass1 ? cb : d_cls(S, q.vol_at));
    // the channel drawn from the reference rates (estimator.choose, uniform 1); with one channel present it is that
    // channel whatever the uniform
    float chl[LUMEN_N_CHANNEL], chr_[LUMEN_N_CHANNEL];
    const int32_t* mrec = S.med_i + (size_t)mi * LUMEN_MED_I;
    if (__ldg(mrec + LUMEN_MI_MIE) < 0 && __ldg(mrec + LUMEN_MI_WLS) < 0) {
      // Rayleigh alone: the summed rate is the Rayleigh rate itself (plus exact zeros)
      chl[0] = ml.mu_c; chl[1] = 0.0f; chl[2] = 0.0f;
      chr_[0] = mr.mu_c; chr_[1] = 0.0f; chr_[2] = 0.0f;
    } else {
      d_channel_rates(S, R.live, ph.lam, mi, chl);
      if (R.shared) {
#pragma unroll
        for (int c = 0; c < LUMEN_N_CHANNEL; ++c) chr_[c] = chl[c];
      } else {
        d_channel_rates(S, R.ref, ph.lam, mi, chr_);
      }
    }
    int n_ch = (chr_[0] > 0.0f) + (chr_[1] > 0.0f) + (chr_[2] > 0.0f);
    int cs = chr_[0] > 0.0f ? 0 : (chr_[1] > 0.0f ? 1 : 2);
    if (n_ch > 1) {
      float c0 = chr_[0], c1 = c0 + chr_[1], c2 = c1 + chr_[2];
      float thr = uniform(vkey, 1) * c2;
      cs = c0 > thr ? 0 : (c1 > thr ? 1 : (c2 > thr ? 2 : 0));
    }
    float mu_c_r = chr_[cs], mu_c_l = chl[cs];
    float e_r = l_exp(-mu_r * s), e_l = l_exp(-mu * s);
    float path_r = mu_c_r * e_r;
    float w_path = d_ratio(mu_c_l * e_l, path_r);
    float att = l_exp(-ml.mu_abs * s);
    float w = w_path * att;
    float w_r = d_ratio(path_r, path_r) * l_exp(-mr.mu_abs * s);
#pragma unroll
    for (int a = 0; a < 3; ++a) nx_x[a] = ph.x[a] + s * ph.d[a];
    float rlw = 1.0f, y_w = 1.0f, y_r = 1.0f, delay = 0.0f;
    Bulk2 b2;
    Jmp J;
    J.ok = 0;
    if (cs == 0) {  // Rayleigh: the polarised dipole draw, the state projected (phase.py:57)
      d_rayleigh_sample(er0, ei0, uniform(vkey, 3), uniform(vkey, 4), uniform(vkey, 5), nx_d);
#pragma unroll
      for (int a = 0; a < 3; ++a) { nx_er[a] = er0[a]; nx_ei[a] = ei0[a]; }
      d_project(nx_er, nx_ei, nx_d);
      if (R.jump_on) {  // the diffusion jump (step.py:421)
        if constexpr (sizeof(NF) == 8) {  // the grids are float32: the walk acts at x in float32 (fastpath.py:177)
          const float xs[3] = {(float)nx_x[0], (float)nx_x[1], (float)nx_x[2]};
          d_diffuse(S, mi, xs, nx_d, nx_er, nx_ei, mu_r, ph.alive, vkey, J);
        } else {
          d_diffuse(S, mi, nx_x, nx_d, nx_er, nx_ei, mu_r, ph.alive, vkey, J);
        }
        if (J.ok) {
#pragma unroll
          for (int a = 0; a < 3; ++a) { nx_x[a] = nx_x[a] + J.y[a]; nx_d[a] = J.d[a]; nx_er[a] = J.er[a]; }
        }
      }
    } else {  // Mie (G4OpMieHG) or WLS (G4OpWLS)
      d_bulk_other(S, R.live, R.ref, R.shared, cs, mi, ph.lam, ph.d, er0, ei0, vkey, P, R.gt, b2);
#pragma unroll
      for (int a = 0; a < 3; ++a) { nx_d[a] = b2.d[a]; nx_er[a] = b2.er[a]; nx_ei[a] = b2.ei[a]; }
      rlw = b2.rlw; y_w = b2.y_w; y_r = b2.y_r; delay = b2.delay;
      nx_lam = b2.lam;
      nx_gen = ph.gen + (cs == 2);  // a WLS event re-emits (medium.py:126 reemitted)
    }
    float w_at = ph.w * w_path;
    fates0 = w_at * att * y_w;
    fates1 = w_at * (1.0f - att * y_w);
    fates2 = 0.0f;
    nx_w = ph.w * w * rlw * y_w;
    float wj = 1.0f;
    if (J.ok) {  // the walk's likelihood ratio (fastpath.py:212): its absorption and its path, live over reference
      float lr = l_log(d_max(mu, D_FLOOR32) / d_max(mu_r, D_FLOOR32));
      wj = l_exp(-ml.mu_abs * J.L) * l_exp((float)J.n * lr - (mu - mu_r) * J.L);
      fates1 = fates1 + fates0 * (1.0f - wj);
      fates0 = fates0 * wj;
      nx_w = nx_w * wj;
    }
    if (G > 0)
      for (int p = 0; p < P; ++p) {
        float dwp = (dch[p][cs] * e_l + mu_c_l * (-(dmu_c[p] * s) * e_l)) / path_r;
        if (!(path_r != 0.0f)) dwp = 0.0f;
        float datt = -(dmu_abs[p] * s) * att;
        float dwf = dwp * att + w_path * datt;
        if (cs == 0) nx_dw[p] = dw[p] * w + ph.w * dwf;
        else nx_dw[p] = (dw[p] * w + ph.w * dwf) * rlw * y_w + ph.w * w * rlw * (b2.dlob[p] * y_w + b2.dyld[p]);
        if (J.ok) {
          float dlr = mu > D_FLOOR32 ? dmu_c[p] / mu : 0.0f;
          float dwj = wj * (-(dmu_abs[p] * J.L) + (float)J.n * dlr - dmu_c[p] * J.L);
          nx_dw[p] = nx_dw[p] * wj + ph.w * w * dwj;
        }
      }
    nx_cls = next_cls;
    nx_ok = 1;
    nx_dtime = s / v_g + delay;
    if (J.ok) nx_dtime = nx_dtime + J.L / v_g;
    wr = ph.wr * w_r * y_r;
    if (J.ok) wr = wr * l_exp(-mr.mu_abs * J.L);
  } else {
    float pl = le.probs[os_], pp = p_prop[os_];
    float r_live = drawn ? (pp != 0.0f ? pl / pp : 0.0f) : 0.0f;
    float w_if = ph.w * rr * att_if * r_live;
    float dirn[3], wi[3] = {ph.d[0], ph.d[1], ph.d[2]};
    float lobe_w = 1.0f, lobe_dls = 0.0f, lobe_wd = 1.0f, lobe_sign = 1.0f;  // GLISUR: r = 1 - polish
    int lobe_far = 0;
    const float* nrm = q.normal;
    float eta = ml.n / n2l;
    float s_ax[3];
    d_s_axis(wi, nrm, s_ax);
    Cf es, ep;
    d_components(er0, ei0, wi, s_ax, &es, &ep);
#pragma unroll
    for (int a = 0; a < 3; ++a) { nx_er[a] = er0[a]; nx_ei[a] = ei0[a]; }
    if (os_ == REFRACT) {
      float cos_i = -d_dot(wi, nrm);
      float sin2_t = eta * eta * (1.0f - cos_i * cos_i);
      int tir = sin2_t >= 1.0f;
      float ct2 = 1.0f - sin2_t;
      float cos_t = ct2 > 0.0f ? sqrtf(ct2) : 0.0f;
      if (tir) {
#pragma unroll
        for (int a = 0; a < 3; ++a) dirn[a] = wi[a] + 2.0f * cos_i * nrm[a];
      } else {
        float k = eta * cos_i - cos_t;
#pragma unroll
        for (int a = 0; a < 3; ++a) dirn[a] = eta * wi[a] + k * nrm[a];
        d_unit(dirn);
      }
      float du[3] = {dirn[0], dirn[1], dirn[2]};
      d_unit(du);
      d_recombine(es, ep, le.amps[2], le.amps[3], s_ax, du, nx_er, nx_ei);
    } else if (os_ == SPECULAR) {
      float wn = d_dot(wi, nrm);
#pragma unroll
      for (int a = 0; a < 3; ++a) dirn[a] = wi[a] - 2.0f * wn * nrm[a];
      float du[3] = {dirn[0], dirn[1], dirn[2]};
      d_unit(du);
      d_recombine(es, ep, le.amps[0], le.amps[1], s_ax, du, nx_er, nx_ei);
    } else if (os_ == BACKSCATTER) {
#pragma unroll
      for (int a = 0; a < 3; ++a) { dirn[a] = -wi[a]; nx_er[a] = -er0[a]; nx_ei[a] = -ei0[a]; }
    } else if (os_ == DIFFUSE) {
      d_lambert(nrm, uniform(vkey, 3), uniform(vkey, 4), dirn);
      float h[3] = {dirn[0] - wi[0], dirn[1] - wi[1], dirn[2] - wi[2]};
      d_unit(h);
      d_mirror(nx_er, nx_ei, h);
    } else if (os_ == GLOSSY) {
      Glossy gy;
      d_glossy(R, row, re.sigma, le.sigma, ml.n, n2l, wi, nrm, vkey, P > 0, nx_er, nx_ei, gy);
#pragma unroll
      for (int a = 0; a < 3; ++a) dirn[a] = gy.d[a];
      lobe_w = gy.w; lobe_wd = gy.wd; lobe_dls = gy.dls; lobe_sign = gy.sign; lobe_far = gy.far;
    } else {
#pragma unroll
      for (int a = 0; a < 3; ++a) dirn[a] = wi[a];
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) nx_d[a] = dirn[a];
    d_unit(nx_d);
    int far_side = (os_ == STRAIGHT || os_ == REFRACT);
    int far_ = (far_side || lobe_far) && drawn;
    int ok = q.hit && drawn && row >= 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) nx_x[a] = ph.x[a] + q.t * ph.d[a];
    float r_o = drawn ? (p_prop[os_] != 0.0f ? re.probs[os_] / p_prop[os_] : 0.0f) : 0.0f;
    wr = ph.wr * (reach_ref != 0.0f ? 1.0f : 0.0f) * att_r * r_o * lobe_wd;
    float w_at = ph.w * rr;
    float s_cont = 0.0f;
#pragma unroll
    for (int o = 0; o < N_OUT; ++o) s_cont = o == 0 ? le.probs[0] : s_cont + le.probs[o];
    fates0 = ok ? w_at * att_if * s_cont : 0.0f;
    fates1 = q.hit ? w_at * (1.0f - att_if) : 0.0f;
    fates2 = (q.hit && row >= 0) ? w_at * att_if * (1.0f - s_cont) : 0.0f;
    nx_w = w_if * lobe_w;
    if (G > 0) {
      int t_sig = row >= 0 ? __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_COL +
                                  (lobe_sign > 0.0f ? LUMEN_COL_SIGMA : LUMEN_COL_POLISH)) : -1;
      for (int p = 0; p < P; ++p) {
        float dpl = dprobs[p][os_];
        float dr_live = drawn ? (pp != 0.0f ? dpl / pp : 0.0f) : 0.0f;
        float drr = reach_ref != 0.0f ? d_reach[p] / reach_ref : 0.0f;
        float X = rr * att_if * r_live;
        float dX = drr * att_if * r_live + rr * d_att[p] * r_live + rr * att_if * dr_live;
        float dsig = (t_sig >= 0 && t_sig == R.gt[p]) ? lobe_sign : 0.0f;
        nx_dw[p] = (dw[p] * X + ph.w * dX) * lobe_w + w_if * lobe_w * (lobe_dls * dsig);
      }
    }
    nx_cls = far_ ? ca : cb;
    nx_ok = ok;
    nx_dtime = dist / v_g;
    nx_far = far_;
  }
  float a_surf = ph.alive ? fates2 : 0.0f;
  int far_end = ph.alive && !q.hit && !scatter;
  float d_end = d_min(dist, R.max_distance);
  float w_far = ph.w * d_ratio(l_exp(-mu * d_end), l_exp(-mu_r * d_end));
  float att_far = l_exp(-ml.mu_abs * d_end);
  int cut = R.max_distance < R.reach;
  float escaped = (far_end && !cut) ? w_far * att_far : 0.0f;
  float distance_cut = (far_end && cut) ? w_far * att_far : 0.0f;
  float a_bulk = (ph.alive ? fates1 : 0.0f) + (far_end ? w_far * (1.0f - att_far) : 0.0f);
  float reweighted = (ph.alive && nx_ok) ? fates0 - nx_w : 0.0f;
  float time = ph.t + dist / v_g;
  float w_new = nx_w;
  int low = wr < R.roulette;
  float p_s = wr / R.roulette;
  int keep;
  if (ANALOG) {
    // step.py:625 _analog_crossing: absorbed at the crossing's reached share (x < share), else x - share; decided
    // once x is beyond the weight the event leaves
    const float inf = __int_as_float(0x7f800000);
    float share = (at_if && !scatter) ? ph.w * att_if * p_det : 0.0f;
    if (an.x < share) {
      an.sensor = at_if ? sensor_q : -1;
      an.time = time;
      an.lam = ph.lam;
      an.scale = 1.0f;
      if (row >= 0 && __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_PER_NORMAL)) {
        float a = d_normal_absorptance(S, R.live, row, ph.lam, ml.n, q.normal);
        an.scale = a > 0.0f ? 1.0f / a : 0.0f;
      }
#pragma unroll
      for (int a = 0; a < 3; ++a) an.pos[a] = (float)(ph.x[a] + q.t * ph.d[a]);
      an.vol = v_sens;
      an.x = inf;
    } else {
      float xr = an.x - share;
      an.x = xr < nx_w ? xr : inf;
    }
    // step.py:649 _analog_roulette: an open analog fate is always kept; the keep's total stays p_s
    float pi = wr * an.k;
    float extra = (p_s - pi) / (pi < 1.0f ? 1.0f - pi : 1.0f);
    keep = low ? (an.x < inf || uniform(vkey, 6) < extra) : 0;
  } else {
    keep = low ? (uniform(vkey, 6) < p_s) : 0;
  }
  int kept = low && keep, lostr = low && !keep;
  float p_kept = kept ? p_s : 1.0f;
  if (ANALOG && kept && an.x < __int_as_float(0x7f800000)) an.x = an.x / p_kept;
  float w_in = w_new;
  w_new = kept ? w_new / p_kept : (lostr ? 0.0f : w_new);
  float rouletted = (ph.alive && nx_ok) ? w_in - w_new : 0.0f;
  float wr_new = kept ? wr / p_kept : (lostr ? 0.0f : wr);
  int alive = ph.alive && nx_ok && !lostr;
  int nz_new = (q.hit && !scatter && dist <= D_ZERO_STEP_BANDS * b0) ? ph.nz + 1 : 0;
  int abandon = alive && nz_new >= D_ZSBK;
  float abandoned = abandon ? w_new : 0.0f;
  alive = alive && !abandon;
  int vol_b = s < q.t_pass0 ? q.vol_start : (s > q.t_pass1 ? q.vol_before : q.vol_at);
  int vol = scatter ? vol_b : (nx_far ? q.vol_after : q.vol_before);
  int held = scatter && s <= D_ZERO_STEP_BANDS * b0 && ph.srf >= 0;
  int srf = held ? ph.srf : ((scatter || !q.hit) ? -1 : q.srf);
  float pushed = (ph.alive && ph.nz == D_ZSBP) ? ph.w : 0.0f;
  dep.sensor = at_if ? sensor_q : -1;
  dep.time = time;
  if (R.rec && dep.sensor >= 0) {  // the readout groups' record, at the crossing (step.py:687 _local)
    float xc[3] = {(float)(ph.x[0] + q.t * ph.d[0]), (float)(ph.x[1] + q.t * ph.d[1]), (float)(ph.x[2] + q.t * ph.d[2])};
    ph.last = d_record(R, ph.last, dep.sensor, dep.q, time, ph.lam, ph.gen, row, ml.n, v_sens, xc, ph.d,
                       q.normal);
  }
  dep.fates[0] = lost;
  dep.fates[1] = abandoned;
  dep.fates[2] = escaped;
  dep.fates[3] = distance_cut;
  dep.fates[4] = a_bulk;
  dep.fates[5] = a_surf;
  dep.fates[6] = rouletted;
  dep.fates[7] = reweighted;
  dep.pushed = pushed;
#pragma unroll
  for (int a = 0; a < 3; ++a) { ph.x[a] = nx_x[a]; ph.d[a] = nx_d[a]; ph.er[a] = nx_er[a]; ph.ei[a] = nx_ei[a]; }
  ph.t = ph.t + nx_dtime;
  ph.lam = nx_lam;
  ph.gen = nx_gen;
  ph.w = alive ? w_new : 0.0f;
  ph.wr = alive ? wr_new : 0.0f;
  if (G > 0)
    for (int p = 0; p < P; ++p) {
      float v = kept ? nx_dw[p] / p_kept : (lostr ? 0.0f : nx_dw[p]);
      dw[p] = alive ? v : 0.0f;
    }
  ph.alive = alive;
  ph.vertex += 1;
  ph.vol = vol;
  ph.srf = srf;
  if (!held) {
#pragma unroll
    for (int a = 0; a < 3; ++a) ph.sn[a] = q.normal[a];
  }
  ph.nz = nz_new;
  ph.cls = nx_cls;
}

// A photon born inside a sensor that counts by volume (LumenSceneDesc.cls_born, step.py:574 _born): the entry class
// of its sensor at its first step, else -2
template <class NF>
L_DEV int d_born_entry(const DScene& S, const PhotonT<NF>& ph) {
  if (!S.cls_born || ph.vertex != 0 || !ph.alive || ph.vol < 0) return -2;
  const int bp = __ldg(S.cls_born + ph.cls);
  return (bp >= 0 && vI(S, ph.vol, LUMEN_VI_SENSOR) >= 0) ? bp : -2;
}

// that first step: the deposit of what the sensor's entry (row_of[bp][cls]) detects, evaluated unpolarised at normal
// incidence with both indices 1 (step.py:589), at the emission time; the photon ends, its whole weight absorbed at a
// surface
template <int G, int ANALOG = 0, class NF = float>
L_DEV void d_born(const Run& R, PhotonT<NF>& ph, float* dw, int bp, Dep& dep, float* dq, Ana& an) {
  const DScene& S = R.S;
  const int P = G > 0 ? R.P : 0;
  const int row = __ldg(S.row_of + bp * S.n_cls + ph.cls);
  const int sensor = vI(S, ph.vol, LUMEN_VI_SENSOR);
  float nrm[3] = {-ph.d[0], -ph.d[1], -ph.d[2]};
  float dprobs[G > 0 ? G : 1][N_OUT], ddet[G > 0 ? G : 1];
  Eval ev;
  d_type_eval<G, true>(S, R.live, row, ph.lam, ph.d, nrm, 1.0f, 1.0f, nullptr, nullptr, ev, P, R.gt, dprobs, ddet);
  const float d = ev.detect;
  dep.sensor = sensor;
  dep.q = ph.w * d;
  dep.time = ph.t;
  if (G > 0)
    for (int p = 0; p < P; ++p) dq[p] = dw[p] * d + ph.w * ddet[p];
#pragma unroll
  for (int k = 0; k < 8; ++k) dep.fates[k] = 0.0f;
  dep.fates[5] = ph.w;
  dep.pushed = 0.0f;
  float inv_an = 1.0f;
  if (ANALOG && row >= 0 && __ldg(S.row_i + (size_t)row * LUMEN_ROW_I + LUMEN_RI_PER_NORMAL)) {
    float a = d_normal_absorptance(S, R.live, row, ph.lam, 1.0f, nrm);
    inv_an = a > 0.0f ? 1.0f / a : 0.0f;
  }
  if (R.rec) {  // the readout groups' record at the emission: the point, direction and normal -d, the volume
    float xc[3] = {(float)ph.x[0], (float)ph.x[1], (float)ph.x[2]};
    ph.last = d_record(R, ph.last, sensor, dep.q, ph.t, ph.lam, ph.gen, row, 1.0f, ph.vol, xc, ph.d, nrm);
  }
  if (ANALOG) {  // step.py:597: the analog photon absorbed with the detected share, else decided
    if (an.x < ph.w * d) {
      an.sensor = sensor;
      an.time = ph.t;
      an.lam = ph.lam;
      an.scale = inv_an;
#pragma unroll
      for (int a = 0; a < 3; ++a) an.pos[a] = (float)ph.x[a];
      an.vol = ph.vol;
    }
    an.x = __int_as_float(0x7f800000);
  }
  ph.alive = 0;
  ph.w = 0.0f;
  ph.wr = 0.0f;
  if (G > 0)
    for (int p = 0; p < P; ++p) dw[p] = 0.0f;
  ph.vertex += 1;
}

// one whole step: the megakernel's (k_trace)
template <int G, int TORUS, int ANALOG = 0, class NF = float>
L_DEV void d_step(const Run& R, PhotonT<NF>& ph, float* dw, Key pkey, Dep& dep, float* dq, Ana& an) {
  const int bp = d_born_entry(R.S, ph);
  if (bp != -2) {
    d_born<G, ANALOG>(R, ph, dw, bp, dep, dq, an);
    return;
  }
  PreT<NF> pr;
  d_pre<(TORUS & 1)>(R, ph, pkey, pr);
  QueryT<NF> q = d_step_query<TORUS>(R, ph, pr);
  d_post<G, ANALOG>(R, ph, dw, pr, q, dep, dq, an);
}

// ------------------------------------------------------------------------------------------------ sources
// vol: the start point's volume when the call knows it (every photon of a point-like event starts at the event's
// point, located once: Launch.ev_vol), else -1 (located here)
struct Row { float x[3], d[3], t, lam, w0, er[3], ei[3]; int event; int vol; };

L_DEV float d_gaussian(float u) {
  float f = u - 5.9604644775390625e-8f;
  float v = f * (1.0f - D_NORMAL_LO) + D_NORMAL_LO;
  v = v > D_NORMAL_LO ? v : D_NORMAL_LO;
  return D_SQRT2 * l_erfinv(v);
}

L_DEV int d_event_of(const int64_t* first, int n_ev, int64_t gid) {
  int lo = 0, hi = n_ev - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) / 2;
    if (__ldg((const long long*)first + mid) <= gid) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// 2 pi alpha (Frank-Tamm), the product formed in double and rounded once, as the reference's constant expression
#define D_TWO_PI_ALPHA ((float)(6.283185307179586 * (1.0 / 137.035999084)))

// the components' shares of a material's light (scintillation.py:48 shares): one takes all; two y1 / s and the rest;
// three y_i / s, s = y1 + y2 + y3 (Geant4's default yields 1, 0, 0)
L_DEV void d_scint_shares(const DScene& S, const float* __restrict__ pool, const int32_t* m, float* f) {
  int nc = m[LUMEN_SM_N];
  float y[3];
  for (int i = 0; i < 3; ++i) {
    int t = m[LUMEN_SM_SHARE + i];
    y[i] = t >= 0 ? d_tab(S, pool, t, 1.0f) : (i == 0 ? 1.0f : 0.0f);
  }
  float s = (y[0] + y[1]) + y[2];
  f[0] = 1.0f; f[1] = 0.0f; f[2] = 0.0f;
  if (nc == 2) { f[0] = y[0] / s; f[1] = 1.0f - y[0] / s; }
  if (nc == 3) { f[0] = y[0] / s; f[1] = y[1] / s; f[2] = y[2] / s; }
}

// a photon of a material's scintillation (scintillation.py:69 flash): the component drawn at the reference shares under
// the one defensive mixture (estimator.py:101 defensive_q) and moved to one with light (_base.py:298 lit), its
// wavelength drawn from its reference spectrum under the defensive cover and weighted to the live one (_base.py:337),
// an isotropic direction, the component's decay (and rise) delay, a point or a place along the segment
L_DEV void d_scint_row(const DScene& S, const float* __restrict__ live, const float* __restrict__ ref,
                        const LumenSource& src, const float* f, Key rk, Row& r) {
  const int32_t* m = src.mat;
  const int nc = m[LUMEN_SM_N], seg = m[LUMEN_SM_SEGMENT], rises = m[LUMEN_SM_RISES];
  float fl[3], q[3];
  d_scint_shares(S, live, m, fl);
  d_scint_shares(S, ref, m, q);
  int n_off = 0;
  for (int i = 0; i < nc; ++i) n_off += q[i] <= 0.0f;
  if (n_off > 0) {  // the defensive mixture: a component of share 0 gets e / (1 - e) / n, then all normalised
    float eps = (float)(0.01 / 0.99) / (float)n_off, sum = 0.0f;
    for (int i = 0; i < nc; ++i) { q[i] = q[i] <= 0.0f ? eps : q[i]; sum = i == 0 ? q[i] : sum + q[i]; }
    for (int i = 0; i < nc; ++i) q[i] = q[i] / sum;
  }
  const float u_lam = uniform(rk, 0), u_d0 = uniform(rk, 1), u_d1 = uniform(rk, 2), u_c = uniform(rk, 3);
  const float u_t = uniform(rk, 4);
  int c = 0;
  float cs = 0.0f;
  for (int i = 0; i + 1 < nc; ++i) {
    cs = i == 0 ? q[0] : cs + q[i];
    c += u_c >= cs;
  }
  int nxt = nc, last = 0;  // lit: the first share above zero at or after c, else the last one
  for (int i = nc - 1; i >= 0; --i)
    if (q[i] > 0.0f && i >= c) nxt = i;
  for (int i = 0; i < nc; ++i)
    if (q[i] > 0.0f) last = i;
  c = nxt < last ? nxt : last;
  // the wavelength: the reference spectrum under the cover, the live density over the drawn one
  const int ts = m[LUMEN_SM_SPEC + c];
  const int off = __ldg(S.tab + 2 * ts), k = __ldg(S.tab + 2 * ts + 1);
  const float* er_ = ref + off;
  const float* el = live + off;
  DSpec qs = d_spec(er_, er_ + k, k, 1);
  r.lam = D_HC / d_spec_invert(qs, u_lam);
  const float energy = D_HC / r.lam;
  const float wt = d_safe_div(d_spec_density(el, el + k, k, 0, energy), d_spec_density(er_, er_ + k, k, 1, energy));
  // the direction: z = 1 - 2 u, phi = 2 pi u'
  const float z = 1.0f - 2.0f * u_d0;
  const float sq = 1.0f - z * z;
  const float rr = sq > 0.0f ? sqrtf(sq) : 0.0f;
  float sp, cp;
  l_sincos2pi(u_d1, &sp, &cp);
  r.d[0] = rr * cp; r.d[1] = rr * sp; r.d[2] = z;
  // the delay: Exp(tau), plus Exp(tau rise / (tau + rise)) with rise times (emission.py:48)
  const float tau = d_tab(S, live, m[LUMEN_SM_TAU + c], 1.0f);
  float delay = -tau * l_log(u_t);
  if (rises) {
    const float u_r = uniform(rk, 5 + seg);
    const float rise = d_tab(S, live, m[LUMEN_SM_RISE + c], 1.0f);
    const float s2 = tau + rise;
    delay = delay + -(tau * rise / (s2 > 0.0f ? s2 : 1.0f)) * l_log(u_r);
  }
  // the photons: the yield times the energy, Birks-quenched along a segment (scintillation.py:42 visible_energy)
  const float yl = d_tab(S, live, m[LUMEN_SM_YIELD], 1.0f);
  const float edep = __ldg(f + 8), birks = __ldg(f + 9);
  float n_ph;
  if (seg) {
    float dx = __ldg(f + 4) - __ldg(f + 0), dy = __ldg(f + 5) - __ldg(f + 1), dz = __ldg(f + 6) - __ldg(f + 2);
    float len = sqrtf((dx * dx + dy * dy) + dz * dz);
    float qb = 1.0f + birks * edep / (len > 0.0f ? len : 1.0f);
    n_ph = yl * ((len > 0.0f && edep > 0.0f) ? edep / qb : d_max(edep, 0.0f));
  } else {
    n_ph = yl * edep;
  }
  r.w0 = n_ph / __ldg(f + 10) * d_safe_div(fl[c], q[c]) * wt;
  if (seg) {
    const float u = uniform(rk, 5);
#pragma unroll
    for (int a = 0; a < 3; ++a) r.x[a] = __ldg(f + a) + u * (__ldg(f + 4 + a) - __ldg(f + a));
    r.t = __ldg(f + 3) + u * (__ldg(f + 7) - __ldg(f + 3)) + delay;
  } else {
#pragma unroll
    for (int a = 0; a < 3; ++a) r.x[a] = __ldg(f + a);
    r.t = __ldg(f + 3) + delay;
  }
}

L_DEV void d_source_row(const DScene& S, const float* __restrict__ pool, const float* __restrict__ ref,
                        const LumenSource& src, Key key, int64_t gid, Row& r) {
  Key sk = fold_in(key, D_SOURCE_STREAM);
  Key rk = fold_in(fold_in(sk, (uint32_t)gid), 0u);
  int e = d_event_of(src.ev_first, src.n_events, gid);
  const float* f = src.ev_f + (size_t)e * LUMEN_EV_F;
  r.event = e;
  r.w0 = __ldg(src.ev_w + e);
#pragma unroll
  for (int a = 0; a < 3; ++a) { r.er[a] = 0.0f; r.ei[a] = 0.0f; }
  if (src.kind == LUMEN_SRC_TRACK) {
    float u0 = uniform(rk, 0), u1 = uniform(rk, 1), u2 = uniform(rk, 2);
    float ax[3] = {__ldg(f + 3), __ldg(f + 4), __ldg(f + 5)};
    float along = u0 * __ldg(f + 6);
#pragma unroll
    for (int a = 0; a < 3; ++a) r.x[a] = __ldg(f + a) + along * ax[a];
    float c = src.cone_cos;
    float sn = sqrtf(1.0f - c * c);
    float sp, cp;
    l_sincos2pi(u1, &sp, &cp);
    float l[3] = {sn * cp, sn * sp, c};
    d_to_world(l, ax, r.d);
    r.t = __ldg(f + 7) + along / D_C_VACUUM;
    r.lam = src.lam1 > src.lam0 ? src.lam0 + (src.lam1 - src.lam0) * u2 : src.lam0;
    float ad = d_dot(ax, r.d);
#pragma unroll
    for (int a = 0; a < 3; ++a) r.er[a] = ad * r.d[a] - ax[a];
    d_unit(r.er);
    return;
  }
  if (src.kind == LUMEN_SRC_SCINT_MATERIAL) {
    d_scint_row(S, pool, ref, src, f, rk, r);
    return;
  }
  if (src.kind == LUMEN_SRC_CHERENKOV) {  // cherenkov.py:33 cone: uniforms lam, pos, phi
    float u0 = uniform(rk, 0), u1 = uniform(rk, 1), u2 = uniform(rk, 2);
    float ax[3] = {__ldg(f + 3), __ldg(f + 4), __ldg(f + 5)};
    const float len = __ldg(f + 6), beta = __ldg(f + 8), charge = __ldg(f + 9), samples = __ldg(f + 10);
    float zq = 1.0f / src.lam0 - 1.0f / src.lam1;
    float lam = 1.0f / (1.0f / src.lam0 - u0 * zq);  // ~ 1 / lam^2 over the index table's span
    float n = d_tab(S, pool, src.rindex_tab, D_HC / lam);
    float bn2 = beta * beta * n * n;
    int emits = 1.0f - 1.0f / bn2 > 0.0f;
    float s = emits ? 1.0f - 1.0f / bn2 : 0.0f;
    r.w0 = D_TWO_PI_ALPHA * (charge * charge) * len * s * zq / samples * 1e9f;  // photons per nm -> per m
    float cos_c = emits ? 1.0f / (beta * n) : 1.0f;
    float sq = 1.0f - cos_c * cos_c;
    float sin_c = sq > 0.0f ? sqrtf(sq) : 0.0f;
    float sp, cp;
    l_sincos2pi(u2, &sp, &cp);
    float l[3] = {sin_c * cp, sin_c * sp, cos_c};
    d_to_world(l, ax, r.d);
    float xs = u1 * len;
#pragma unroll
    for (int a = 0; a < 3; ++a) r.x[a] = __ldg(f + a) + xs * ax[a];
    r.t = __ldg(f + 7) + xs / (beta * D_C_VACUUM);
    r.lam = lam;
    float ad = d_dot(ax, r.d);  // Geant4's polarisation (polar.py:81 cherenkov)
#pragma unroll
    for (int a = 0; a < 3; ++a) r.er[a] = ad * r.d[a] - ax[a];
    d_unit(r.er);
    return;
  }
  float g[3] = {d_gaussian(uniform(rk, 0)), d_gaussian(uniform(rk, 1)), d_gaussian(uniform(rk, 2))};
  d_unit(g);
#pragma unroll
  for (int a = 0; a < 3; ++a) { r.x[a] = __ldg(f + a); r.d[a] = g[a]; }
  float u3 = uniform(rk, 3);
  r.lam = src.lam1 > src.lam0 ? src.lam0 + (src.lam1 - src.lam0) * u3 : src.lam0;
  r.t = __ldg(f + 3);
  if (src.kind == LUMEN_SRC_SCINT) {
    float u4 = uniform(rk, 4), u5 = uniform(rk, 5);
    float tau = u4 < src.frac1 ? src.tau1 : src.tau2;
    r.t = __ldg(f + 3) + -l_log(u5) * tau;
  }
}

L_DEV void d_rows_row(const LumenRows& rows, int64_t i, Row& r) {
  r.x[0] = __ldg(rows.x + i); r.x[1] = __ldg(rows.y + i); r.x[2] = __ldg(rows.z + i);
  r.d[0] = __ldg(rows.dx + i); r.d[1] = __ldg(rows.dy + i); r.d[2] = __ldg(rows.dz + i);
  r.t = __ldg(rows.t + i); r.lam = __ldg(rows.lam + i); r.w0 = __ldg(rows.w + i);
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    r.er[a] = rows.pol ? __ldg(rows.pol + 6 * i + a) : 0.0f;
    r.ei[a] = rows.pol ? __ldg(rows.pol + 6 * i + 3 + a) : 0.0f;
  }
  r.event = rows.event ? __ldg(rows.event + i) : 0;
}

template <int EXT = 0, class NF>
L_DEV void d_start(const DScene& S, const Row& r, PhotonT<NF>& ph) {
#pragma unroll
  for (int a = 0; a < 3; ++a) { ph.x[a] = r.x[a]; ph.d[a] = r.d[a]; ph.er[a] = r.er[a]; ph.ei[a] = r.ei[a]; ph.sn[a] = 0.0f; }
  ph.t = r.t;
  ph.lam = r.lam;
  ph.w = 1.0f;
  ph.wr = 1.0f;
  ph.alive = 1;
  ph.vertex = 0;
  ph.vol = r.vol >= 0 ? r.vol : nav_locate<EXT>(S, ph.x);
  ph.cls = d_cls(S, ph.vol);
  ph.srf = -1;
  ph.nz = 0;
  ph.gen = 0;
  ph.last = -1;
}

}  // namespace lb
