/* The checker's readout groups: the histograms of src/lumen/readout/grid.py (charge_cells :183, time_cells :210,
 * hats :165, cells :173, _time_weights :195) filled from one photon's deposit records as src/lumen/readout/fill.py:88
 * readout does (the adds of every record; the moments :200 charge2 and pe2 summed per photon before the square), and
 * the deposit's 1 / A_n (src/lumen/surfaces/types.py:397 normal_absorptance). Test infrastructure: the engine's
 * records and k_bin are checked against it. */
#pragma once

#include <map>
#include <utility>
#include <vector>

/* one deposit record: the crossing's facts in world coordinates (the features read them in the sensor placement's
   frame, src/lumen/transport/step.py:663 sensor_frame, :670 _frame_fields) */
typedef struct ORec {
  int sensor, gen, vol;
  float q, time, lam, inv_an;
  float x[3], d[3], n[3];
} ORec;

/* A_n of a row at normal incidence, unpolarised, eff 1 (types.py:391 _normal_incidence: wi = -n): the chain's
   absorbed rest of the cut reflectance and T; a complex index's reflectance 0.5 (|r_s|^2 + |r_p|^2) (fresnel.py:53) */
static inline float o_normal_absorptance(const LumenSceneDesc* D, const float* pool, int row, float lam, float n1,
                                         const float* nrm) {
  const int32_t* ri = D->row_i + (size_t)row * LUMEN_ROW_I;
  float E = O_HC / lam;
  float Rc = o_tab(D, pool, ri[LUMEN_RI_COL + LUMEN_COL_R], E, 0);
  if (ri[LUMEN_RI_MODEL] == 2) {
    float wi[3] = {-nrm[0], -nrm[1], -nrm[2]};
    float cos_i = o_clip01(-((wi[0] * nrm[0] + wi[1] * nrm[1]) + wi[2] * nrm[2]));
    Oc amps[4];
    o_amplitudes(cos_i, n1, oc(o_tab(D, pool, ri[LUMEN_RI_COL + LUMEN_COL_NR], E, 0),
                               o_tab(D, pool, ri[LUMEN_RI_COL + LUMEN_COL_NK], E, 0)), amps);
    Rc = o_clip01(0.5f * (oc_abs2(amps[0]) + oc_abs2(amps[1])));
  }
  float cut[2] = {Rc, o_tab(D, pool, ri[LUMEN_RI_COL + LUMEN_COL_T], E, 0)}, z[2] = {0.0f, 0.0f}, out[3], dout[3];
  o_chained(2, cut, z, out, dout);
  return out[2];
}

/* v in the frame of volume pose vf (R row-major, then t): R^T v */
static inline void o_to_placement(const float* vf, const float* v, float* l) {
  for (int j = 0; j < 3; ++j) l[j] = (v[0] * vf[j] + v[1] * vf[3 + j]) + v[2] * vf[6 + j];
}

/* a deposit's feature (src/lumen/sensors/features.py) */
static float o_feature(const LumenSceneDesc* D, int f, const ORec& r) {
  if (f == LUMEN_FEAT_WAVELENGTH) return r.lam;
  if (f == LUMEN_FEAT_GENERATION) return (float)r.gen;
  const float* vf = D->vol_f + (size_t)r.vol * LUMEN_VOL_F;
  if (f == LUMEN_FEAT_COS_INCIDENCE) { /* features.py:40 |dir . normal| */
    float dl[3], nl[3];
    o_to_placement(vf, r.d, dl);
    o_to_placement(vf, r.n, nl);
    return fabsf((dl[0] * nl[0] + dl[1] * nl[1]) + dl[2] * nl[2]);
  }
  float y[3] = {r.x[0] - vf[9], r.x[1] - vf[10], r.x[2] - vf[11]}, p[3];
  o_to_placement(vf, y, p);
  if (f == LUMEN_FEAT_THETA) return o_atan2(sqrtf((p[0] * p[0] + p[1] * p[1]) + 1e-30f), p[2]); /* :20 polar_angle */
  if (f == LUMEN_FEAT_X) return p[0];
  if (f == LUMEN_FEAT_Y) return p[1];
  if (f == LUMEN_FEAT_Z) return p[2];
  return sqrtf(p[0] * p[0] + p[1] * p[1]); /* rho */
}

static inline int o_axis_size(const LumenAxis& a) { return a.knots ? a.n : a.n - 1; }

/* (index, weight) pairs of a value on one axis (grid.py:90 Axis.cells, :165 hats) */
static void o_axis_pairs(const LumenAxis& a, float x, std::vector<std::pair<int, float>>& out) {
  out.clear();
  int below = 0; /* searchsorted(values, x, side="right") */
  while (below < a.n && a.values[below] <= x) ++below;
  if (a.knots) {
    int i = below - 1;
    if (i < 0) i = 0;
    if (i > a.n - 2) i = a.n - 2;
    float f = o_clip01((x - a.values[i]) / (a.values[i + 1] - a.values[i]));
    out.push_back({i, 1.0f - f});
    out.push_back({i + 1, f});
  } else {
    int b = below - 1;
    out.push_back({(b >= 0 && b < a.n - 1) ? b : -1, 1.0f});
  }
}

/* the row-major cells of a record over axes [a0, a0 + na) of a group (grid.py:173 cells; [(0, 1)] without) */
static std::vector<std::pair<int, float>> o_group_cells(const LumenSceneDesc* D, const LumenGroup& G, int a0, int na,
                                                        const ORec& r) {
  std::vector<std::pair<int, float>> cur, ax;
  if (na == 0) return {{0, 1.0f}};
  o_axis_pairs(G.axes[a0], o_feature(D, G.axes[a0].feature, r), cur);
  for (int k = 1; k < na; ++k) {
    const LumenAxis& A = G.axes[a0 + k];
    o_axis_pairs(A, o_feature(D, A.feature, r), ax);
    std::vector<std::pair<int, float>> nx;
    for (auto& p : cur)
      for (auto& q : ax)
        nx.push_back({(p.first >= 0 && q.first >= 0) ? p.first * o_axis_size(A) + q.first : -1, p.second * q.second});
    cur.swap(nx);
  }
  return cur;
}

static int o_cells_of(const LumenGroup& G, int a0, int na) {
  int c = 1;
  for (int k = 0; k < na; ++k) c *= o_axis_size(G.axes[a0 + k]);
  return c;
}

/* one thread's group cells (FP64), merged into the caller's at the end */
typedef struct OGroupT {
  std::vector<std::vector<double>> charge, charge2, time, over_q, over_qt;
  std::vector<double> pe2;
} OGroupT;

static void o_groups_init(OGroupT* T, const LumenTallies* out, int E, int S) {
  int ng = out->n_groups;
  T->charge.resize(ng); T->charge2.resize(ng); T->time.resize(ng); T->over_q.resize(ng); T->over_qt.resize(ng);
  for (int g = 0; g < ng; ++g) {
    const LumenGroup& G = out->groups[g];
    size_t nc = (size_t)E * G.n_sensors * o_cells_of(G, 0, G.n_axes);
    size_t nd = (size_t)E * G.n_sensors * o_cells_of(G, G.n_axes, G.n_delay);
    T->charge[g].assign(nc, 0.0);
    T->charge2[g].assign(nc, 0.0);
    T->time[g].assign(G.nt > 0 ? nd * G.nt : 0, 0.0);
    T->over_q[g].assign(G.nt > 0 ? nd * 2 : 0, 0.0);
    T->over_qt[g].assign(G.nt > 0 ? nd * 2 : 0, 0.0);
  }
  T->pe2.assign(out->pe2 ? (size_t)E * S : 0, 0.0);
}

/* the group and the position in it of a detector sensor (-1: none) */
static int o_group_of(const LumenTallies* out, int s, int* pos) {
  for (int g = 0; g < out->n_groups; ++g) {
    const LumenGroup& G = out->groups[g];
    int p = G.index ? G.index[s] : (s < G.n_sensors ? s : -1);
    if (p >= 0) { *pos = p; return g; }
  }
  return -1;
}

/* one photon's records into the groups' cells (fill.py:88 readout: emits and moments), row weight w0, event e */
static void o_bin_photon(const LumenSceneDesc* D, const LumenTallies* out, const std::vector<ORec>& recs, double w0,
                         int e, int S, OGroupT* T) {
  std::map<std::pair<int, long long>, double> m2; /* (group, cell) -> the photon's adds, squared at the end */
  std::map<int, double> mpe;                      /* sensor -> the photon's pe at the groups' acceptance */
  for (const ORec& r : recs) {
    int pos = -1, g = o_group_of(out, r.sensor, &pos);
    float pe_v = 0.0f;
    int has_pe = 0;
    if (g >= 0) {
      const LumenGroup& G = out->groups[g];
      const float qd = G.normalise ? r.q * r.inv_an : r.q;
      const auto cells = o_group_cells(D, G, 0, G.n_axes, r);
      const long long base = ((long long)e * G.n_sensors + pos) * o_cells_of(G, 0, G.n_axes);
      float acc = 0.0f; /* the acceptance at the record's cells (fill.py:314 detection_weight) */
      for (auto& c : cells) {
        if (c.first < 0) continue;
        double v = (double)(qd * c.second) * w0;
        T->charge[g][base + c.first] += v;
        m2[{g, base + c.first}] += v;
        if (G.weights) acc = acc + c.second * G.weights[c.first];
      }
      if (G.weights) { pe_v = qd * acc; has_pe = 1; }
      if (G.nt > 0) { /* grid.py:195 the four nodes' cubic Lagrange weights, the overflow beyond the ends */
        const float qq = qd * (G.weighted ? acc : 1.0f);
        float x = (r.time - G.t0) / G.dt;
        if (x < -4.0f) x = -4.0f;
        if (x > (float)G.nt + 4.0f) x = (float)G.nt + 4.0f;
        const float jf = floorf(x), gg = x - jf;
        const int j = (int)jf;
        const int node[4] = {j - 1, j, j + 1, j + 2};
        const float f[4] = {-gg * (gg - 1.0f) * (gg - 2.0f) / 6.0f, (gg + 1.0f) * (gg - 1.0f) * (gg - 2.0f) / 2.0f,
                            -(gg + 1.0f) * gg * (gg - 2.0f) / 2.0f, (gg + 1.0f) * gg * (gg - 1.0f) / 6.0f};
        float late = 0.0f, early = 0.0f;
        for (int k = 0; k < 4; ++k) {
          late = late + (node[k] >= G.nt ? f[k] : 0.0f);
          early = early + (node[k] < 0 ? f[k] : 0.0f);
        }
        const int nd = o_cells_of(G, G.n_axes, G.n_delay);
        for (auto& b : o_group_cells(D, G, G.n_axes, G.n_delay, r)) {
          if (b.first < 0) continue;
          const long long row = ((long long)e * G.n_sensors + pos) * nd + b.first;
          for (int k = 0; k < 4; ++k)
            if (node[k] >= 0 && node[k] < G.nt) T->time[g][row * G.nt + node[k]] += (double)(qq * (b.second * f[k])) * w0;
          const float ow[2] = {b.second * late, b.second * early};
          for (int side = 0; side < 2; ++side) {
            float a = qq * ow[side];
            T->over_q[g][row * 2 + side] += (double)a * w0;
            T->over_qt[g][row * 2 + side] += (double)(a * r.time) * w0;
          }
        }
      }
    }
    if (!T->pe2.empty() && r.sensor >= 0 && r.sensor < S && has_pe) mpe[r.sensor] += (double)pe_v * w0;
  }
  for (auto& kv : m2) T->charge2[kv.first.first][kv.first.second] += kv.second * kv.second;
  for (auto& kv : mpe) T->pe2[(size_t)e * S + kv.first] += kv.second * kv.second;
}
