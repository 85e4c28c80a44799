// The readout groups' histograms from the deposit records (src/lumen/readout/grid.py charge_cells :183, time_cells
// :210, hats :165, cells :173; src/lumen/readout/fill.py:88 readout with its moments :200 and detection_weight :314).
//
// The trace appends one record per sensor deposit (d_record) and links each to the photon's previous one; the
// photon's last record is its chain's head (d_record_head: the row weight and the event). k_bin gives each head's
// photon to one thread, which walks the chain: the charge cells and the time nodes take every record's adds, and the
// per-photon moments (charge2 per cell, pe2 per sensor) sum the photon's adds to a key before squaring them, exactly
// (the first record of a key in the walk sums the chain's adds to it).
#pragma once

namespace lb {

#define D_MAX_CELLS 16  // 2^LUMEN_MAX_AXES: the (cell, weight) pairs of one deposit over a group's axes

struct Bin {
  LumenGroup g[LUMEN_MAX_GROUPS];
  int n_groups, E, S_;
  const uint32_t* rec;
  const unsigned long long* n;   // the call's record count
  long long cap;
  double* pe2;
  const float* vol_f;            // the volumes' poses (the sensor placement's frame)
  unsigned long long* counts;    // counts[LUMEN_C_RECORDS] takes the call's record count
};

L_DEV float rec_f(const uint32_t* r, int k) { return __uint_as_float(__ldg(r + k)); }
L_DEV int rec_i(const uint32_t* r, int k) { return (int)__ldg(r + k); }

// R^T v of a volume's pose (R row-major): the vector in the placement's frame (step.py:678 R.T @ v)
L_DEV void d_local(const float* vf, const float* v, float* l) {
#pragma unroll
  for (int j = 0; j < 3; ++j) l[j] = (v[0] * __ldg(vf + j) + v[1] * __ldg(vf + 3 + j)) + v[2] * __ldg(vf + 6 + j);
}

// a deposit's feature (src/lumen/sensors/features.py BUILTIN), from its record
L_DEV float d_feature(const Bin& B, int f, const uint32_t* r) {
  if (f == LUMEN_FEAT_WAVELENGTH) return rec_f(r, 4);
  if (f == LUMEN_FEAT_GENERATION) return (float)rec_i(r, 6);
  const float* vf = B.vol_f + (size_t)rec_i(r, 7) * LUMEN_VOL_F;
  if (f == LUMEN_FEAT_COS_INCIDENCE) {  // |dir . normal| in the placement's frame
    float d[3] = {rec_f(r, 11), rec_f(r, 12), rec_f(r, 13)}, n[3] = {rec_f(r, 14), rec_f(r, 15), rec_f(r, 16)};
    float dl[3], nl[3];
    d_local(vf, d, dl);
    d_local(vf, n, nl);
    return fabsf((dl[0] * nl[0] + dl[1] * nl[1]) + dl[2] * nl[2]);
  }
  float y[3] = {rec_f(r, 8) - __ldg(vf + 9), rec_f(r, 9) - __ldg(vf + 10), rec_f(r, 10) - __ldg(vf + 11)}, p[3];
  d_local(vf, y, p);
  switch (f) {
    case LUMEN_FEAT_THETA: return l_atan2(sqrtf((p[0] * p[0] + p[1] * p[1]) + 1e-30f), p[2]);
    case LUMEN_FEAT_X: return p[0];
    case LUMEN_FEAT_Y: return p[1];
    case LUMEN_FEAT_Z: return p[2];
    default: return sqrtf(p[0] * p[0] + p[1] * p[1]);  // LUMEN_FEAT_RHO
  }
}

L_DEV int d_axis_size(const LumenAxis& a) { return a.knots ? a.n : a.n - 1; }

// (cell, weight) pairs of x on one axis: hat functions on knots (constant beyond the end knots), else one cell
// between edges (-1 outside); returns the pair count
L_DEV int d_axis_cells(const LumenAxis& a, float x, int* idx, float* w) {
  const float* v = a.values;
  int lo = 0, hi = a.n;  // searchsorted(v, x, side="right"): the values <= x
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (__ldg(v + mid) <= x) lo = mid + 1;
    else hi = mid;
  }
  if (a.knots) {
    int i = lo - 1;
    i = i < 0 ? 0 : (i > a.n - 2 ? a.n - 2 : i);
    float k0 = __ldg(v + i), k1 = __ldg(v + i + 1);
    float f = d_clip01((x - k0) / (k1 - k0));
    idx[0] = i; w[0] = 1.0f - f;
    idx[1] = i + 1; w[1] = f;
    return 2;
  }
  int b = lo - 1;
  idx[0] = (b >= 0 && b < a.n - 1) ? b : -1;
  w[0] = 1.0f;
  return 1;
}

// the row-major (cell, weight) pairs of a record over axes a0 .. a0 + na - 1 of a group ((0, 1) without axes)
L_DEV int d_cells(const Bin& B, const LumenGroup& G, int a0, int na, const uint32_t* r, int* idx, float* w) {
  if (na == 0) { idx[0] = 0; w[0] = 1.0f; return 1; }
  int m = d_axis_cells(G.axes[a0], d_feature(B, G.axes[a0].feature, r), idx, w);
  for (int k = 1; k < na; ++k) {
    const LumenAxis& A = G.axes[a0 + k];
    int ci[2];
    float cw[2];
    int mc = d_axis_cells(A, d_feature(B, A.feature, r), ci, cw);
    int size = d_axis_size(A);
    int ni[D_MAX_CELLS];
    float nw[D_MAX_CELLS];
    int t = 0;
    for (int p = 0; p < m; ++p)
      for (int q = 0; q < mc; ++q) {
        ni[t] = (idx[p] >= 0 && ci[q] >= 0) ? idx[p] * size + ci[q] : -1;
        nw[t] = w[p] * cw[q];
        ++t;
      }
    for (int j = 0; j < t; ++j) { idx[j] = ni[j]; w[j] = nw[j]; }
    m = t;
  }
  return m;
}

L_DEV int d_n_cells(const LumenGroup& G, int a0, int na) {
  int c = 1;
  for (int k = 0; k < na; ++k) c *= d_axis_size(G.axes[a0 + k]);
  return c;
}

// a record's group and position in it (-1: in no group), its charge cells and its deposit (over A_n on a
// normalising grid)
struct RecCells {
  int g, pos, m;
  int idx[D_MAX_CELLS];
  float w[D_MAX_CELLS];
  float qd;
};

L_DEV void d_rec_cells(const Bin& B, const uint32_t* r, RecCells& c) {
  int s = rec_i(r, 1);
  c.g = -1;
  c.pos = -1;
  c.m = 0;
  for (int g = 0; g < B.n_groups && c.g < 0; ++g) {
    const LumenGroup& G = B.g[g];
    int p = G.index ? __ldg(G.index + s) : (s < G.n_sensors ? s : -1);
    if (p >= 0) { c.g = g; c.pos = p; }
  }
  if (c.g < 0) return;
  const LumenGroup& G = B.g[c.g];
  c.m = d_cells(B, G, 0, G.n_axes, r, c.idx, c.w);
  float q = rec_f(r, 2);
  c.qd = G.normalise ? q * rec_f(r, 5) : q;
}

// the acceptance read at a record's charge cells (fill.py:314 detection_weight)
L_DEV float d_acceptance(const LumenGroup& G, const RecCells& c) {
  float a = 0.0f;
  for (int j = 0; j < c.m; ++j)
    if (c.idx[j] >= 0) a = a + c.w[j] * __ldg(G.weights + c.idx[j]);
  return a;
}

L_DEV long long rec_prev(const Bin& B, long long k) { return (long long)rec_i(B.rec + k * LUMEN_REC_WORDS, 0); }

L_DEV void d_bin_photon(const Bin& B, long long head) {
  const uint32_t* h = B.rec + head * LUMEN_REC_WORDS;
  const double w0 = (double)rec_f(h, 18);
  const int e = rec_i(h, 19);
  if ((unsigned)e >= (unsigned)B.E) return;
  for (long long k = head; k >= 0; k = rec_prev(B, k)) {  // every record's adds
    const uint32_t* r = B.rec + k * LUMEN_REC_WORDS;
    RecCells c;
    d_rec_cells(B, r, c);
    if (c.g < 0) continue;
    const LumenGroup& G = B.g[c.g];
    const size_t base = ((size_t)e * G.n_sensors + c.pos) * (size_t)d_n_cells(G, 0, G.n_axes);
    for (int j = 0; j < c.m; ++j)
      if (c.idx[j] >= 0) {
        double v = (double)(c.qd * c.w[j]) * w0;
        if (v != 0.0) atomicAdd(G.charge + base + c.idx[j], v);
      }
    if (G.nt > 0) {  // the time nodes: the cubic Lagrange split over the four nearest (grid.py:195 _time_weights)
      const float qq = c.qd * (G.weighted ? d_acceptance(G, c) : 1.0f);
      const float t = rec_f(r, 3);
      float x = (t - G.t0) / G.dt;
      x = x < -4.0f ? -4.0f : (x > (float)G.nt + 4.0f ? (float)G.nt + 4.0f : x);
      const float j0 = floorf(x), g = x - j0;
      const int ji = (int)j0;
      const float f[4] = {-g * (g - 1.0f) * (g - 2.0f) / 6.0f, (g + 1.0f) * (g - 1.0f) * (g - 2.0f) / 2.0f,
                          -(g + 1.0f) * g * (g - 2.0f) / 2.0f, (g + 1.0f) * g * (g - 1.0f) / 6.0f};
      float late = 0.0f, early = 0.0f;
      for (int m = 0; m < 4; ++m) {
        int node = ji - 1 + m;
        late = late + (node >= G.nt ? f[m] : 0.0f);
        early = early + (node < 0 ? f[m] : 0.0f);
      }
      int di[D_MAX_CELLS];
      float dwt[D_MAX_CELLS];
      const int md = d_cells(B, G, G.n_axes, G.n_delay, r, di, dwt);
      const size_t nd = (size_t)d_n_cells(G, G.n_axes, G.n_delay);
      for (int b = 0; b < md; ++b) {
        if (di[b] < 0) continue;
        const size_t row = ((size_t)e * G.n_sensors + c.pos) * nd + di[b];
        for (int m = 0; m < 4; ++m) {
          int node = ji - 1 + m;
          if (node < 0 || node >= G.nt) continue;
          double v = (double)(qq * (dwt[b] * f[m])) * w0;
          if (v != 0.0) atomicAdd(G.time + row * G.nt + node, v);
        }
        const float ow[2] = {dwt[b] * late, dwt[b] * early};
        for (int side = 0; side < 2; ++side) {
          float a = qq * ow[side];
          if (a == 0.0f) continue;
          atomicAdd(G.over_q + row * 2 + side, (double)a * w0);
          atomicAdd(G.over_qt + row * 2 + side, (double)(a * t) * w0);
        }
      }
    }
  }
  // charge2: per cell, the square of the photon's adds summed (the first record of the cell in the walk sums them)
  for (long long k = head; k >= 0; k = rec_prev(B, k)) {
    RecCells c;
    d_rec_cells(B, B.rec + k * LUMEN_REC_WORDS, c);
    if (c.g < 0) continue;
    const LumenGroup& G = B.g[c.g];
    const size_t base = ((size_t)e * G.n_sensors + c.pos) * (size_t)d_n_cells(G, 0, G.n_axes);
    for (int j = 0; j < c.m; ++j) {
      const int cell = c.idx[j];
      if (cell < 0) continue;
      int dup = 0;
      for (int jj = 0; jj < j; ++jj) dup = dup || c.idx[jj] == cell;
      for (long long k2 = head; k2 != k && !dup; k2 = rec_prev(B, k2)) {
        RecCells c2;
        d_rec_cells(B, B.rec + k2 * LUMEN_REC_WORDS, c2);
        if (c2.g == c.g && c2.pos == c.pos)
          for (int j2 = 0; j2 < c2.m; ++j2) dup = dup || c2.idx[j2] == cell;
      }
      if (dup) continue;
      double x = 0.0;
      for (long long k3 = head; k3 >= 0; k3 = rec_prev(B, k3)) {
        RecCells c3;
        d_rec_cells(B, B.rec + k3 * LUMEN_REC_WORDS, c3);
        if (c3.g == c.g && c3.pos == c.pos)
          for (int j3 = 0; j3 < c3.m; ++j3)
            if (c3.idx[j3] == cell) x += (double)(c3.qd * c3.w[j3]) * w0;
      }
      if (x != 0.0) atomicAdd(G.charge2 + base + cell, x * x);
    }
  }
  if (!B.pe2) return;
  // pe2: per detector sensor, the square of the photon's pe at the groups' acceptance (fill.py:200 moments)
  for (long long k = head; k >= 0; k = rec_prev(B, k)) {
    const int s = rec_i(B.rec + k * LUMEN_REC_WORDS, 1);
    if ((unsigned)s >= (unsigned)B.S_) continue;
    int dup = 0;
    for (long long k2 = head; k2 != k && !dup; k2 = rec_prev(B, k2)) dup = rec_i(B.rec + k2 * LUMEN_REC_WORDS, 1) == s;
    if (dup) continue;
    double x = 0.0;
    for (long long k3 = head; k3 >= 0; k3 = rec_prev(B, k3)) {
      const uint32_t* r3 = B.rec + k3 * LUMEN_REC_WORDS;
      if (rec_i(r3, 1) != s) continue;
      RecCells c3;
      d_rec_cells(B, r3, c3);
      if (c3.g < 0 || !B.g[c3.g].weights) continue;
      x += (double)(c3.qd * d_acceptance(B.g[c3.g], c3)) * w0;
    }
    if (x != 0.0) atomicAdd(B.pe2 + (size_t)e * B.S_ + s, x * x);
  }
}

// one thread per record; the heads bin their photons (a grid-stride loop over the call's records)
__global__ void __launch_bounds__(256) k_bin(Bin B) {
  const unsigned long long n = *B.n;
  if (blockIdx.x == 0 && threadIdx.x == 0 && B.counts && n) atomicAdd(B.counts + LUMEN_C_RECORDS, n);
  if (n > (unsigned long long)B.cap) return;  // past the scratch: the chains are incomplete (LUMEN_ERR_RECORDS)
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)n; i += stride)
    if (__ldg(B.rec + i * LUMEN_REC_WORDS + 17)) d_bin_photon(B, i);
}

}  // namespace lb
