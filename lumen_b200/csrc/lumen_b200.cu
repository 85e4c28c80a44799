// lumen_b200: the B200 photon-transport engine behind the C ABI of include/lumen_b200.h.
//
// The reference's photon loop (src/lumen/run.py:293-368) is a tallymap kernel with one item per photon and a lane
// refill per step, followed by record launches that fold deposits into per-sensor cells (run.py:443-557). Here one
// persistent kernel does both: each thread carries one photon in registers, steps it, and when it ends takes the
// next photon id from a global counter (one atomic per warp, ballot-compacted), so lanes stay busy as paths end at
// different steps. Deposits go straight into FP64 per-sensor tallies (arrival, arrival x time, time histograms,
// Jacobian); the per-photon second moment is formed from a four-entry per-thread cache of the photon's per-sensor
// sums, squared when the photon ends; a photon's sums past its first four sensors go to the call's moment table (a
// hash of (photon, event x sensor) to its sum in HBM), squared by a pass after the launch, so the moment is exact for
// any number of sensors; health fates and counters are reduced per block before their atomics.
//
// Numerics: compiled with -fmad=false; every fused multiply-add is an explicit fmaf, every elementary function the
// library's own (dmath.cuh), so a photon's path is the CPU checker's bit for bit.
#include <limits>

#include "engine.cuh"
#include "dreadout.cuh"

// ------------------------------------------------------------------------------------------- error handling
std::string& lumen_err() {
  static thread_local std::string e;
  return e;
}
long long& lumen_launches() {
  static thread_local long long n = 0;
  return n;
}
#define g_err lumen_err()
// every entry point starts here: no error yet, no kernel launched
static void begin_call() {
  lumen_err().clear();
  lumen_launches() = 0;
}

// the launchers instantiated in the other parts of the build
#define LUMEN_EXTERN_SHAPE(G, B, M, T, A, N) extern template LUMEN_SHAPE_DECL(G, B, M, T, A, N)
LUMEN_SHAPES(LUMEN_EXTERN_SHAPE)
extern template int run_wave<0>(const Launch&, const Pick&, unsigned long long*, cudaStream_t, int, int, int, float*);
extern template int run_wave<LUMEN_MAX_GRAD>(const Launch&, const Pick&, unsigned long long*, cudaStream_t, int, int,
                                             int, float*);
extern template int launch_event_locate<0>(const DScene&, const LumenSource&, int32_t*, cudaStream_t);
extern template int launch_event_locate<1>(const DScene&, const LumenSource&, int32_t*, cudaStream_t);
extern template int launch_photons<0>(const Launch&, int32_t*, float*, cudaStream_t);
extern template int launch_photons<1>(const Launch&, int32_t*, float*, cudaStream_t);
extern template int launch_query<float>(const DScene&, const float*, const int32_t*, const int32_t*, float, int64_t,
                                        int32_t*, float*, cudaStream_t);
extern template int launch_query<double>(const DScene&, const double*, const int32_t*, const int32_t*, double, int64_t,
                                         int32_t*, double*, cudaStream_t);
extern template int launch_locate<float>(const DScene&, const float*, int64_t, int32_t*, cudaStream_t);
extern template int launch_locate<double>(const DScene&, const double*, int64_t, int32_t*, cudaStream_t);

// squares every held sum into arrival2 and frees its slot (grid-stride over the table)
__global__ void k_moment_flush(Tally T) {
  for (size_t h = (size_t)blockIdx.x * blockDim.x + threadIdx.x; h <= T.mt_mask; h += (size_t)gridDim.x * blockDim.x) {
    const unsigned long long k = T.mt_key[h];
    if (k == MT_EMPTY) continue;
    const double v = T.mt_sum[h];
    atomicAdd(T.arrival2 + (unsigned)(k & 0xffffffffull), v * v);
    T.mt_key[h] = MT_EMPTY;
  }
}

// ------------------------------------------------------------------------------------------- host helpers
static int upload_raw(LumenScene* sc, const void* h, size_t bytes, void** out) {
  *out = nullptr;
  if (bytes == 0 || !h) return 0;
  void* p = nullptr;
  CK(cudaMalloc(&p, bytes));
  sc->allocs.push_back(p);
  CK(cudaMemcpy(p, h, bytes, cudaMemcpyHostToDevice));
  *out = p;
  return 0;
}
#define UPLOAD(field, host, count)                                                  \
  do {                                                                              \
    void* p_ = nullptr;                                                             \
    e |= upload_raw(sc, (host), (size_t)(count) * sizeof(*(host)), &p_);           \
    field = (decltype(field))p_;                                                    \
  } while (0)

static void value_roles(const LumenSceneDesc* d, std::vector<std::pair<int, int>>& out);
static int check_values(const std::vector<std::pair<int, int>>& roles, const int32_t* tab, int n_tab, const float* pool);

static int check_desc(const LumenSceneDesc* d) {
  if (!d || d->n_vol <= 0 || !d->vol_i || !d->vol_f || !d->kind_i || !d->leaf_f || !d->leaf_i || !d->prog_i ||
      !d->cls_medium || !d->row_of || !d->med_i || !d->tab || !d->pool || d->n_cls <= 0 || d->n_pool <= 0)
    return set_err(LUMEN_ERR_ARG, "scene_create: a required array is null or empty");
  if (d->n_node < 0 || d->n_item < 0 || (d->n_node > 0 && (!d->node_f || !d->node_i)) || (d->n_item > 0 && !d->items))
    return set_err(LUMEN_ERR_ARG, "scene_create: BVH nodes or items without their arrays");
  if (d->precision != LUMEN_PREC_FLOAT32 && d->precision != LUMEN_PREC_FLOAT64)
    return set_err(LUMEN_ERR_ARG, "scene_create: precision is LUMEN_PREC_FLOAT32 or LUMEN_PREC_FLOAT64");
  if (d->precision == LUMEN_PREC_FLOAT64 && (!d->vol_f64 || !d->leaf_f64 || (d->n_node > 0 && !d->node_f64) ||
                                             (d->n_plane > 0 && !d->plane_f64) || (d->n_tri > 0 && !d->mesh_tri64)))
    return set_err(LUMEN_ERR_ARG, "scene_create: a float64 scene without its float64 geometry arrays");
  if (d->n_group < 0 || (d->n_group > 0 && (!d->group_i || !d->group_r || (d->precision == LUMEN_PREC_FLOAT64 && !d->group_r64))))
    return set_err(LUMEN_ERR_ARG, "scene_create: frame groups without their tables");
  for (int g = 0; g < d->n_group; ++g) {
    const int32_t* gr = d->group_i + 4 * (size_t)g;
    if (gr[0] < 0 || gr[0] > d->n_vol || gr[1] < 0 || gr[2] < gr[1] || gr[2] > d->n_node || (g > 0 && gr[0] < gr[-4]))
      return set_err(LUMEN_ERR_ARG, "scene_create: a frame group out of range (groups in volume order)");
    int same = 1;
    for (int h = g - 1; h >= 0 && d->group_i[4 * (size_t)h] == gr[0]; --h) same++;
    if (same > LUMEN_MAX_GROUPS_PER_VOLUME) return set_err(LUMEN_ERR_SCENE, "scene_create: too many frame groups in a volume");
  }
  if (d->n_mesh < 0 || d->n_chunk < 0 || d->n_tri < 0 || (d->n_mesh > 0) != (d->n_chunk > 0) ||
      (d->n_chunk > 0 && (!d->mesh_tri || !d->mesh_chunk)))
    return set_err(LUMEN_ERR_ARG, "scene_create: meshes without their triangles or chunks");
  for (int c = 0; c < d->n_chunk; ++c) {
    const int32_t* cr = d->mesh_chunk + 4 * (size_t)c;
    if (cr[0] < 0 || cr[1] < 1 || cr[1] > LUMEN_MESH_CHUNK || cr[0] + cr[1] > d->n_tri || cr[2] < 0 || cr[2] >= d->n_mesh)
      return set_err(LUMEN_ERR_ARG, "scene_create: a mesh chunk out of range");
  }
  for (int k = 0; k < d->n_kind; ++k) {
    int nl = d->kind_i[k * LUMEN_KIND_I + 1];
    if (nl < 1 || nl > LUMEN_MAX_LEAVES) return set_err(LUMEN_ERR_SCENE, "scene_create: a solid has too many leaves");
  }
  for (int g = 0; g < d->n_leaf; ++g)
    if (d->leaf_i[g * LUMEN_LEAF_I + 2] > LUMEN_MAX_PLANES)
      return set_err(LUMEN_ERR_SCENE, "scene_create: a leaf has too many planes");
  for (int t = 0; t < d->n_tab; ++t) {
    int off = d->tab[2 * t], k = d->tab[2 * t + 1];
    if (k < 1 || off < 0 || off + 2 * k > d->n_pool) return set_err(LUMEN_ERR_ARG, "scene_create: a table is out of the pool");
  }
  for (int m = 0; m < d->n_med; ++m) {  // every medium's tables in range; a Mie or WLS channel with its constants
    const int32_t* mr = d->med_i + (size_t)m * LUMEN_MED_I;
    for (int f = 0; f <= LUMEN_MI_WLS_SPEC; ++f)
      if (mr[f] < -1 || mr[f] >= d->n_tab) return set_err(LUMEN_ERR_ARG, "scene_create: a medium table is out of range");
    if (mr[LUMEN_MI_MIE] >= 0 && (mr[LUMEN_MI_MIE_GF] < 0 || mr[LUMEN_MI_MIE_GB] < 0 || mr[LUMEN_MI_MIE_R] < 0))
      return set_err(LUMEN_ERR_ARG, "scene_create: a Mie channel without its lobe constants");
    if (mr[LUMEN_MI_WLS] >= 0 && (mr[LUMEN_MI_WLS_YIELD] < 0 || mr[LUMEN_MI_WLS_TAU] < 0 || mr[LUMEN_MI_WLS_SPEC] < 0 ||
                                  d->tab[2 * mr[LUMEN_MI_WLS_SPEC] + 1] < 2 ||
                                  (mr[LUMEN_MI_WLS_PROFILE] != 0 && mr[LUMEN_MI_WLS_PROFILE] != 1)))
      return set_err(LUMEN_ERR_ARG, "scene_create: a WLS channel without its yield, time constant, spectrum (>= 2 "
                                    "knots) or profile (0 delta, 1 exponential)");
  }
  for (int m = 0; m < d->n_med; ++m) {
    int ti = d->med_i[m * LUMEN_MED_I + LUMEN_MI_INDEX];
    if (ti >= 0 && d->tab[2 * ti + 1] > LUMEN_MAX_KNOTS) return set_err(LUMEN_ERR_SCENE, "scene_create: an index table has too many knots");
  }
  for (int v = 0; v <= d->n_vol; ++v) {
    const int32_t* vi = d->vol_i + (size_t)v * LUMEN_VOL_I;
    if (vi[LUMEN_VI_SENSOR] >= d->n_sensor) return set_err(LUMEN_ERR_ARG, "scene_create: a sensor index is out of range");
    if (vi[LUMEN_VI_CLS] < 0 || vi[LUMEN_VI_CLS] >= d->n_cls) return set_err(LUMEN_ERR_ARG, "scene_create: a class is out of range");
    if (v < d->n_vol && (vi[LUMEN_VI_KIND] < 0 || vi[LUMEN_VI_KIND] >= d->n_kind)) return set_err(LUMEN_ERR_ARG, "scene_create: a kind is out of range");
    if (vi[LUMEN_VI_NODE0] < 0 || vi[LUMEN_VI_NODE1] > d->n_node || vi[LUMEN_VI_NODE0] > vi[LUMEN_VI_NODE1]) return set_err(LUMEN_ERR_ARG, "scene_create: a BVH range is out of range");
  }
  for (int v = 0; v <= d->n_vol; ++v) {  /* every daughter BVH within the traversal's stack */
    int n0 = d->vol_i[(size_t)v * LUMEN_VOL_I + LUMEN_VI_NODE0], n1 = d->vol_i[(size_t)v * LUMEN_VOL_I + LUMEN_VI_NODE1];
    if (n0 >= n1) continue;
    std::vector<std::pair<int, int>> todo{{n0, 1}};
    while (!todo.empty()) {
      auto [nd, dp] = todo.back();
      todo.pop_back();
      if (nd < n0 || nd >= n1 || dp > LUMEN_MAX_BVH_DEPTH) return set_err(LUMEN_ERR_SCENE, "scene_create: a BVH is malformed or deeper than LUMEN_MAX_BVH_DEPTH");
      if (d->node_i[(size_t)nd * LUMEN_NODE_I + 1] < 0) return set_err(LUMEN_ERR_SCENE, "scene_create: a BVH node with a negative count");
      if (d->node_i[(size_t)nd * LUMEN_NODE_I + 1] == 0) {
        todo.push_back({nd + 1, dp + 1});
        todo.push_back({d->node_i[(size_t)(nd + 1) * LUMEN_NODE_I], dp + 1});
      } else {
        int st = d->node_i[(size_t)nd * LUMEN_NODE_I + 2], cnt = d->node_i[(size_t)nd * LUMEN_NODE_I + 1];
        if (st < 0 || st + cnt > d->n_item) return set_err(LUMEN_ERR_SCENE, "scene_create: a BVH leaf is out of the items");
      }
    }
  }
  {  // every BVH item a volume or a mesh chunk (CH0 + c), every candidate one of the navigator's ids
    const int ch0 = d->n_vol + 1 + d->n_mesh;
    for (int i = 0; i < d->n_item; ++i) {
      const int it = d->items[i];
      if (!((it >= 0 && it < d->n_vol) || (it >= ch0 && it < ch0 + d->n_chunk)))
        return set_err(LUMEN_ERR_ARG, "scene_create: a BVH item is neither a volume nor a mesh chunk");
    }
    for (int i = 0; i < d->n_cand; ++i)
      if (d->cand[i] < 0 || d->cand[i] >= ch0 + d->n_chunk)
        return set_err(LUMEN_ERR_ARG, "scene_create: a candidate is not a volume, a mesh or a mesh chunk");
  }
  for (int c = 0; c < d->n_cls; ++c)
    if (d->cls_medium[c] < 0 || d->cls_medium[c] >= d->n_med) return set_err(LUMEN_ERR_ARG, "scene_create: a medium is out of range");
  if (d->cls_born)
    for (int c = 0; c < d->n_cls; ++c)
      if (d->cls_born[c] < -1 || d->cls_born[c] >= d->n_cls)
        return set_err(LUMEN_ERR_ARG, "scene_create: cls_born names a class out of range");
  if (d->pair_pre)
    for (long long k = 0; k < (long long)d->n_cls * d->n_cls; ++k)
      if (d->pair_pre[k] != 0 && d->pair_pre[k] != 1) return set_err(LUMEN_ERR_ARG, "scene_create: pair_pre is 0 or 1");
  for (int r = 0; r < d->n_row; ++r) {
    const int32_t* ri = d->row_i + r * LUMEN_ROW_I;
    for (int c = 0; c < LUMEN_N_COL; ++c)
      if (ri[LUMEN_RI_COL + c] < 0 || ri[LUMEN_RI_COL + c] >= d->n_tab) return set_err(LUMEN_ERR_ARG, "scene_create: a column table is out of range");
    if (ri[LUMEN_RI_GLISUR] < 0 || ri[LUMEN_RI_GLISUR] > 2)
      return set_err(LUMEN_ERR_ARG, "scene_create: a row's glisur flag is not 0 (unified), 1 (GLISUR metal) or 2 "
                                    "(GLISUR dielectric)");
    if (ri[LUMEN_RI_MODEL] == 0 && !ri[LUMEN_RI_NORMAL] && !ri[LUMEN_RI_GLISUR] && !d->unified)
      return set_err(LUMEN_ERR_ARG, "scene_create: a unified facet row needs the unified tables (desc->unified)");
  }
  if (d->n_jump > 0) {  // the diffusion jump's grids: a medium each, nodes inside the clearance array
    if (!d->jump_f || !d->jump_i || !d->clear || d->n_clear <= 0)
      return set_err(LUMEN_ERR_ARG, "scene_create: inconsistent diffusion jump arrays");
    for (int g = 0; g < d->n_jump; ++g) {
      const int32_t* ji = d->jump_i + (size_t)g * LUMEN_JUMP_I;
      int64_t nn = (int64_t)ji[1] * ji[2] * ji[3];
      if (ji[0] < 0 || ji[0] >= d->n_med || ji[1] < 1 || ji[2] < 1 || ji[3] < 1 || ji[4] < 0 || ji[4] + nn > d->n_clear ||
          !(d->jump_f[(size_t)g * LUMEN_JUMP_F + 3] > 0.0f))
        return set_err(LUMEN_ERR_ARG, "scene_create: a diffusion jump grid is out of range");
    }
  }
  if (d->comp) {  // the sensor reach arrays
    if (!d->comp_box || d->n_comp <= 0 || d->n_fnode < 0 || (d->n_fnode > 0 && (!d->fnode_f || !d->fnode_i)))
      return set_err(LUMEN_ERR_ARG, "scene_create: inconsistent sensor reach arrays");
    for (int v = 0; v <= d->n_vol; ++v)
      if (d->comp[v] < -1 || d->comp[v] >= d->n_comp) return set_err(LUMEN_ERR_ARG, "scene_create: a component is out of range");
    for (int k = 0; k < d->n_fnode; ++k) {
      int sk = d->fnode_i[(size_t)k * LUMEN_NODE_I];
      if (sk <= k || sk > d->n_fnode) return set_err(LUMEN_ERR_ARG, "scene_create: a sensor-box tree skip is out of order");
    }
  }
  std::vector<std::pair<int, int>> roles;  // the values of every table a run reads, inside their ranges
  value_roles(d, roles);
  return check_values(roles, d->tab, d->n_tab, d->pool);
}

// sigma_alpha of every unified facet row within the tables' span (src/lumen/rules/choices.py:103 SIGMA_MIN/MAX)
// The admissible values of the tables a run reads, by their role (src/lumen/_core/domains.py: a range with both ends
// included, never a value that is not finite; src/lumen/build/values.py:235 _check_params refuses a concrete value
// outside it): the knots of every such table strictly ascending and finite, its values inside the role's range.
enum { DOM_FRACTION = 0, DOM_POSITIVE, DOM_INDEX, DOM_MIE_G };
static void value_roles(const LumenSceneDesc* d, std::vector<std::pair<int, int>>& out) {
  out.clear();
  static const int med_role[][2] = {{LUMEN_MI_INDEX, DOM_INDEX}, {LUMEN_MI_ABS, DOM_POSITIVE}, {LUMEN_MI_RAY, DOM_POSITIVE},
                                    {LUMEN_MI_MIE, DOM_POSITIVE}, {LUMEN_MI_MIE_GF, DOM_MIE_G}, {LUMEN_MI_MIE_GB, DOM_MIE_G},
                                    {LUMEN_MI_MIE_R, DOM_FRACTION}, {LUMEN_MI_WLS, DOM_POSITIVE},
                                    {LUMEN_MI_WLS_YIELD, DOM_POSITIVE}, {LUMEN_MI_WLS_TAU, DOM_POSITIVE},
                                    {LUMEN_MI_WLS_SPEC, DOM_POSITIVE}};  // fmt: skip
  for (int m = 0; m < d->n_med; ++m)
    for (const auto& mr : med_role) {
      const int t = d->med_i[(size_t)m * LUMEN_MED_I + mr[0]];
      if (t >= 0) out.push_back({t, mr[1]});
    }
  static const int col_role[LUMEN_N_COL] = {DOM_FRACTION, DOM_FRACTION, DOM_FRACTION, DOM_FRACTION, DOM_FRACTION,
                                            DOM_FRACTION, DOM_POSITIVE, DOM_FRACTION, DOM_INDEX, DOM_POSITIVE};
  for (int r = 0; r < d->n_row; ++r)
    for (int c = 0; c < LUMEN_N_COL; ++c) {
      const int t = d->row_i[(size_t)r * LUMEN_ROW_I + LUMEN_RI_COL + c];
      if (t >= 0) out.push_back({t, col_role[c]});
    }
}

static int check_values(const std::vector<std::pair<int, int>>& roles, const int32_t* tab, int n_tab, const float* pool) {
  static const char* what[] = {"a fraction outside [0, 1]", "a negative length, yield, time or intensity",
                               "a refractive index below 1", "a Mie asymmetry |g| above 0.999"};
  for (const auto& tr : roles) {
    const int t = tr.first;
    if (t < 0 || t >= n_tab) continue;  // the table index itself is checked with the arrays
    const int off = tab[2 * t], k = tab[2 * t + 1];
    for (int j = 0; j < k; ++j) {
      const float e = pool[off + j], v = pool[off + k + j];
      if (!std::isfinite(e) || (j > 0 && !(e > pool[off + j - 1])))
        return set_err(LUMEN_ERR_ARG, "table " + std::to_string(t) + ": its knot energies must be finite and strictly "
                                      "ascending");
      bool ok = std::isfinite(v);
      switch (tr.second) {
        case DOM_FRACTION: ok = ok && v >= 0.0f && v <= 1.0f; break;
        case DOM_POSITIVE: ok = ok && v >= 0.0f; break;
        case DOM_INDEX: ok = ok && v >= 1.0f; break;
        default: ok = ok && fabsf(v) <= 0.999f; break;
      }
      if (!ok)
        return set_err(LUMEN_ERR_ARG, "table " + std::to_string(t) + " holds " + what[tr.second] +
                                          " or a value that is not finite (" + std::to_string(v) + ")");
    }
  }
  return 0;
}

static int check_widths(const LumenScene* sc, const float* pool) {
  const double lo = exp(LUMEN_UNI_Y0 + LUMEN_UNI_DY * LUMEN_UNI_J_LO);
  const double hi = exp(LUMEN_UNI_Y0 + LUMEN_UNI_DY * (LUMEN_UNI_J_LO + LUMEN_UNI_NY - 1));
  for (int t : sc->sigma_tabs) {
    int off = sc->tab[2 * t], k = sc->tab[2 * t + 1];
    for (int j = off + k; j < off + 2 * k; ++j)
      if (!(pool[j] >= (float)lo * 0.9999f && pool[j] <= (float)hi * 1.0001f))
        return set_err(LUMEN_ERR_ARG, "a unified facet row's sigma_alpha is outside [0.00276, 1] rad");
  }
  return 0;
}

static int fill_run(const LumenScene* sc, const LumenControls* c, Run& R) {
  if (!c) return set_err(LUMEN_ERR_ARG, "controls is null");
  if (!(c->roulette > 0.0f)) return set_err(LUMEN_ERR_ARG, "the roulette's epsilon must be > 0");
  if (c->n_grad < 0 || c->n_grad > LUMEN_MAX_GRAD) return set_err(LUMEN_ERR_NOT_SUPPORTED, "too many gradient parameters");
  if (c->max_vertices < 1) return set_err(LUMEN_ERR_ARG, "max_vertices must be >= 1");
  if (c->variant < 0 || c->variant >= LUMEN_N_VARIANT) return set_err(LUMEN_ERR_ARG, "unknown launch variant");
  R.S = sc->S;
  R.live = sc->pool_live;
  R.ref = sc->pool_ref;
  R.shared = sc->pool_ref == sc->pool_live;
  R.reach = sc->S.reach;
  R.max_distance = c->max_distance > 0.0f ? c->max_distance : sc->S.reach;
  R.roulette = c->roulette;
  R.max_vertices = c->max_vertices;
  for (int p = 0; p < c->n_grad; ++p)
    for (int t : sc->spectrum_tabs)
      if (c->grad_tab[p] == t)
        return set_err(LUMEN_ERR_NOT_SUPPORTED, "a WLS emission spectrum as a gradient parameter is not built");
  R.P = c->n_grad;
  for (int p = 0; p < LUMEN_MAX_GRAD; ++p) R.gt[p] = p < c->n_grad ? c->grad_tab[p] : -1;
  R.reach_on = (c->flags & LUMEN_F_REACH) && sc->S.comp != nullptr;
  R.jump_on = (c->flags & LUMEN_F_JUMP) && sc->S.med_jump != nullptr;
  return 0;
}

static int fill_launch(const LumenScene* sc, const LumenRows* rows, const LumenSource* source, uint32_t k0,
                       uint32_t k1, int64_t first_id, int64_t n, const LumenControls* c, Launch& L, Pick& pk) {
  memset(&L, 0, sizeof(L));
  if (!sc) return set_err(LUMEN_ERR_ARG, "scene is null");
  if ((rows == nullptr) == (source == nullptr)) return set_err(LUMEN_ERR_ARG, "give exactly one of rows / source");
  if (n < 0 || first_id < 0 || first_id + n > 2147483647LL) return set_err(LUMEN_ERR_ARG, "photon ids must fit int32");
  int st = fill_run(sc, c, L.R);
  if (st) return st;
  if (rows) {
    if (!rows->x || !rows->y || !rows->z || !rows->dx || !rows->dy || !rows->dz || !rows->t || !rows->lam || !rows->w)
      return set_err(LUMEN_ERR_ARG, "rows: a required array is null");
    L.rows = *rows;
    L.use_rows = 1;
  } else {
    if (source->n_events < 1 || !source->ev_f || !source->ev_first || !source->ev_w)
      return set_err(LUMEN_ERR_ARG, "source: events are missing");
    if (source->kind < 0 || source->kind > LUMEN_SRC_SCINT_MATERIAL) return set_err(LUMEN_ERR_ARG, "source: unknown kind");
    if (source->kind == LUMEN_SRC_SCINT_MATERIAL) {
      const int32_t* m = source->mat;
      const int nt = (int)(sc->tab.size() / 2), nc = m[LUMEN_SM_N];
      auto ok = [&](int t) { return t >= 0 && t < nt; };
      int good = nc >= 1 && nc <= 3 && ok(m[LUMEN_SM_YIELD]);
      for (int i = 0; i < nc && good; ++i)
        good = ok(m[LUMEN_SM_SPEC + i]) && ok(m[LUMEN_SM_TAU + i]) && (!m[LUMEN_SM_RISES] || ok(m[LUMEN_SM_RISE + i]));
      for (int i = 0; i < 3 && good; ++i) good = m[LUMEN_SM_SHARE + i] == -1 || ok(m[LUMEN_SM_SHARE + i]);
      if (!good) return set_err(LUMEN_ERR_ARG, "source: a scintillation material's tables are incomplete");
      for (int p = 0; p < (c ? c->n_grad : 0); ++p)
        for (int w = LUMEN_SM_YIELD; w < LUMEN_SM_WORDS; ++w)
          if (m[w] >= 0 && c->grad_tab[p] == m[w])
            return set_err(LUMEN_ERR_NOT_SUPPORTED, "a scintillation source's own tables are not gradient parameters "
                                                    "of this engine");
    }
    if (source->kind == LUMEN_SRC_CHERENKOV) {
      if (source->rindex_tab < 0 || source->rindex_tab >= (int)(sc->tab.size() / 2))
        return set_err(LUMEN_ERR_ARG, "source: a Cherenkov segment needs its medium's RINDEX table");
      if (!(source->lam0 > 0.0f) || !(source->lam1 >= source->lam0))
        return set_err(LUMEN_ERR_ARG, "source: a Cherenkov segment's wavelengths span [lam0, lam1] nm, lam0 > 0");
      for (int p = 0; p < (c ? c->n_grad : 0); ++p)
        if (c->grad_tab[p] == source->rindex_tab)
          return set_err(LUMEN_ERR_NOT_SUPPORTED, "the index of a Cherenkov segment's medium moves its photons' "
                                                  "directions: a pathwise derivative, not a reweighting one");
    }
    L.src = *source;
  }
  L.key.k0 = k0;
  L.key.k1 = k1;
  L.first_id = first_id;
  L.n = n;
  L.step_budget = c->step_budget;
  pk.torus = sc->has_torus;
  pk.single = sc->single;
  pk.clip = sc->clip;
  pk.groups = sc->groups;
  pk.nav64 = sc->nav64;
  pk.born = sc->S.cls_born != nullptr;
  pk.vol_f32 = sc->vol_f32;
  pk.analog = (c->flags & LUMEN_F_TRUTH) != 0;
  if (pk.analog && (c->n_grad > 0 || !L.R.shared))
    return set_err(LUMEN_ERR_ARG, "truth rows decide each photon's fate at one set of values: no gradient parameters "
                                  "and no reference pool of its own");
  return 0;
}

template <int G>
static int launch_trace(const Launch& L, const Pick& pk, int variant, int bps, cudaStream_t stream) {
  if (pk.nav64) {  // the float64 navigator: shape 0, extended (with frame groups or not) or single-leaf geometry
    if constexpr (G == 0)
      if (L.truth) return pk.groups ? launch_shape<0, 256, 4, 3, 1, 1>(L, bps, stream, 0)
                                    : launch_shape<0, 256, 4, 1, 1, 1>(L, bps, stream, 0);  // fmt: skip
    if (pk.single) return launch_shape<G, 256, 4, 2, 0, 1>(L, bps, stream, 0);
    if (pk.groups) return launch_shape<G, 256, 4, 3, 0, 1>(L, bps, stream, 0);
    return launch_shape<G, 256, 4, 1, 0, 1>(L, bps, stream, 0);
  }
  if constexpr (G == 0) {
    if (L.truth)  // truth rows: the analog instantiation of shape 0
      return pk.groups ? launch_shape<0, 256, 4, 3, 1>(L, bps, stream, 0)
                       : (pk.torus ? launch_shape<0, 256, 4, 1, 1>(L, bps, stream, 0)
                                   : launch_shape<0, 256, 4, 0, 1>(L, bps, stream, 0));  // fmt: skip
  }
  if (pk.groups) return launch_shape<G, 256, 4, 3>(L, bps, stream, 0);  // frame groups: shape 0 whatever the variant
  if (pk.torus) return launch_shape<G, 256, 4, 1>(L, bps, stream, 0);  // tori: shape 0 whatever the variant
  if (pk.single) switch (variant) {  // single-leaf solids: the scan of one leaf, no postfix program
      case 1: return launch_shape<G, 128, 8, 2>(L, bps, stream, 0);
      case 2: return launch_shape<G, 256, 3, 2>(L, bps, stream, 0);
      default: return launch_shape<G, 256, 4, 2>(L, bps, stream, 0);
    }
  switch (variant) {
    case 1: return launch_shape<G, 128, 8, 0>(L, bps, stream, 0);
    case 2: return launch_shape<G, 256, 3, 0>(L, bps, stream, 0);
    default: return launch_shape<G, 256, 4, 0>(L, bps, stream, 0);
  }
}

// ------------------------------------------------------------------------------------ the readout groups
static int check_groups(int n_sensor, const LumenTallies* out) {
  if (out->n_groups < 0 || out->n_groups > LUMEN_MAX_GROUPS) return set_err(LUMEN_ERR_ARG, "groups: 0 .. LUMEN_MAX_GROUPS");
  if (!out->groups) return set_err(LUMEN_ERR_ARG, "groups: the array is null");
  if (!out->records || ((uintptr_t)out->records & 15) || out->rec_capacity <= 0 || out->rec_capacity > 2147483647LL)
    return set_err(LUMEN_ERR_ARG, "groups: records must be a 16-byte aligned scratch of 1 .. 2^31 - 1 records");
  for (int g = 0; g < out->n_groups; ++g) {
    const LumenGroup& G = out->groups[g];
    const std::string w = "group " + std::to_string(g) + ": ";
    if (G.n_axes < 0 || G.n_delay < 0 || G.n_axes + G.n_delay > LUMEN_MAX_AXES)
      return set_err(LUMEN_ERR_ARG, w + "at most LUMEN_MAX_AXES axes");
    for (int a = 0; a < G.n_axes + G.n_delay; ++a) {
      const LumenAxis& A = G.axes[a];
      if (A.feature < 0 || A.feature >= LUMEN_N_FEAT) return set_err(LUMEN_ERR_ARG, w + "unknown feature");
      if (A.n < 2 || !A.values) return set_err(LUMEN_ERR_ARG, w + "an axis needs two values or more");
    }
    if (G.n_sensors <= 0 || (!G.index && G.n_sensors != n_sensor))
      return set_err(LUMEN_ERR_ARG, w + "n_sensors: the group's sensors (every detector sensor without an index)");
    if (!G.charge || !G.charge2) return set_err(LUMEN_ERR_ARG, w + "charge and charge2 are required");
    if (G.nt < 0 || (G.nt > 0 && (!(G.dt > 0.0f) || !G.time || !G.over_q || !G.over_qt)))
      return set_err(LUMEN_ERR_ARG, w + "a timed grid needs dt > 0, time, over_q and over_qt");
    if (G.weighted && !G.weights) return set_err(LUMEN_ERR_ARG, w + "a weighted grid needs its weights");
  }
  return 0;
}

static int launch_bin(const Launch& L, const Pick& pk, const LumenTallies* out, cudaStream_t stream) {
  Bin B;
  memset(&B, 0, sizeof(B));
  for (int g = 0; g < out->n_groups; ++g) B.g[g] = out->groups[g];
  B.n_groups = out->n_groups;
  B.E = L.T.E;
  B.S_ = L.T.S_;
  B.rec = L.R.rec;
  B.n = L.R.rec_n;
  B.cap = L.R.rec_cap;
  B.pe2 = out->pe2;
  B.vol_f = pk.vol_f32;
  B.counts = out->counts;
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  k_bin<<<sms * 8, 256, 0, stream>>>(B);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

// the moment table's slots for n photons: n / 8 rounded up to a power of two, at least 2^16 (16 bytes a slot); the
// photons of the benchmark's LAr box hold about 0.03 sums each past their first four, the tank's none
static size_t moment_slots(int64_t n) {
  size_t want = (size_t)(n / 8), s = (size_t)1 << 16;
  while (s < want) s <<= 1;
  return s;
}

static int launch_moment_flush(const Tally& T, cudaStream_t stream) {
  int dev = 0, sms = 0;
  CK(cudaGetDevice(&dev));
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  k_moment_flush<<<sms * 8, 256, 0, stream>>>(T);
  CK(cudaGetLastError());
  ++lumen_launches();
  return 0;
}

static int check_cells(const Tally& T) {
  if ((unsigned long long)T.E * (unsigned long long)T.S_ >= (1ull << 32))
    return set_err(LUMEN_ERR_ARG, "tallies: events x sensors must stay below 2^32");
  return 0;
}

static int run_trace(Launch& L, Pick pk, const LumenTallies* out, const double* cot, int n_events_cot, double* grads,
                     cudaStream_t stream, int variant = 0, int bps = 0, int async = 0, int slots_log2 = 0,
                     int rounds = 0, float* rpp = nullptr) {
  Tally& T = L.T;
  T.E = out ? (out->n_events > 0 ? out->n_events : 1) : (n_events_cot > 0 ? n_events_cot : 1);
  T.S_ = L.R.S.n_sensor > 0 ? L.R.S.n_sensor : 1;
  T.P = L.R.P;
  T.cot = cot;
  if (pk.analog) {  // truth rows: the persistent loop writes each photon's analog record
    if (!out || !out->truth) return set_err(LUMEN_ERR_ARG, "LUMEN_F_TRUTH: tallies.truth (n records) is required");
    L.truth = out->truth;
    if (variant == LUMEN_VARIANT_WAVEFRONT) variant = 0;
  }
  if ((pk.nav64 || pk.clip) && variant == LUMEN_VARIANT_WAVEFRONT) variant = 0;  // the wavefront's slots hold float32 positions
  T.grads = grads;
  // scratch: the photon counter, the abort flag, the steps used, the wavefront's live slots and the record count (one
  // small allocation per call)
  const int groups = out && out->n_groups > 0;
  int st0 = 0;
  if (groups && (st0 = check_groups(L.R.S.n_sensor, out))) return st0;
  if ((st0 = check_cells(T))) return st0;
  unsigned long long* scratch = nullptr;
  CK(cudaMallocAsync((void**)&scratch, 5 * sizeof(unsigned long long), stream));
  CK(cudaMemsetAsync(scratch, 0, 5 * sizeof(unsigned long long), stream));
  L.next = scratch;
  L.abort_flag = (int*)(scratch + 1);
  L.steps_used = scratch + 2;
  if (groups) {
    L.R.rec = (uint32_t*)out->records;
    L.R.rec_cap = out->rec_capacity;
    L.R.rec_n = scratch + 4;
  }
  // adjoint calls with no tallies of their own accumulate health and counts into the scratch's tail
  double* dummy = nullptr;
  if (!out) {
    CK(cudaMallocAsync((void**)&dummy, (LUMEN_N_HEALTH + LUMEN_N_COUNT + 4) * sizeof(double), stream));
    CK(cudaMemsetAsync(dummy, 0, (LUMEN_N_HEALTH + LUMEN_N_COUNT + 4) * sizeof(double), stream));
    T.nb = 0;
    T.arrival = T.arrival_t = T.arrival2 = nullptr;
  } else {
    T.nb = out->hist ? out->n_bins : 0;
    T.bin0 = out->bin0;
    T.bin_w = out->bin_w;
    T.arrival = out->arrival;
    T.arrival_t = out->arrival_t;
    T.arrival2 = out->arrival2;
    T.hist = out->hist;
    T.jac = out->jac;
    T.health = out->health;
    T.counts = out->counts;
  }
  // the moment table (the photons' sums past their first four sensors), every key free
  unsigned long long* mt = nullptr;
  if (T.arrival2 && L.n > 0) {
    const size_t slots = moment_slots(L.n);
    CK(cudaMallocAsync((void**)&mt, slots * 16, stream));
    CK(cudaMemsetAsync(mt, 0xff, slots * 8, stream));
    T.mt_key = mt;
    T.mt_sum = (double*)(mt + slots);
    T.mt_mask = (unsigned)(slots - 1);
  }
  int st = 0;
  // a point-like source's events: each located once, its photons starting in that volume (the locate each would
  // make; the float64 navigator's scenes locate per photon in float64)
  int32_t* ev_vol = nullptr;
  if (L.n > 0 && !L.use_rows && (L.src.kind == LUMEN_SRC_POINT || L.src.kind == LUMEN_SRC_SCINT) && !pk.nav64 &&
      L.src.n_events > 0) {
    CK(cudaMallocAsync((void**)&ev_vol, (size_t)L.src.n_events * sizeof(int32_t), stream));
    st = (pk.torus || pk.groups) ? launch_event_locate<1>(L.R.S, L.src, ev_vol, stream)
                                 : launch_event_locate<0>(L.R.S, L.src, ev_vol, stream);  // fmt: skip
    if (st) return st;
    L.ev_vol = ev_vol;
  }
  if (L.n > 0) {
    if (L.R.P > 0 || cot) {
      Launch L2 = L;
      if (!out) {  // an adjoint without tallies: the health and counts go to scratch (the arrivals are not written)
        L2.T.health = dummy;
        L2.T.counts = (unsigned long long*)(dummy + LUMEN_N_HEALTH);
      }
      st = variant == LUMEN_VARIANT_WAVEFRONT
               ? run_wave<LUMEN_MAX_GRAD>(L2, pk, scratch + 3, stream, slots_log2, async, rounds, rpp)
               : launch_trace<LUMEN_MAX_GRAD>(L2, pk, variant, bps, stream);
      if (st) return st;
    } else {
      st = variant == LUMEN_VARIANT_WAVEFRONT ? run_wave<0>(L, pk, scratch + 3, stream, slots_log2, async, rounds, rpp)
                                              : launch_trace<0>(L, pk, variant, bps, stream);
      if (st) return st;
    }
  }
  if (ev_vol) CK(cudaFreeAsync(ev_vol, stream));
  if (mt) {
    if ((st = launch_moment_flush(T, stream))) return st;
    CK(cudaFreeAsync(mt, stream));
  }
  if (groups && (st = launch_bin(L, pk, out, stream))) return st;
  if (async) {  // enqueue only: the abort flag reaches counts[LUMEN_C_ABORTED] on the device
    CK(cudaFreeAsync(scratch, stream));
    if (dummy) CK(cudaFreeAsync(dummy, stream));
    return 0;
  }
  int flag = 0;
  unsigned long long n_rec = 0;
  CK(cudaMemcpyAsync(&flag, L.abort_flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CK(cudaMemcpyAsync(&n_rec, scratch + 4, sizeof(n_rec), cudaMemcpyDeviceToHost, stream));
  CK(cudaFreeAsync(scratch, stream));
  if (dummy) CK(cudaFreeAsync(dummy, stream));
  CK(cudaStreamSynchronize(stream));
  if (flag) return set_err(LUMEN_ERR_STEP_BUDGET, "the call's step budget ran out before every photon ended");
  if (groups && n_rec > (unsigned long long)out->rec_capacity)
    return set_err(LUMEN_ERR_RECORDS, "the deposit records outgrew rec_capacity (" + std::to_string(n_rec) +
                                          " needed): the groups are not filled");
  return 0;
}

// ------------------------------------------------------------------------- the scratch that needs no allocation
// lumen_b200_trace_static's scratch: a fixed array in the library's device memory (one per GPU that loads the
// library, held until the process exits), for callers that cannot allocate during a call. Host code cannot use the
// array's name as an address (it names a host-side stand-in); each device's address is looked up once, with that
// device current, by cudaGetSymbolAddress.
static __device__ __align__(256) unsigned long long g_static_scratch[LUMEN_STATIC_SCRATCH_WORDS];
// its moment table: keys, then sums (LUMEN_STATIC_MOMENT_SLOTS each, 16 bytes a slot)
static __device__ __align__(256) unsigned long long g_static_moment[2 * LUMEN_STATIC_MOMENT_SLOTS];
static const int STATIC_SCRATCH_NEED = 4;  // photon counter, abort flag, steps used, record count
static std::mutex g_static_mu;
static void* g_static_addr[256][2];

static int static_scratch(unsigned long long** out, unsigned long long** moment) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return set_err(LUMEN_ERR_NO_DEVICE, "trace_static: device index out of range");
  std::lock_guard<std::mutex> lock(g_static_mu);
  if (!g_static_addr[dev][0]) {
    void *p = nullptr, *m = nullptr;
    CK(cudaGetSymbolAddress(&p, g_static_scratch));
    CK(cudaGetSymbolAddress(&m, g_static_moment));
    g_static_addr[dev][0] = p;
    g_static_addr[dev][1] = m;
  }
  *out = (unsigned long long*)g_static_addr[dev][0];
  *moment = (unsigned long long*)g_static_addr[dev][1];
  return 0;
}

// run_trace with the scratch and moment table of the fixed arrays (no allocation, no free); variant and bps as in
// run_trace (the wavefront, whose slot pool is an allocation, runs as the persistent shape 0); async: enqueue only
static int run_trace_static(Launch& L, Pick pk, const LumenTallies* out, cudaStream_t stream, int variant, int bps,
                            int async) {
  if (STATIC_SCRATCH_NEED > LUMEN_STATIC_SCRATCH_WORDS)
    return set_err(LUMEN_ERR_ARG, "trace_static: the call needs more scratch than LUMEN_STATIC_SCRATCH_WORDS");
  if (variant == LUMEN_VARIANT_WAVEFRONT) variant = 0;
  unsigned long long *scratch = nullptr, *moment = nullptr;
  int st = static_scratch(&scratch, &moment);
  if (st) return st;
  Tally& T = L.T;
  T.E = out->n_events > 0 ? out->n_events : 1;
  T.S_ = L.R.S.n_sensor > 0 ? L.R.S.n_sensor : 1;
  T.P = L.R.P;
  T.cot = nullptr;
  if (pk.analog) {
    if (!out->truth) return set_err(LUMEN_ERR_ARG, "LUMEN_F_TRUTH: tallies.truth (n records) is required");
    L.truth = out->truth;
  }
  T.grads = nullptr;
  T.nb = out->hist ? out->n_bins : 0;
  T.bin0 = out->bin0;
  T.bin_w = out->bin_w;
  T.arrival = out->arrival;
  T.arrival_t = out->arrival_t;
  T.arrival2 = out->arrival2;
  T.hist = out->hist;
  T.jac = out->jac;
  T.health = out->health;
  T.counts = out->counts;
  const int groups = out->n_groups > 0;
  if (groups && (st = check_groups(L.R.S.n_sensor, out))) return st;
  if ((st = check_cells(T))) return st;
  // the arrays keep the previous call's contents: clear the words this call reads before they are written, and free
  // every slot of the moment table
  CK(cudaMemsetAsync(scratch, 0, STATIC_SCRATCH_NEED * sizeof(unsigned long long), stream));
  CK(cudaMemsetAsync(moment, 0xff, LUMEN_STATIC_MOMENT_SLOTS * sizeof(unsigned long long), stream));
  T.mt_key = moment;
  T.mt_sum = (double*)(moment + LUMEN_STATIC_MOMENT_SLOTS);
  T.mt_mask = LUMEN_STATIC_MOMENT_SLOTS - 1;
  L.next = scratch;
  L.abort_flag = (int*)(scratch + 1);
  L.steps_used = scratch + 2;
  if (groups) {
    L.R.rec = (uint32_t*)out->records;
    L.R.rec_cap = out->rec_capacity;
    L.R.rec_n = scratch + 3;
  }
  if (L.n > 0) {
    if (L.R.P > 0) st = launch_trace<LUMEN_MAX_GRAD>(L, pk, variant, bps, stream);
    else st = launch_trace<0>(L, pk, variant, bps, stream);
    if (st) return st;
    if ((st = launch_moment_flush(T, stream))) return st;
  }
  if (groups && (st = launch_bin(L, pk, out, stream))) return st;
  if (async) return 0;  // enqueue only: the abort flag reaches counts[LUMEN_C_ABORTED] on the device
  int flag = 0;
  unsigned long long n_rec = 0;
  CK(cudaMemcpyAsync(&flag, L.abort_flag, sizeof(int), cudaMemcpyDeviceToHost, stream));
  CK(cudaMemcpyAsync(&n_rec, scratch + 3, sizeof(n_rec), cudaMemcpyDeviceToHost, stream));
  CK(cudaStreamSynchronize(stream));
  if (flag) return set_err(LUMEN_ERR_STEP_BUDGET, "the call's step budget ran out before every photon ended");
  if (groups && n_rec > (unsigned long long)out->rec_capacity)
    return set_err(LUMEN_ERR_RECORDS, "the deposit records outgrew rec_capacity (" + std::to_string(n_rec) +
                                          " needed): the groups are not filled");
  return 0;
}

// ------------------------------------------------------------------------------------------------- the ABI
extern "C" {

int32_t lumen_b200_trace_static(const LumenScene* sc, const LumenRows* rows, const LumenSource* source, uint32_t key0,
                                uint32_t key1, int64_t first_id, int64_t n, const LumenControls* c, LumenTallies* out,
                                void* stream) {
  begin_call();
  if (!out || !out->arrival || !out->arrival_t || !out->arrival2 || !out->health || !out->counts)
    return set_err(LUMEN_ERR_ARG, "tallies: a required output is null");
  if (c && c->n_grad > 0 && !out->jac) return set_err(LUMEN_ERR_ARG, "tallies: jac is null with gradient parameters");
  if (out->hist && (out->n_bins <= 0 || !(out->bin_w > 0.0f))) return set_err(LUMEN_ERR_ARG, "tallies: bad histogram");
  if (source && out->n_events < source->n_events) return set_err(LUMEN_ERR_ARG, "tallies: fewer events than the source's");
  Launch L;
  Pick pk;
  int st = fill_launch(sc, rows, source, key0, key1, first_id, n, c, L, pk);
  if (st) return st;
  return run_trace_static(L, pk, out, (cudaStream_t)stream, c ? c->variant : 0, c ? c->blocks_per_sm : 0,
                          c ? (c->flags & LUMEN_F_ASYNC) != 0 : 0);
}

int32_t lumen_b200_abi_version(void) { return LUMEN_B200_ABI_VERSION; }

const char* lumen_b200_last_error(void) { return g_err.c_str(); }

int64_t lumen_b200_last_launches(void) { return lumen_launches(); }

int32_t lumen_b200_scene_create(const LumenSceneDesc* d, LumenScene** out) {
  begin_call();
  if (!out) return set_err(LUMEN_ERR_ARG, "out is null");
  *out = nullptr;
  int st = check_desc(d);
  if (st) return st;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return set_err(LUMEN_ERR_NO_DEVICE, "no CUDA device");
  LumenScene* sc = new LumenScene();
  CK(cudaGetDevice(&sc->dev));
  {  // the calls' scratch and moment tables come from the device's default pool (cudaMallocAsync): the pool keeps
     // what it has once held in this process, so a later call reuses it without mapping memory again
    cudaMemPool_t pool;
    CK(cudaDeviceGetDefaultMemPool(&pool, sc->dev));
    uint64_t keep = UINT64_MAX;
    CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
  }
  DScene& S = sc->S;
  S.n = d->n_vol;
  S.LM = 1;
  S.FM = 1;
  for (int k = 0; k < d->n_kind; ++k) {
    int l0 = d->kind_i[k * LUMEN_KIND_I], nl = d->kind_i[k * LUMEN_KIND_I + 1];
    if (nl > S.LM) S.LM = nl;
    for (int l = 0; l < nl; ++l) {
      int np_ = d->leaf_i[(l0 + l) * LUMEN_LEAF_I + 2];
      if (np_ + 1 > S.FM) S.FM = np_ + 1;
    }
  }
  const int ch0 = d->n_vol + 1 + d->n_mesh;  // the first mesh chunk's id; plain items end after the chunks
  S.SU = ch0 + d->n_chunk;
  S.n_cls = d->n_cls;
  S.n_sensor = d->n_sensor;
  S.reach = d->reach;
  int e = 0;
  UPLOAD(S.vol_i, d->vol_i, (size_t)(ch0 + d->n_chunk) * LUMEN_VOL_I);
  UPLOAD(S.vol_f, d->vol_f, (size_t)d->n_vol * LUMEN_VOL_F);
  S.mesh = nullptr;  // the candidate lists are the checker's: the engine walks the BVH
  if (d->n_mesh > 0 || d->n_group > 0) {  // the extended block: header, chunks, each triangle's chunk, frame groups
    const long long sm = (long long)S.SU + (long long)d->n_vol * S.LM * S.FM * 4;
    if (sm + 4LL * d->n_tri >= (1LL << 31)) {
      for (void* p : sc->allocs) cudaFree(p);
      delete sc;
      return set_err(LUMEN_ERR_SCENE, "scene_create: the surface codes of the volumes and mesh triangles exceed int32");
    }
    const size_t gto = 8 + 4 * (size_t)d->n_chunk + d->n_tri;  // the frame groups' table
    std::vector<int32_t> blk(gto + 2 * (size_t)(d->n_vol + 1) + 2 * (size_t)d->n_group, 0);
    blk[0] = d->n_mesh; blk[1] = d->n_chunk; blk[2] = d->n_tri; blk[3] = d->n_leaf * LUMEN_LEAF_F;
    blk[4] = (int32_t)sm; blk[5] = ch0;
    blk[6] = d->n_leaf * LUMEN_LEAF_F + d->n_tri * LUMEN_TRI_F;  // the groups' frames in the leaf array
    blk[7] = d->n_group > 0 ? (int32_t)gto : 0;
    for (int g = 0; g < d->n_group; ++g) {  // per volume its first group and count; per group its node range
      int v = d->group_i[4 * g];
      if (blk[gto + 2 * v + 1] == 0) blk[gto + 2 * v] = g;
      blk[gto + 2 * v + 1] += 1;
      blk[gto + 2 * (size_t)(d->n_vol + 1) + 2 * g] = d->group_i[4 * g + 1];
      blk[gto + 2 * (size_t)(d->n_vol + 1) + 2 * g + 1] = d->group_i[4 * g + 2];
    }
    for (int c = 0; c < d->n_chunk; ++c) {
      for (int j = 0; j < 4; ++j) blk[8 + 4 * c + j] = d->mesh_chunk[4 * c + j];
      for (int k = 0; k < d->mesh_chunk[4 * c + 1]; ++k) blk[8 + 4 * (size_t)d->n_chunk + d->mesh_chunk[4 * c] + k] = c;
    }
    UPLOAD(S.mesh, blk.data(), blk.size());
  }
  UPLOAD(S.node_f, d->node_f, (size_t)d->n_node * LUMEN_NODE_F);
  UPLOAD(S.node_i, d->node_i, (size_t)d->n_node * LUMEN_NODE_I);
  UPLOAD(S.items, d->items, (size_t)d->n_item);
  {  // the float32 ray traversal's node records (DScene::node_w) and the leaves' item lists
    const int nn = d->n_node;
    std::vector<int32_t> code((size_t)(nn > 0 ? nn : 1), -1), witem;
    for (int n = 0; n < nn; ++n) {
      const int32_t* ni = d->node_i + (size_t)n * LUMEN_NODE_I;
      if (ni[1] > 0 && (ni[2] < 0 || ni[2] + ni[1] > d->n_item)) {
        code[n] = -1;  // outside every BVH the checks above walked: never reached
      } else if (ni[1] > 0) {
        code[n] = -2 - (int32_t)witem.size();
        for (int k = 0; k < ni[1]; ++k) witem.push_back(d->items[ni[2] + k]);
        witem.push_back(-1);
      } else {
        code[n] = n;
      }
    }
    // a record without children (a leaf's, or a node outside every BVH) has NaN boxes, which no slab test meets
    // (every comparison with NaN is false), and codes -1
    std::vector<float> rec((size_t)(nn > 0 ? nn : 1) * 16, std::numeric_limits<float>::quiet_NaN());
    for (int n = 0; n < nn; ++n) {
      float* r = rec.data() + (size_t)n * 16;
      const int32_t none = -1, zero = 0;
      memcpy(r + 12, &none, 4);
      memcpy(r + 13, &none, 4);
      memcpy(r + 15, &zero, 4);
      const int lc = n + 1, rc = lc < nn ? d->node_i[(size_t)lc * LUMEN_NODE_I] : -1;
      if (d->node_i[(size_t)n * LUMEN_NODE_I + 1] == 0 && lc < nn && rc >= 0 && rc < nn) {
        std::copy(d->node_f + (size_t)lc * LUMEN_NODE_F, d->node_f + (size_t)lc * LUMEN_NODE_F + 6, r);
        std::copy(d->node_f + (size_t)rc * LUMEN_NODE_F, d->node_f + (size_t)rc * LUMEN_NODE_F + 6, r + 6);
        memcpy(r + 12, &code[lc], 4);
        memcpy(r + 13, &code[rc], 4);
      }
      memcpy(r + 14, &code[n], 4);
    }
    if (nn > 0) {
      UPLOAD(S.node_w, reinterpret_cast<const float4*>(rec.data()), (size_t)nn * 4);
      UPLOAD(S.witem, witem.data(), witem.size());
    } else {
      S.node_w = nullptr;
      S.witem = nullptr;
    }
  }
  UPLOAD(S.kind_i, d->kind_i, (size_t)d->n_kind * LUMEN_KIND_I);
  if (d->n_tri > 0 || d->n_group > 0) {  // the triangles and the groups' frames after the leaves (one allocation)
    const size_t nl = (size_t)d->n_leaf * LUMEN_LEAF_F, nt = (size_t)d->n_tri * LUMEN_TRI_F;
    std::vector<float> lt(nl + nt + 9 * (size_t)d->n_group);
    std::copy(d->leaf_f, d->leaf_f + nl, lt.begin());
    if (nt) std::copy(d->mesh_tri, d->mesh_tri + nt, lt.begin() + nl);
    if (d->n_group) std::copy(d->group_r, d->group_r + 9 * (size_t)d->n_group, lt.begin() + nl + nt);
    UPLOAD(S.leaf_f, lt.data(), lt.size());
  } else {
    UPLOAD(S.leaf_f, d->leaf_f, (size_t)d->n_leaf * LUMEN_LEAF_F);
  }
  UPLOAD(S.leaf_i, d->leaf_i, (size_t)d->n_leaf * LUMEN_LEAF_I);
  UPLOAD(S.plane_f, d->plane_f, (size_t)d->n_plane * LUMEN_PLANE_F);
  UPLOAD(S.prog_i, d->prog_i, (size_t)d->n_prog * LUMEN_PROG_I);
  sc->nav64 = d->precision == LUMEN_PREC_FLOAT64;
  sc->vol_f32 = S.vol_f;
  if (sc->nav64) {  // the float64 navigator reads its arrays through the same pointers (checked non-null above)
    const double *vd = nullptr, *nd = nullptr, *ld = nullptr, *pd = nullptr;
    UPLOAD(vd, d->vol_f64, (size_t)d->n_vol * LUMEN_VOL_F);
    UPLOAD(nd, d->node_f64, (size_t)d->n_node * LUMEN_NODE_F);
    const size_t nl = (size_t)d->n_leaf * LUMEN_LEAF_F, nt = (size_t)d->n_tri * LUMEN_TRI_F;
    std::vector<double> lt(nl + nt + 9 * (size_t)d->n_group);
    std::copy(d->leaf_f64, d->leaf_f64 + nl, lt.begin());
    if (nt) std::copy(d->mesh_tri64, d->mesh_tri64 + nt, lt.begin() + nl);
    if (d->n_group) std::copy(d->group_r64, d->group_r64 + 9 * (size_t)d->n_group, lt.begin() + nl + nt);
    UPLOAD(ld, lt.data(), lt.size());
    UPLOAD(pd, d->plane_f64, (size_t)d->n_plane * LUMEN_PLANE_F);
    S.vol_f = reinterpret_cast<const float*>(vd);
    S.node_f = reinterpret_cast<const float*>(nd);
    S.leaf_f = reinterpret_cast<const float*>(ld);
    S.plane_f = reinterpret_cast<const float*>(pd);
  }
  UPLOAD(S.cls_medium, d->cls_medium, (size_t)d->n_cls);
  if (d->cls_born) UPLOAD(S.cls_born, d->cls_born, (size_t)d->n_cls);
  if (d->pair_pre) UPLOAD(S.pair_pre, d->pair_pre, (size_t)d->n_cls * d->n_cls);
  UPLOAD(S.row_of, d->row_of, (size_t)d->n_cls * d->n_cls);
  UPLOAD(S.med_i, d->med_i, (size_t)d->n_med * LUMEN_MED_I);
  UPLOAD(S.row_i, d->row_i, (size_t)d->n_row * LUMEN_ROW_I);
  UPLOAD(S.tab, d->tab, (size_t)d->n_tab * 2);
  const float* pl = nullptr;
  UPLOAD(pl, d->pool, (size_t)d->n_pool);
  S.uni = nullptr;
  if (d->unified) UPLOAD(S.uni, d->unified, (size_t)LUMEN_UNI_WORDS);
  S.comp = nullptr;
  S.comp_box = S.fnode_f = nullptr;
  S.fnode_i = nullptr;
  S.n_fnode = 0;
  if (d->comp) {
    UPLOAD(S.comp, d->comp, (size_t)d->n_vol + 1);
    UPLOAD(S.comp_box, d->comp_box, (size_t)d->n_comp * 6);
    if (d->n_fnode > 0) {
      UPLOAD(S.fnode_f, d->fnode_f, (size_t)d->n_fnode * LUMEN_NODE_F);
      UPLOAD(S.fnode_i, d->fnode_i, (size_t)d->n_fnode * LUMEN_NODE_I);
    }
    S.n_fnode = d->n_fnode;
  }
  S.med_jump = nullptr;
  S.jump_f = nullptr;
  S.jump_i = nullptr;
  S.clear = nullptr;
  if (d->n_jump > 0) {  // the diffusion jump's grids, and each medium's grid index
    std::vector<int32_t> mj(d->n_med > 0 ? d->n_med : 1, -1);
    for (int g = 0; g < d->n_jump; ++g) mj[d->jump_i[(size_t)g * LUMEN_JUMP_I]] = g;
    UPLOAD(S.med_jump, mj.data(), mj.size());
    UPLOAD(S.jump_f, d->jump_f, (size_t)d->n_jump * LUMEN_JUMP_F);
    UPLOAD(S.jump_i, d->jump_i, (size_t)d->n_jump * LUMEN_JUMP_I);
    UPLOAD(S.clear, d->clear, (size_t)d->n_clear);
  }
  if (e) {
    for (void* p : sc->allocs) cudaFree(p);
    delete sc;
    return LUMEN_ERR_CUDA;
  }
  for (int r = 0; r < d->n_row; ++r) {
    const int32_t* ri = d->row_i + r * LUMEN_ROW_I;
    if (ri[LUMEN_RI_MODEL] == 0 && !ri[LUMEN_RI_NORMAL] && !ri[LUMEN_RI_GLISUR])
      sc->sigma_tabs.push_back(ri[LUMEN_RI_COL + LUMEN_COL_SIGMA]);
  }
  sc->tab.assign(d->tab, d->tab + 2 * (size_t)d->n_tab);
  sc->has_torus = d->n_mesh > 0 || d->n_group > 0;  // the extended instantiation: tori, meshes, frame groups
  sc->clip = d->n_group > 0;  // the extended locate (frame groups, protrusion clips): no wavefront (its fill's locate)
  sc->groups = d->n_group > 0;
  for (int l = 0; l < d->n_leaf; ++l) sc->has_torus = sc->has_torus || d->leaf_i[(size_t)l * LUMEN_LEAF_I] == 2;
  for (int v = 0; v < d->n_vol && !sc->clip; ++v) {  // a protrusion clip: the extended instantiation
    const int32_t* vr = d->vol_i + (size_t)v * LUMEN_VOL_I;
    for (int k = 0; k < vr[LUMEN_VI_CN]; ++k) {
      int i = d->cand[vr[LUMEN_VI_C0] + k];
      if (i >= 0 && i < v && v < i + d->vol_i[(size_t)i * LUMEN_VOL_I + LUMEN_VI_SIZE]) sc->has_torus = sc->clip = 1;
    }
  }
  sc->single = !sc->has_torus;  // every kind one leaf (a quadric and / or planes) whose program is that leaf
  for (int k = 0; k < d->n_kind; ++k)
    sc->single = sc->single && d->kind_i[(size_t)k * LUMEN_KIND_I + 1] == 1 && d->kind_i[(size_t)k * LUMEN_KIND_I + 3] == 1;
  for (int m = 0; m < d->n_med; ++m) {
    const int32_t* mr = d->med_i + (size_t)m * LUMEN_MED_I;
    if (mr[LUMEN_MI_WLS] >= 0) sc->spectrum_tabs.push_back(mr[LUMEN_MI_WLS_SPEC]);
  }
  value_roles(d, sc->roles);
  if (check_widths(sc, d->pool)) {
    for (void* p : sc->allocs) cudaFree(p);
    delete sc;
    return LUMEN_ERR_ARG;
  }
  sc->pool_live = const_cast<float*>(pl);
  sc->pool_ref = sc->pool_live;
  sc->n_pool = d->n_pool;
  *out = sc;
  return 0;
}

int32_t lumen_b200_scene_set_pools(LumenScene* sc, const float* live, const float* ref) {
  begin_call();
  if (!sc || !live) return set_err(LUMEN_ERR_ARG, "scene or live pool is null");
  if (check_widths(sc, live) || (ref && check_widths(sc, ref))) return LUMEN_ERR_ARG;
  const int n_tab = (int)(sc->tab.size() / 2);
  int sv = check_values(sc->roles, sc->tab.data(), n_tab, live);
  if (!sv && ref) sv = check_values(sc->roles, sc->tab.data(), n_tab, ref);
  if (sv) return sv;
  CK(cudaMemcpy(sc->pool_live, live, sc->n_pool * sizeof(float), cudaMemcpyHostToDevice));
  if (ref && ref != live) {
    if (sc->pool_ref == sc->pool_live) {
      void* p = nullptr;
      CK(cudaMalloc(&p, sc->n_pool * sizeof(float)));
      sc->allocs.push_back(p);
      sc->pool_ref = (float*)p;
    }
    CK(cudaMemcpy(sc->pool_ref, ref, sc->n_pool * sizeof(float), cudaMemcpyHostToDevice));
  } else {
    sc->pool_ref = sc->pool_live;
  }
  return 0;
}

int32_t lumen_b200_scene_destroy(LumenScene* sc) {
  begin_call();
  if (!sc) return 0;
  for (void* p : sc->allocs) cudaFree(p);
  delete sc;
  return 0;
}

int32_t lumen_b200_trace(const LumenScene* sc, const LumenRows* rows, const LumenSource* source, uint32_t key0,
                         uint32_t key1, int64_t first_id, int64_t n, const LumenControls* c, LumenTallies* out,
                         void* stream) {
  begin_call();
  if (!out || !out->arrival || !out->arrival_t || !out->arrival2 || !out->health || !out->counts)
    return set_err(LUMEN_ERR_ARG, "tallies: a required output is null");
  if (c && c->n_grad > 0 && !out->jac) return set_err(LUMEN_ERR_ARG, "tallies: jac is null with gradient parameters");
  if (out->hist && (out->n_bins <= 0 || !(out->bin_w > 0.0f))) return set_err(LUMEN_ERR_ARG, "tallies: bad histogram");
  if (source && out->n_events < source->n_events) return set_err(LUMEN_ERR_ARG, "tallies: fewer events than the source's");
  Launch L;
  Pick pk;
  int st = fill_launch(sc, rows, source, key0, key1, first_id, n, c, L, pk);
  if (st) return st;
  return run_trace(L, pk, out, nullptr, 0, nullptr, (cudaStream_t)stream, c->variant, c->blocks_per_sm,
                   c->flags & LUMEN_F_ASYNC, c->wave_slots_log2, c->wave_rounds, &sc->wave_rpp);
}

int32_t lumen_b200_adjoint(const LumenScene* sc, const LumenRows* rows, const LumenSource* source, uint32_t key0,
                           uint32_t key1, int64_t first_id, int64_t n, const LumenControls* c,
                           const double* cotangent, int32_t n_events, double* grads, void* stream) {
  begin_call();
  if (!cotangent || !grads) return set_err(LUMEN_ERR_ARG, "adjoint: cotangent and grads are required");
  if (!c || c->n_grad <= 0) return set_err(LUMEN_ERR_ARG, "adjoint: no gradient parameters");
  Launch L;
  Pick pk;
  int st = fill_launch(sc, rows, source, key0, key1, first_id, n, c, L, pk);
  if (st) return st;
  if (pk.analog) return set_err(LUMEN_ERR_ARG, "the adjoint replays no truth rows");
  return run_trace(L, pk, nullptr, cotangent, n_events, grads, (cudaStream_t)stream, c->variant, c->blocks_per_sm,
                   c->flags & LUMEN_F_ASYNC, c->wave_slots_log2, c->wave_rounds, &sc->wave_rpp);
}

int32_t lumen_b200_trace_photons(const LumenScene* sc, const LumenRows* rows, const LumenSource* source,
                                 uint32_t key0, uint32_t key1, int64_t first_id, int64_t n,
                                 const LumenControls* c, int32_t* out_i, float* out_f, void* stream) {
  begin_call();
  if (!out_i || !out_f) return set_err(LUMEN_ERR_ARG, "trace_photons: outputs are null");
  Launch L;
  Pick pk;
  int st = fill_launch(sc, rows, source, key0, key1, first_id, n, c, L, pk);
  if (st) return st;
  if (n == 0) return 0;
  st = pk.nav64 ? launch_photons<1>(L, out_i, out_f, (cudaStream_t)stream)
               : launch_photons<0>(L, out_i, out_f, (cudaStream_t)stream);
  if (st) return st;
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  return 0;
}

int32_t lumen_b200_query(const LumenScene* sc, const float* ray, const int32_t* vol, const int32_t* srf, float t_max,
                         int64_t n, int32_t* out_i, float* out_f, void* stream) {
  begin_call();
  if (!sc || !ray || !vol || !srf || !out_i || !out_f) return set_err(LUMEN_ERR_ARG, "query: a pointer is null");
  if (sc->nav64) return set_err(LUMEN_ERR_ARG, "query: a float64 scene: use lumen_b200_query64");
  if (n == 0) return 0;
  int st = launch_query(sc->S, ray, vol, srf, t_max, n, out_i, out_f, (cudaStream_t)stream);
  if (st) return st;
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  return 0;
}

int32_t lumen_b200_locate(const LumenScene* sc, const float* pts, int64_t n, int32_t* vol, void* stream) {
  begin_call();
  if (!sc || !pts || !vol) return set_err(LUMEN_ERR_ARG, "locate: a pointer is null");
  if (sc->nav64) return set_err(LUMEN_ERR_ARG, "locate: a float64 scene: use lumen_b200_locate64");
  if (n == 0) return 0;
  int st = launch_locate(sc->S, pts, n, vol, (cudaStream_t)stream);
  if (st) return st;
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  return 0;
}

int32_t lumen_b200_query64(const LumenScene* sc, const double* ray, const int32_t* vol, const int32_t* srf,
                           double t_max, int64_t n, int32_t* out_i, double* out_f, void* stream) {
  begin_call();
  if (!sc || !ray || !vol || !srf || !out_i || !out_f) return set_err(LUMEN_ERR_ARG, "query64: a pointer is null");
  if (!sc->nav64) return set_err(LUMEN_ERR_ARG, "query64: a float32 scene: use lumen_b200_query");
  if (n == 0) return 0;
  int st = launch_query(sc->S, ray, vol, srf, t_max, n, out_i, out_f, (cudaStream_t)stream);
  if (st) return st;
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  return 0;
}

int32_t lumen_b200_locate64(const LumenScene* sc, const double* pts, int64_t n, int32_t* vol, void* stream) {
  begin_call();
  if (!sc || !pts || !vol) return set_err(LUMEN_ERR_ARG, "locate64: a pointer is null");
  if (!sc->nav64) return set_err(LUMEN_ERR_ARG, "locate64: a float32 scene: use lumen_b200_locate");
  if (n == 0) return 0;
  int st = launch_locate(sc->S, pts, n, vol, (cudaStream_t)stream);
  if (st) return st;
  CK(cudaStreamSynchronize((cudaStream_t)stream));
  return 0;
}

}  // extern "C"
