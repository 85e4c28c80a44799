// The navigator on the device: CSG leaf intervals, the postfix boolean, first_change, and Geant4 volume tracking
// with surface identity, over per-volume BVHs of the daughters' world boxes. The body (dnav.cuh) is compiled in both
// of the reference's precisions: nav32 (float32, the default) and nav64 (float64 navigator: the load option
// precision="float64", src/lumen/rules/navigation.py:96); nav_* below pick one by the position's type.
//
// Semantics follow src/lumen/geometry/csg.py (first_change :417, _nearest :369, _change :395, _mem_at :346,
// _program :320, _q_iv :138, _planes :116), leaf_kernels.py:81 (quad_line), navigate.py (_unit_visit :376,
// _on_face :334, enter :482, _next_volume :515, _settle :254, _round :557, _finish :617, query :663) and
// surface_id.py (srf codes, hit_grad, face_dist). The arithmetic of each function is operation for operation the
// CPU checker's, so ray queries agree bit for bit; the candidates are found by BVH traversal (stack of 32, nearer
// child first, pruned by the best event) instead of the checker's scan of every daughter.
#pragma once
#include "../../include/lumen_b200.h"
#include "dmath.cuh"

namespace lb {

#define D_HUGE 1e30f
#define D_BIG 1e29f
#define D_EPS32 1.1920928955078125e-7f
#define D_BAND_ULPS_EPS 9.5367431640625e-07f
#define D_BAND_FLOOR 1e-9f
#define D_K_ON 4.0f
#define D_RELOCATE_BANDS 0.25f
#define D_ZERO_STEP_BANDS 0.125f
#define D_PUSH_BANDS 8.0f
#define D_TANGENT_ULPS 16.0f
#define D_DIVISOR_FLOOR 1e-30f
#define D_TINY_DIR 1e-30f
#define D_LINEAR_REL 1e-12f
#define D_PARALLEL 1e-12f
#define D_GRAZE 256.0f
#define D_ZSBP 10
#define D_ZSBK 25
#define D_MAX_SCAN_PER_LEAF 4
#define D_MAX_SCAN_EXTRA 5
#define D_TINY_NORMAL 1.17549435e-38f
#define D_STACK LUMEN_MAX_BVH_DEPTH

// the scene on the device (the LumenSceneDesc arrays, device pointers)
struct DScene {
  int n, LM, FM, SU;
  int n_cls, n_sensor;
  float reach;
  const int32_t* __restrict__ vol_i;
  const float* __restrict__ vol_f;  // vol_f, node_f, leaf_f, plane_f: float64 data on a float64 scene (nav64)
  const int32_t* __restrict__ mesh;  // the meshes' block (dnav.cuh: header, chunks, triangle chunks), null: none
  const float* __restrict__ node_f;
  const int32_t* __restrict__ node_i;
  const int32_t* __restrict__ items;
  // the float32 ray traversal's node records, 16 words a node: an inner node's left and right child boxes (lo, hi:
  // words 0-5 and 6-11) and codes (12, 13), every node's own code (14); a code is an inner node's index or -2 - p for
  // a leaf whose items are witem[p], witem[p + 1], ... up to a -1
  const float4* __restrict__ node_w;
  const int32_t* __restrict__ witem;
  const int32_t* __restrict__ kind_i;
  const float* __restrict__ leaf_f;
  const int32_t* __restrict__ leaf_i;
  const float* __restrict__ plane_f;
  const int32_t* __restrict__ prog_i;
  const int32_t* __restrict__ cls_medium;
  const int32_t* __restrict__ cls_born;  // per class the entry class of a sensor counting photons born in it, or null
  const int32_t* __restrict__ pair_pre;  // per class pair 1: the deposit goes to the volume left's sensor, or null
  const int32_t* __restrict__ row_of;
  const int32_t* __restrict__ med_i;
  const int32_t* __restrict__ row_i;
  const int32_t* __restrict__ tab;
  const float* __restrict__ uni;  // the unified facet tables (LUMEN_UNI_WORDS), null without a unified facet row
  const int32_t* __restrict__ comp;   // sensor reach: each volume's component (null: never bounded)
  const float* __restrict__ comp_box;
  const float* __restrict__ fnode_f;
  const int32_t* __restrict__ fnode_i;
  int n_fnode;
  const int32_t* __restrict__ med_jump;  // the diffusion jump: each medium's grid (-1 none; null: no grid at all)
  const float* __restrict__ jump_f;
  const int32_t* __restrict__ jump_i;
  const float* __restrict__ clear;
};

L_DEV float d_dot(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
L_DEV float d_min(float a, float b) { return a < b ? a : b; }
L_DEV float d_max(float a, float b) { return a > b ? a : b; }
L_DEV float d_maxabs3(const float* a) {
  float m = fabsf(a[0]);
  if (fabsf(a[1]) > m) m = fabsf(a[1]);
  if (fabsf(a[2]) > m) m = fabsf(a[2]);
  return m;
}
L_DEV float d_band(float scale) { return D_BAND_ULPS_EPS * scale + D_BAND_FLOOR; }
L_DEV float d_safe_norm(const float* v) { return sqrtf(d_max(d_dot(v, v), D_TINY_NORMAL)); }

L_DEV int vI(const DScene& S, int v, int f) { return __ldg(S.vol_i + (size_t)v * LUMEN_VOL_I + f); }
L_DEV float vF(const DScene& S, int v, int f) { return __ldg(S.vol_f + (size_t)v * LUMEN_VOL_F + f); }
L_DEV int d_cls(const DScene& S, int v) { return vI(S, v, LUMEN_VI_CLS); }
L_DEV int d_parent(const DScene& S, int v) { return vI(S, v, LUMEN_VI_PARENT); }
L_DEV int d_rank(const DScene& S, int i) { return i >= 0 ? -vI(S, i, LUMEN_VI_PRIO) : 0; }


// the precision-generic helpers of the body: overloads in float and double
L_DEV float n_sqrt(float x) { return sqrtf(x); }
L_DEV double n_sqrt(double x) { return sqrt(x); }
L_DEV float n_abs(float x) { return fabsf(x); }
L_DEV double n_abs(double x) { return fabs(x); }
L_DEV float n_cbrt(float x) { return l_cbrt(x); }
L_DEV double n_cbrt(double x) { return l_cbrt64(x); }
// a constant's value in the body's precision: the float32 literal in float, the float64 literal in double
#define NK(x) (sizeof(NF) == 4 ? (NF)(x##f) : (NF)(x))

// a query's result (navigate.py:617 _finish as the step reads it, step.py:260 _query): t in the navigator's precision
// (for the position), every other float in float32
template <class NF>
struct QueryT {
  NF t;
  int hit, cont;
  int vol_after, vol_before, vol_start, cls_before, cls_start, cls_after;
  float normal[3];
  int item, leaf, face, zero;
  float t_pass0, t_pass1;
  int n_pass, vol_at, srf, rounds;
};

namespace nav32 {
using NF = float;
using NF3 = float3;
using NF4 = float4;
#define NAV_IS64 0
#define NAV_VOL(S) (S).vol_f
#define NAV_NODE(S) (S).node_f
#define NAV_LEAF(S) (S).leaf_f
#define NAV_PLANE(S) (S).plane_f
#include "dnav.cuh"
#undef NAV_IS64
#undef NAV_VOL
#undef NAV_NODE
#undef NAV_LEAF
#undef NAV_PLANE
}  // namespace nav32

namespace nav64 {
using NF = double;
using NF3 = double3;
using NF4 = double4;
#define NAV_IS64 1
#define NAV_VOL(S) reinterpret_cast<const double*>((S).vol_f)
#define NAV_NODE(S) reinterpret_cast<const double*>((S).node_f)
#define NAV_LEAF(S) reinterpret_cast<const double*>((S).leaf_f)
#define NAV_PLANE(S) reinterpret_cast<const double*>((S).plane_f)
#include "dnav.cuh"
#undef NAV_IS64
#undef NAV_VOL
#undef NAV_NODE
#undef NAV_LEAF
#undef NAV_PLANE
}  // namespace nav64

using Query = QueryT<float>;

// the step's entry points, by the position's precision
L_DEV float nav_band(float scale) { return nav32::d_band(scale); }
L_DEV double nav_band(double scale) { return nav64::d_band(scale); }
L_DEV float nav_maxabs3(const float* x) { return nav32::d_maxabs3(x); }
L_DEV double nav_maxabs3(const double* x) { return nav64::d_maxabs3(x); }
// EXT: the extended instantiation's locate (skips ancestors among the candidates: protrusion clips)
template <int EXT = 0>
L_DEV int nav_locate(const DScene& S, const float* x) {
  if constexpr (EXT) return nav32::d_locate_x(S, x);
  else return nav32::d_locate(S, x);
}
template <int EXT = 0>
L_DEV int nav_locate(const DScene& S, const double* x) {
  if constexpr (EXT) return nav64::d_locate_x(S, x);
  else return nav64::d_locate(S, x);
}
template <int TORUS>
L_DEV QueryT<float> nav_query(const DScene& S, const float* o, const float* d, int vol, float t_max, int last,
                              const float* sn, float s_at) {
  return nav32::d_query<TORUS>(S, o, d, vol, t_max, last, sn, s_at);
}
template <int TORUS>
L_DEV QueryT<double> nav_query(const DScene& S, const double* o, const double* d, int vol, double t_max, int last,
                               const float* sn, double s_at) {
  return nav64::d_query<TORUS>(S, o, d, vol, t_max, last, sn, s_at);
}
L_DEV float nav_reach_bound(const DScene& S, const float* x, const float* d, int vol, int srf, float s, float t_max) {
  return nav32::d_reach_bound(S, x, d, vol, srf, s, t_max);
}
L_DEV double nav_reach_bound(const DScene& S, const double* x, const float* d, int vol, int srf, float s,
                             double t_max) {
  return nav64::d_reach_bound(S, x, d, vol, srf, s, t_max);
}

}  // namespace lb
