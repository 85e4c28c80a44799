/*
 * ORACLE (test infrastructure): the reference's navigator and CSG evaluator, restated for one ray on the CPU.
 *
 * Follows src/lumen/geometry/csg.py (leaf intervals, the postfix boolean, first_change), leaf_kernels.py (quadric
 * pieces), navigate.py (Geant4 volume tracking with surface identity) and surface_id.py. Candidates are scanned by
 * brute force over each volume's daughters (no acceleration structure), so the engine's BVH is checked against it.
 * Scope: quadric, plane and torus leaves, no meshes, volumes nested in a tree (no overlap owners, no ancestor
 * clipping, no frame groups), plain vertex table (a crossing is visible where the class changes). The body
 * (geom_nav.h) is compiled in both of the reference's precisions: onav32 (float32) and onav64 (the float64 navigator,
 * src/lumen/rules/navigation.py:96); onav_* below pick one by the position's type.
 */
#ifndef LUMEN_ORACLE_GEOM_H
#define LUMEN_ORACLE_GEOM_H

#include <algorithm>

#include "../include/lumen_b200.h"
#include "lmath.h"

#define O_HUGE 1e30f
#define O_BIG 1e29f
#define O_EPS32 1.1920928955078125e-7f
#define O_BAND_ULPS_EPS 9.5367431640625e-07f /* BAND_ULPS (8) x eps32 (src/lumen/rules/tolerances.py:76) */
#define O_BAND_FLOOR 1e-9f
#define O_K_ON 4.0f
#define O_RELOCATE_BANDS 0.25f
#define O_ZERO_STEP_BANDS 0.125f
#define O_PUSH_BANDS 8.0f
#define O_TANGENT_ULPS 16.0f
#define O_DIVISOR_FLOOR 1e-30f
#define O_TINY_DIR 1e-30f
#define O_LINEAR_REL 1e-12f
#define O_PARALLEL 1e-12f
#define O_GRAZE 256.0f
#define O_ZSBP 10 /* ZERO_STEPS_BEFORE_PUSH */
#define O_ZSBK 25 /* ZERO_STEPS_BEFORE_KILL */
#define O_MAX_SCAN_PER_LEAF 4
#define O_MAX_SCAN_EXTRA 5
#define O_TINY_NORMAL 1.17549435e-38f

typedef struct OScene {
  const LumenSceneDesc* D;
  int n;      /* volumes; n = the outside */
  int LM, FM; /* most leaves of a kind, most faces of a leaf (1 + planes) */
  int SU;     /* first face code: a code below it is a plain item */
  int nav64;  /* LUMEN_PREC_FLOAT64: the navigator reads the desc's float64 arrays */
  int n_chunk, ch0, sm; /* mesh chunks, the first chunk id, the first mesh surface code (INT_MAX: no mesh) */
} OScene;

/* ------------------------------------------------------------------------------------------- small vector math */
static inline float o_dot(const float* a, const float* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static inline float o_maxabs3(const float* a) {
  float m = fabsf(a[0]);
  if (fabsf(a[1]) > m) m = fabsf(a[1]);
  if (fabsf(a[2]) > m) m = fabsf(a[2]);
  return m;
}
static inline float o_min(float a, float b) { return a < b ? a : b; }
static inline float o_max(float a, float b) { return a > b ? a : b; }
/* band(scale) = BAND_ULPS eps scale + BAND_FLOOR (src/lumen/rules/navigation.py:121) */
static inline float o_band(float scale) { return O_BAND_ULPS_EPS * scale + O_BAND_FLOOR; }
static inline float o_safe_norm(const float* v) { return sqrtf(o_max(o_dot(v, v), O_TINY_NORMAL)); }

/* ------------------------------------------------------------------------------------------------ accessors */
static inline const int32_t* o_vi(const OScene* S, int v) { return S->D->vol_i + (size_t)v * LUMEN_VOL_I; }
static inline const float* o_vf(const OScene* S, int v) { return S->D->vol_f + (size_t)v * LUMEN_VOL_F; }
static inline const int32_t* o_ki(const OScene* S, int k) { return S->D->kind_i + (size_t)k * LUMEN_KIND_I; }
static inline const float* o_lf(const OScene* S, int g) { return S->D->leaf_f + (size_t)g * LUMEN_LEAF_F; }
static inline const int32_t* o_li(const OScene* S, int g) { return S->D->leaf_i + (size_t)g * LUMEN_LEAF_I; }
static inline const float* o_pl(const OScene* S, int q) { return S->D->plane_f + (size_t)q * LUMEN_PLANE_F; }
static inline int o_cls(const OScene* S, int v) { return o_vi(S, v)[LUMEN_VI_CLS]; }
static inline int o_parent(const OScene* S, int v) { return o_vi(S, v)[LUMEN_VI_PARENT]; }
/* whether volume i is an ancestor of volume v (navigate.py:199 is_ancestor; the walk is depth first) */
static inline int o_is_anc(const OScene* S, int i, int v) {
  return i >= 0 && i < v && v < S->n && v < i + o_vi(S, i)[LUMEN_VI_SIZE];
}
/* rank of a candidate: minus its place in the rule's order (navigate.py:208) */
static inline int o_rank(const OScene* S, int i) { return i >= 0 ? -o_vi(S, i)[LUMEN_VI_PRIO] : 0; }


/* the precision-generic helpers of the body: overloads in float and double */
static inline float n_sqrt(float x) { return sqrtf(x); }
static inline double n_sqrt(double x) { return sqrt(x); }
static inline float n_abs(float x) { return fabsf(x); }
static inline double n_abs(double x) { return fabs(x); }
static inline float n_cbrt(float x) { return o_cbrt(x); }
static inline double n_cbrt(double x) { return o_cbrt64(x); }
/* a constant's value in the body's precision: the float32 literal in float, the float64 literal in double */
#define NK(x) (sizeof(NF) == 4 ? (NF)(x##f) : (NF)(x))

/* a query's result (navigate.py:617 _finish as the step reads it, step.py:260 _query): t in the navigator's
   precision (for the position), every other float in float32 */
template <class NF>
struct OQueryT {
  NF t;
  int hit, cont;
  int vol_after, vol_before, vol_start, cls_before, cls_start, cls_after;
  float normal[3];
  int item, leaf, face, zero;
  float t_pass0, t_pass1;
  int n_pass, vol_at, srf, rounds;
};

namespace onav32 {
typedef float NF;
#define O_NAV_VOL(S) (S)->D->vol_f
#define O_NAV_LEAF(S) (S)->D->leaf_f
#define O_NAV_PLANE(S) (S)->D->plane_f
#define O_NAV_TRI(S) (S)->D->mesh_tri
#define O_NAV_CBOX(S) (S)->D->chunk_box
#include "geom_nav.h"
#undef O_NAV_VOL
#undef O_NAV_LEAF
#undef O_NAV_PLANE
#undef O_NAV_TRI
#undef O_NAV_CBOX
}  // namespace onav32

namespace onav64 {
typedef double NF;
#define O_NAV_VOL(S) (S)->D->vol_f64
#define O_NAV_LEAF(S) (S)->D->leaf_f64
#define O_NAV_PLANE(S) (S)->D->plane_f64
#define O_NAV_TRI(S) (S)->D->mesh_tri64
#define O_NAV_CBOX(S) (S)->D->chunk_box64
#include "geom_nav.h"
#undef O_NAV_VOL
#undef O_NAV_LEAF
#undef O_NAV_PLANE
#undef O_NAV_TRI
#undef O_NAV_CBOX
}  // namespace onav64

typedef OQueryT<float> OQuery;

/* the step's entry points, by the position's precision */
static inline float onav_band(float scale) { return onav32::o_band(scale); }
static inline double onav_band(double scale) { return onav64::o_band(scale); }
static inline float onav_maxabs3(const float* x) { return onav32::o_maxabs3(x); }
static inline double onav_maxabs3(const double* x) { return onav64::o_maxabs3(x); }
static inline int onav_locate(const OScene* S, const float* x) { return onav32::o_locate(S, x); }
static inline int onav_locate(const OScene* S, const double* x) { return onav64::o_locate(S, x); }
static inline OQueryT<float> onav_query(const OScene* S, const float* o, const float* d, int vol, float t_max, int last,
                                        const float* sn, float s_at) {
  return onav32::o_query(S, o, d, vol, t_max, last, sn, s_at);
}
static inline OQueryT<double> onav_query(const OScene* S, const double* o, const double* d, int vol, double t_max,
                                         int last, const float* sn, double s_at) {
  return onav64::o_query(S, o, d, vol, t_max, last, sn, s_at);
}

#endif
