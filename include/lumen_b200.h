/*
 * lumen_b200 — C ABI of the B200 photon-transport engine (the photon loop behind lumen.simulate).
 *
 * The reference runs its photon loop through tallymap (src/lumen/run.py:93 `run`, :693 `trace`, :534 `rebuild`):
 * one item per photon loops `step` (src/lumen/transport/step.py:516) until the photon ends, appends a deposit record
 * per sensor crossing, and a second launch folds the records into per-sensor cells. This library replaces that seam:
 * one call traces a batch of photons on the GPU and reduces their deposits straight into per-sensor FP64 tallies
 * (arrival, arrival x time, per-photon second moment, time histograms, health fates, and optionally the Jacobian of
 * the arrivals in the run's gradient parameters).
 *
 * Conventions: plain C types and pointers only; every entry point returns a LumenStatus (0 = OK), never throws; a
 * scene handle is immutable after creation except for its parameter pools (lumen_b200_scene_set_pools), and one
 * handle may serve concurrent calls on different streams. Pointers documented "device" are CUDA device memory owned
 * by the caller; "host" pointers are read during the call only.
 */
#ifndef LUMEN_B200_H
#define LUMEN_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LUMEN_B200_ABI_VERSION 15

typedef enum LumenStatus {
  LUMEN_OK = 0,
  LUMEN_ERR_ARG = 1,          /* a bad argument: null pointer, size out of range, inconsistent scene arrays */
  LUMEN_ERR_CUDA = 2,         /* a CUDA runtime call failed (the message says which) */
  LUMEN_ERR_SCENE = 3,        /* the scene uses a feature this engine does not build (see lumen_b200_last_error) */
  LUMEN_ERR_STEP_BUDGET = 4,  /* the device step budget of the call ran out before every photon ended */
  LUMEN_ERR_NO_DEVICE = 5,    /* no CUDA device, or not an sm_100 device */
  LUMEN_ERR_NOT_SUPPORTED = 6, /* a request outside this build (e.g. more gradient parameters than LUMEN_MAX_GRAD) */
  LUMEN_ERR_RECORDS = 7       /* the deposit records outgrew LumenTallies.rec_capacity (src/lumen/run.py:236
                                 RecordsOverflow): counts[LUMEN_C_RECORDS] is the capacity needed; the groups' cells
                                 are not filled, every other tally is */
} LumenStatus;

/* ---------------------------------------------------------------------------------------------- array layouts */
/* Per volume v (0..n_vol-1; index n_vol is the outside; then, with meshes, mesh k's pseudo-volume at n_vol + 1 + k and
   mesh chunk c at LUMEN's CH0 + c, CH0 = n_vol + 1 + n_mesh: their kind is -1, their parent the mesh's mother, their
   class and order the mesh's, no candidates, no BVH), int record of LUMEN_VOL_I int32: */
enum {
  LUMEN_VI_KIND = 0,   /* the solid (kind) of the volume; -1 for the outside */
  LUMEN_VI_PARENT = 1, /* the mother volume (n_vol for a top volume; -1 for the outside) */
  LUMEN_VI_CLS = 2,    /* the surface lookup's class */
  LUMEN_VI_SENSOR = 3, /* sensor index, -1 none */
  LUMEN_VI_PRIO = 4,   /* the locate rule's order among siblings (lower first) */
  LUMEN_VI_C0 = 5,     /* first candidate (daughter) in cand[] */
  LUMEN_VI_CN = 6,     /* number of candidates */
  LUMEN_VI_NODE0 = 7,  /* first BVH node of the volume's daughter BVH (world frame) */
  LUMEN_VI_NODE1 = 8,  /* one past its last node (NODE0 == NODE1: no daughters) */
  LUMEN_VI_SIZE = 9,   /* the volumes of its subtree, itself included (the walk is depth first: an ancestor of w is a
                          v < w < v + size); a candidate that is an ancestor is one the volume reaches out of (a
                          protrusion clip, src/lumen/geometry/ownership.py:679): its face is an exit */
  LUMEN_VOL_I = 10
};
/* Per volume, float record of LUMEN_VOL_F float32: R (3x3 row-major, world = R local + t), t (3), padded world box */
enum { LUMEN_VF_R = 0, LUMEN_VF_T = 9, LUMEN_VF_LO = 12, LUMEN_VF_HI = 15, LUMEN_VOL_F = 18 };
/* BVH node: float lo (3), hi (3); int skip (next node when not descending), count (items at a leaf), start */
enum { LUMEN_NODE_F = 6, LUMEN_NODE_I = 4 };
/* Kind (one distinct solid): int l0 (first leaf), nl (leaves), p0 (first program op), pl (program length) */
enum { LUMEN_KIND_I = 4 };
/* Leaf: float og (3) plane origin, oq (3) quadric origin, A (9, row-major), b (3), c, sa = max |A_ij| */
enum { LUMEN_LF_OG = 0, LUMEN_LF_OQ = 3, LUMEN_LF_A = 6, LUMEN_LF_B = 15, LUMEN_LF_C = 18, LUMEN_LF_SA = 19,
       LUMEN_LEAF_F = 20 };
/* Leaf ints: typ (0: planes only, 1: quadric and planes, 2: a solid torus {(rho - R)^2 + z^2 <= r^2} in canonical
   coordinates u = M (x - og), M row-major at LUMEN_LF_A, R at LUMEN_LF_B, r at LUMEN_LF_B + 1; a torus reads no
   planes), p0 (first plane), np (planes) */
enum { LUMEN_LEAF_I = 4 };
/* Plane: n (3), h — the leaf holds n . (x - og) <= h */
enum { LUMEN_PLANE_F = 4 };
/* Program op: op (0 push leaf arg, 1 union, 2 intersection, 3 subtraction), arg */
enum { LUMEN_PROG_I = 2 };

/* Surface table: row ints of LUMEN_ROW_I: model (0 reflect, 1 dielectric, 2 complex index), normal, glisur (the
   GLOSSY lobe: 0 the unified facet path, 1 GLISUR's on a metal, 2 GLISUR's reflecting or refracting facets),
   far_opaque, per_normal, cover, then one table index per column (LUMEN_COL_*) read at the photon energy.
   cover: the defensive mixture's outcomes of an edge row (src/lumen/transport/estimator.py:146 edge_floor): bit o set
   for each outcome o (LUMEN_OUT_*) of the row type's support (src/lumen/build/lookup.py:999) when the row reads a
   parameter with a defensive role (src/lumen/api.py:797 _edge_rows); 0 for every other row. At a crossing of such a
   row each covered outcome whose reference probability is 0 is drawn at e / (1 - e) / n, e = 0.01
   (src/lumen/transport/estimator.py:83 defensive). */
enum { LUMEN_OUT_STRAIGHT = 0, LUMEN_OUT_REFRACT, LUMEN_OUT_SPECULAR, LUMEN_OUT_BACKSCATTER, LUMEN_OUT_GLOSSY,
       LUMEN_OUT_DIFFUSE, LUMEN_N_OUT };
enum { LUMEN_COL_R = 0, LUMEN_COL_T, LUMEN_COL_EFF, LUMEN_COL_PSPIKE, LUMEN_COL_PLOBE, LUMEN_COL_PBACK,
       LUMEN_COL_SIGMA, LUMEN_COL_POLISH, LUMEN_COL_NR, LUMEN_COL_NK, LUMEN_N_COL };
enum { LUMEN_RI_MODEL = 0, LUMEN_RI_NORMAL = 1, LUMEN_RI_GLISUR = 2, LUMEN_RI_FAR_OPAQUE = 3,
       LUMEN_RI_PER_NORMAL = 4, LUMEN_RI_COVER = 5, LUMEN_RI_COL = 6, LUMEN_ROW_I = 16 };
/* Medium ints, one table index each (-1: none), src/lumen/media/bulk.py:45 Medium with its channels in Geant4's order
   (bulk.py:21 CHANNEL_ORDER): the index (-1: opaque), the absorption length, the Rayleigh length; the Mie (G4OpMieHG)
   length and its lobe constants g_forward, g_backward, forward_ratio (MIEHG, MIEHG_FORWARD, MIEHG_BACKWARD,
   MIEHG_FORWARD_RATIO); the WLS (G4OpWLS) absorption length, mean photons, time constant (ns) and emission spectrum
   (WLSABSLENGTH, WLSMEANNUMBERPHOTONS, WLSTIMECONSTANT, WLSCOMPONENT: energies as the knots, intensities as the
   values); then the WLS time profile as a plain int (0: delta, Geant4's default; 1: exponential); then a plain int,
   1 where the Mie lobe choice is a defensive part (its forward ratio a keyed parameter, src/lumen/api.py:797
   _edge_rows: drawn at the ratio's cover, src/lumen/media/phase.py:173 _mie_cover, weighted live / covered,
   src/lumen/transport/medium.py:96 channel_draw), else not. A channel whose length table is -1 is absent. */
enum { LUMEN_MI_INDEX = 0, LUMEN_MI_ABS = 1, LUMEN_MI_RAY = 2, LUMEN_MI_MIE = 3, LUMEN_MI_MIE_GF = 4,
       LUMEN_MI_MIE_GB = 5, LUMEN_MI_MIE_R = 6, LUMEN_MI_WLS = 7, LUMEN_MI_WLS_YIELD = 8, LUMEN_MI_WLS_TAU = 9,
       LUMEN_MI_WLS_SPEC = 10, LUMEN_MI_WLS_PROFILE = 11, LUMEN_MI_MIE_COVER = 12, LUMEN_MED_I = 16 };
enum { LUMEN_N_CHANNEL = 3 };  /* bulk channels: Rayleigh, Mie, WLS */
/* Table t: tab[2t] = offset into a pool, tab[2t+1] = knots k >= 1; pool[off .. off+k) energies (eV, ascending),
   pool[off+k .. off+2k) values; linear in photon energy between knots, held beyond (G4PhysicsVector::Value) */

#define LUMEN_MAX_GRAD 8      /* gradient parameters per call */
#define LUMEN_MAX_LEAVES 8    /* leaves per solid */
#define LUMEN_MAX_PLANES 8    /* planes per leaf */
#define LUMEN_MAX_KNOTS 64    /* knots of an index table (its group index is tabulated per call) */
#define LUMEN_MAX_BVH_DEPTH 24 /* levels of a volume's daughter BVH (the traversal's stack) */

/* The unified facet lobe's tables (src/lumen/surfaces/facets.py:127 unified_tables; grid in
   src/lumen/rules/choices.py:101 UNIFIED_TABLE): the facing share F on x = (2/pi) atan2(cos theta, sigma sin theta)
   (NX uniform nodes of [0, 1]) by y = log sigma = Y0 + DY j, j in [J_LO, J_LO + NY), with its node derivatives Fx,
   Fy, Fxy (each NX x NY float32, row-major: F[i * NY + j]), then log zeta = log(Z / sigma^2) and its derivative in
   y (NY each), flat in that order. sigma_alpha of a unified facet row must lie in [exp(Y0 + DY J_LO),
   exp(Y0 + DY (J_LO + NY - 1))] = [0.00276, 1] rad. */
#define LUMEN_UNI_NX 257
#define LUMEN_UNI_NY 69
#define LUMEN_UNI_J_LO (-52)
#define LUMEN_UNI_Y0 (-1.38629436111989061883)  /* log(1/4) */
#define LUMEN_UNI_DY 0.08664339756999316368     /* log(2) / 8 */
#define LUMEN_UNI_WORDS (4 * LUMEN_UNI_NX * LUMEN_UNI_NY + 2 * LUMEN_UNI_NY)

/* the diffusion jump's grid records */
enum { LUMEN_JUMP_F = 4, LUMEN_JUMP_I = 8 };
#define LUMEN_JUMP_STEPS 65536 /* a walk's scatterings at most: any stopping time is exact in law (fastpath.py:5-10);
                                  this one bounds a lane's loop */

/* ------------------------------------------------------------------------------------------ the detector */
typedef struct LumenSceneDesc {
  /* geometry (the navigator's arrays, src/lumen/geometry/navigator_build.py:51, csg_build.py:30) */
  int32_t n_vol, n_kind, n_leaf, n_plane, n_prog, n_node, n_item, n_cand;
  const int32_t* vol_i;   /* host, (n_vol + 1 + n_mesh + n_chunk) * LUMEN_VOL_I */
  const float* vol_f;     /* host, n_vol * LUMEN_VOL_F */
  const int32_t* cand;    /* host, n_cand: daughters per volume (and the outside's top volumes) */
  const float* node_f;    /* host, n_node * LUMEN_NODE_F */
  const int32_t* node_i;  /* host, n_node * LUMEN_NODE_I */
  const int32_t* items;   /* host, n_item: BVH leaf items (volume ids) */
  const int32_t* kind_i;  /* host, n_kind * LUMEN_KIND_I */
  const float* leaf_f;    /* host, n_leaf * LUMEN_LEAF_F */
  const int32_t* leaf_i;  /* host, n_leaf * LUMEN_LEAF_I */
  const float* plane_f;   /* host, n_plane * LUMEN_PLANE_F */
  const int32_t* prog_i;  /* host, n_prog * LUMEN_PROG_I */
  float reach;            /* m: the diagonal of the box holding every volume (transport/step.py:98) */
  /* optics (the surface lookup, src/lumen/build/lookup.py:394; media, src/lumen/media/bulk.py:88) */
  int32_t n_cls, n_med, n_row, n_tab, n_pool, n_sensor;
  const int32_t* cls_medium; /* host, n_cls */
  const int32_t* row_of;     /* host, n_cls * n_cls: surface row of a (class left, class met) pair, -1 none */
  const int32_t* med_i;      /* host, n_med * LUMEN_MED_I */
  const int32_t* row_i;      /* host, n_row * LUMEN_ROW_I */
  const int32_t* tab;        /* host, n_tab * 2 */
  const float* pool;         /* host, n_pool: the table values every call reads unless set_pools replaces them */
  const float* unified;      /* host, LUMEN_UNI_WORDS: the unified facet tables; may be null when no row draws the
                                unified facet lobe (src/lumen/surfaces/facets.py:165 table_operands) */
  /* sensor reach (src/lumen/geometry/reach.py:66 build): a bulk step's query stops just past its free path where the
     segment to its component's box exit meets no sensor box, an exact speed-up. All null / 0: never bounded. */
  int32_t n_comp, n_fnode;
  const int32_t* comp;       /* host, n_vol + 1: each volume's component (volumes joined by crossings without a
                                vertex); the outside's is -1 */
  const float* comp_box;     /* host, n_comp * 6: each component's padded box (lo, hi) */
  const float* fnode_f;      /* host, n_fnode * LUMEN_NODE_F: a depth-first tree over the padded sensor boxes */
  const int32_t* fnode_i;    /* host, n_fnode * LUMEN_NODE_I: skip (the node after the subtree), count (> 0: a leaf) */
  /* the diffusion jump (src/lumen/transport/fastpath.py): one proven clearance grid per medium the jump can act in
     (Rayleigh its only channel), used with LUMEN_F_JUMP. 0 / null: no grid. */
  int32_t n_jump;
  const float* jump_f;       /* host, n_jump * LUMEN_JUMP_F: the grid's origin (3, m) and spacing (m) */
  const int32_t* jump_i;     /* host, n_jump * LUMEN_JUMP_I: medium, nodes per axis (3), first node in clear */
  int64_t n_clear;
  const float* clear;        /* host, n_clear: the grids' clearances (m) at their nodes, node (i, j, k) at
                                first + (i * n1 + j) * n2 + k */
  /* the navigator's precision (src/lumen/rules/navigation.py:96 Precision, the load option precision=): with
     LUMEN_PREC_FLOAT64 the navigator (frames, BVH boxes, leaf coefficients, plane slabs, roots, intervals and the
     band) and the photon's position are float64 and the physics stays float32, as the reference's float64 navigator.
     The float64 arrays below then hold the same geometry as vol_f, node_f, leaf_f and plane_f, built in float64 (not
     widened from the float32 arrays); null with LUMEN_PREC_FLOAT32. The sensor reach and the jump grids stay float32
     in either precision, as the reference's (src/lumen/geometry/reach.py:88, transport/fastpath.py:177). */
  int32_t precision;
  const double* vol_f64;     /* host, n_vol * LUMEN_VOL_F */
  const double* node_f64;    /* host, n_node * LUMEN_NODE_F */
  const double* leaf_f64;    /* host, n_leaf * LUMEN_LEAF_F */
  const double* plane_f64;   /* host, n_plane * LUMEN_PLANE_F */
  /* tessellated meshes (G4TessellatedSolid; src/lumen/geometry/scene.py:33 Mesh, navigator_build.py:266
     _mesh_chunks): opaque parts of closed triangle surfaces. Triangles (world, each LUMEN_TRI_F: V0, V1, V2 and the
     unit normal (V1 - V0) x (V2 - V0), outward) in chunks of at most LUMEN_MESH_CHUNK consecutive triangles; each chunk
     is a BVH item (navigator id CH0 + c) of its mesh's mother. A facet met from either side is an entry into the mesh
     (navigate.py:303 the facet rule); the mesh's class is that of its pseudo-volume. 0 / null: no mesh. */
  int32_t n_mesh, n_chunk, n_tri;
  const float* mesh_tri;     /* host, n_tri * LUMEN_TRI_F */
  const double* mesh_tri64;  /* host, n_tri * LUMEN_TRI_F: the float64 navigator's (LUMEN_PREC_FLOAT64) */
  const int32_t* mesh_chunk; /* host, n_chunk * LUMEN_CHUNK_I: first triangle, count, mesh, 0 */
  const float* chunk_box;    /* host, n_chunk * 6: each chunk's padded world box (lo, hi), its BVH leaf's */
  const double* chunk_box64; /* host, n_chunk * 6: the same in float64 */
  /* frame groups (src/lumen/geometry/navigator_build.py:11, bvh.py:20): a volume's daughters sharing a rotation R
     whose world boxes are much larger than their own (diagonal wire planes) get a BVH of their own in R's frame
     (x_g = R^T x_w), nodes in node_f / node_i after the volume's world-frame BVH; its members are not in that one.
     0 / null: none. */
  int32_t n_group;           /* at most LUMEN_MAX_GROUPS_PER_VOLUME in one volume */
  const int32_t* group_i;    /* host, n_group * 4: the volume, first node, end node, 0 */
  const float* group_r;      /* host, n_group * 9: R row-major */
  const double* group_r64;   /* host, n_group * 9: the float64 navigator's */
  /* sensors that count a photon born inside them (a group counting by volume, Geant4's sensitive detector:
     src/lumen/rules/sensors.py:39 counts_born; Optics.born_pair): per class c the class b whose crossing (b, c) is
     its entry, -1 none. A photon whose first step starts in a sensor volume of such a class deposits there what that
     entry's row (row_of[b][c]; -1: nothing) detects, evaluated unpolarised at normal incidence with both indices 1,
     at its emission time, and ends: its whole weight absorbed at a surface (src/lumen/transport/step.py:574 _born).
     null: no such sensor. */
  const int32_t* cls_born;   /* host, n_cls */
  /* exit sensors (a border out of a sensor's volume whose surface has an EFFICIENCY: Geant4's boundary process
     detects there, src/lumen/rules/boundary.py:92 "credited to pre"; Optics.deposit_pre): per (class left, class met)
     pair 1 where the crossing's deposit goes to the sensor of the volume left (and its local fields are read in that
     volume's frame, src/lumen/transport/step.py:615 _sensor_dep, :653 sensor_frame), else 0. null: none. */
  const int32_t* pair_pre;   /* host, n_cls * n_cls */
} LumenSceneDesc;

enum { LUMEN_TRI_F = 12, LUMEN_CHUNK_I = 4, LUMEN_MESH_CHUNK = 8, LUMEN_MAX_GROUPS_PER_VOLUME = 64 };

enum { LUMEN_PREC_FLOAT32 = 0, LUMEN_PREC_FLOAT64 = 1 };

typedef struct LumenScene LumenScene; /* opaque: the device copy of a LumenSceneDesc */

/* ------------------------------------------------------------------------------------------- the photons */
/* Explicit emission rows, structure of arrays on the device (src/lumen/record.py Photons: x, d, t, lam, w, pol).
   pol may be null: every row unpolarised (E = 0). */
typedef struct LumenRows {
  const float *x, *y, *z;       /* device, n: start position (m) */
  const float *dx, *dy, *dz;    /* device, n: unit direction */
  const float *t, *lam, *w;     /* device, n: time (ns), wavelength (nm), the row's weight w0 */
  const float* pol;             /* device, n * 6 (er xyz, ei xyz) or null */
  const int32_t* event;         /* device, n: the event each row tallies into, or null (event 0) */
} LumenRows;

/* A procedural source drawn on the device from the photon's own key (src/lumen/sources/_base.py:312): photon i of
   the call belongs to the event e with ev_first[e] <= first_id + i < ev_first[e + 1]. */
enum { LUMEN_SRC_POINT = 0,   /* isotropic point (sources/point.py:73): ev_f = x y z, time */
       LUMEN_SRC_TRACK = 1,   /* straight track emitting on a cone: ev_f = x y z (start), ux uy uz (unit), length, time */
       LUMEN_SRC_SCINT = 2,   /* isotropic scintillation point with a two-exponential profile: ev_f = x y z, time */
       LUMEN_SRC_CHERENKOV = 3 }; /* a charged segment's Cherenkov light (src/lumen/sources/cherenkov.py:65
                                    CherenkovSegment): ev_f = x y z (start), ux uy uz (unit), length, time, beta,
                                    charge, the event's photons; the medium's RINDEX table `rindex_tab` read at the live
                                    values; wavelengths over [lam0, lam1] (its span) */
enum { LUMEN_SRC_SCINT_MATERIAL = 4 }; /* a material's scintillation light (src/lumen/sources/scintillation.py:100):
                                    a flash at a point or along a charged segment; ev_f = x0 y0 z0, t0, x1 y1 z1, t1,
                                    energy (MeV), birks (m / MeV); the material's tables in `mat` */
/* LumenSource.mat of LUMEN_SRC_SCINT_MATERIAL: the components (1..3), the segment flag (0: a point at x0, t0), the
   rise flag (the components' rise times), the yield per MeV table, then per component (-1 where absent) its spectrum,
   decay time and rise time tables, then the three share yields (SCINTILLATIONYIELDi; -1: Geant4's defaults 1, 0, 0) */
enum { LUMEN_SM_N = 0, LUMEN_SM_SEGMENT, LUMEN_SM_RISES, LUMEN_SM_YIELD, LUMEN_SM_SPEC = 4, LUMEN_SM_TAU = 7,
       LUMEN_SM_RISE = 10, LUMEN_SM_SHARE = 13, LUMEN_SM_WORDS = 16 };
enum { LUMEN_EV_F = 12 };
typedef struct LumenSource {
  int32_t kind;
  int32_t n_events;
  const float* ev_f;        /* device, n_events * LUMEN_EV_F */
  const int64_t* ev_first;  /* device, n_events + 1: prefix sums of the events' photon counts */
  const float* ev_w;        /* device, n_events: each photon's row weight w0 in that event */
  float lam0, lam1;         /* nm: a fixed wavelength (lam1 <= lam0) or uniform in [lam0, lam1] */
  float cone_cos;           /* LUMEN_SRC_TRACK: cosine of the cone half-angle */
  float tau1, tau2, frac1;  /* LUMEN_SRC_SCINT: decay times (ns) and the first component's share */
  int32_t rindex_tab;       /* LUMEN_SRC_CHERENKOV: the medium's RINDEX table (a gradient parameter it may not be) */
  int32_t reserved;
  int32_t mat[LUMEN_SM_WORDS]; /* LUMEN_SRC_SCINT_MATERIAL: its tables (LUMEN_SM_*; none a gradient parameter) */
} LumenSource;

/* ------------------------------------------------------------------------------------------ the controls */
enum { LUMEN_F_ASYNC = 1,   /* controls.flags: enqueue only (no host wait, no status read back: capturable in a
                                 CUDA graph); a step budget that ran out then shows in counts[LUMEN_C_ABORTED] */
       LUMEN_F_REACH = 2,    /* bound bulk steps' queries by the scene's sensor reach (exact: every tally is the same;
                                off by default, a speed-up only where bulk steps are common and sensors far) */
       LUMEN_F_JUMP = 4,     /* the diffusion jump at bulk Rayleigh events (fastpath.py; lumen.simulate's default):
                                the same estimator in law as the plain walk, not the same photons */
       LUMEN_F_TRUTH = 8 };  /* truth rows (src/lumen/readout/truth.py): each photon carries its analog photon
                                (src/lumen/transport/state.py:30 Analog, step.py:625 _analog_crossing, :649
                                _analog_roulette) and writes its record to LumenTallies.truth; forward runs at one set
                                of values only (no gradient parameters, no distinct reference pool), the persistent
                                loop (shape 0) whatever the variant, row weights <= 1 */
/* A photon's analog record (LumenTallies.truth, one per photon of the call, 32-bit words): the sensor it was absorbed
   on (-1: none), the time (ns) and wavelength (nm) there, the sensor row's 1 / A_n (1 unless read per normal
   incidence), the crossing point (m, world) and the volume entered */
enum { LUMEN_TR_SENSOR = 0, LUMEN_TR_TIME, LUMEN_TR_LAM, LUMEN_TR_SCALE, LUMEN_TR_POS, LUMEN_TR_VOL = 7,
       LUMEN_TRUTH_WORDS = 8 };
enum { LUMEN_VARIANT_WAVEFRONT = 3, LUMEN_N_VARIANT = 4 };
/* launch variants: the persistent photon loop at 0 = 256 threads x 4 blocks / SM (64 registers), 1 = 128 x 8 (64),
   2 = 256 x 3 (85 registers); 3 = the wavefront: rounds of two kernels (the query; the rest of the step and the
   refill) over a pool of slots in HBM, then the persistent loop resuming the slots still live (its drain: one thread
   a slot, then the photons left). A synchronous call reads a live-slot count back every four rounds and drains once
   fewer than a 64th of the slots are live; a LUMEN_F_ASYNC call runs a fixed number of rounds (wave_rounds) and
   drains, reading nothing back. Every variant gives the same photons the same paths. */
typedef struct LumenControls {
  float max_distance;      /* m: a query's reach (<= 0: the scene's reach) */
  float roulette;          /* epsilon > 0 (src/lumen/rules/choices.py:112) */
  int32_t max_vertices;    /* the per-photon vertex guard (src/lumen/run.py:70) */
  int32_t n_grad;          /* gradient parameters (0..LUMEN_MAX_GRAD) */
  int32_t grad_tab[LUMEN_MAX_GRAD];  /* each parameter: the table whose values all move together (d/d value) */
  int64_t step_budget;     /* device step budget of the call (<= 0: none) */
  int32_t flags;           /* LUMEN_F_* */
  int32_t variant;         /* launch variant (0 .. LUMEN_N_VARIANT - 1), from the autotuner */
  int32_t blocks_per_sm;   /* resident blocks per SM launched (<= 0: as many as fit) */
  int32_t wave_slots_log2; /* the wavefront's slots: 2^k photons in flight, k in 16 .. 23 (else 2^21), from the
                              autotuner: each slot carries n / 2^k photons in turn */
  int32_t wave_rounds;     /* the wavefront's rounds in a LUMEN_F_ASYNC call, which reads no round back: after them
                              the persistent loop finishes the live slots and the photons left (<= 0: the scene's
                              rounds per photon a slot carries, measured by its last synchronous wavefront call, else
                              3, times the photons a slot carries). A synchronous call reads the live slots back every
                              fourth round and hands the tail (fewer than a 64th of the slots live) to the
                              persistent loop; it ignores this field. */
} LumenControls;

/* --------------------------------------------------------------------------------------------- the tallies */
/* Device outputs, FP64, ADDED to (the caller zeroes them): per event e and sensor s, index e * n_sensor + s. */
enum { LUMEN_H_LOST = 0, LUMEN_H_ABANDONED, LUMEN_H_ESCAPED, LUMEN_H_DISTANCE_CUT, LUMEN_H_ABSORBED_BULK,
       LUMEN_H_ABSORBED_SURFACE, LUMEN_H_ROULETTED, LUMEN_H_REWEIGHTED, LUMEN_H_TRUNCATED, LUMEN_H_PUSHED,
       LUMEN_H_START, LUMEN_N_HEALTH };
/* Counts: photons ended, steps, deposits (records), photons cut at the vertex guard, MULTI the per-photon sensor sums
   past a photon's first four (each photon's sum per sensor is exact whatever their number: the first four are kept in
   registers, the rest in the call's moment table), ABORTED (the step budget ran out), RECORDS (the readout groups'
   record count), MOMENT_LOST the sums that found the moment table full (each squared alone: the second moment is
   then not exact; 0 in every call whose table is large enough). */
enum { LUMEN_C_PHOTONS = 0, LUMEN_C_STEPS, LUMEN_C_DEPOSITS, LUMEN_C_TRUNCATED, LUMEN_C_MULTI, LUMEN_C_ABORTED,
       LUMEN_C_RECORDS, LUMEN_C_MOMENT_LOST, LUMEN_N_COUNT };

/* ------------------------------------------------------------------------------------ the readout groups */
/* The histograms of src/lumen/readout/grid.py filled from the deposit records (src/lumen/readout/fill.py:88
   readout), per sensor group: charge (S, *axes) on the deposit's features, its per-photon second moment charge2, and
   on a timed grid the time nodes t0 + j dt (S, *delay_axes, nt) with the cubic Lagrange split and the late / early
   overflow (q and q t). A deposit's features are read in the frame of the sensor's placement (the volume entered,
   src/lumen/transport/step.py:663 sensor_frame): src/lumen/sensors/features.py BUILTIN. */
enum { LUMEN_FEAT_WAVELENGTH = 0, LUMEN_FEAT_THETA, LUMEN_FEAT_COS_INCIDENCE, LUMEN_FEAT_GENERATION, LUMEN_FEAT_X,
       LUMEN_FEAT_Y, LUMEN_FEAT_Z, LUMEN_FEAT_RHO, LUMEN_N_FEAT };
#define LUMEN_MAX_AXES 4      /* charge axes + delay axes of one group */
#define LUMEN_MAX_GROUPS 8
typedef struct LumenAxis {    /* grid.py:63 Axis */
  int32_t feature;            /* LUMEN_FEAT_* */
  int32_t n;                  /* values (>= 2, ascending) */
  int32_t knots;              /* 1: hat functions on the values (n cells, constant beyond the ends); 0: cells between
                                 the values as edges (n - 1 cells; none outside) */
  int32_t reserved;
  const float* values;        /* device (host for the checker), n */
} LumenAxis;
typedef struct LumenGroup {   /* one sensor group's grid (grid.py:100 Grid) and its cells */
  int32_t n_axes, n_delay;    /* the charge axes, then the delay axes, in axes[] */
  int32_t nt;                 /* time nodes (0: no time histogram) */
  int32_t weighted;           /* the time histogram weighted by `weights` read at the deposit's charge cells */
  int32_t normalise;          /* each deposit times its surface's 1 / A_n (rows flagged LUMEN_RI_PER_NORMAL) */
  int32_t n_sensors;          /* the group's sensors */
  float t0, dt;               /* ns: the first node and the spacing */
  LumenAxis axes[LUMEN_MAX_AXES];
  const int32_t* index;       /* device, n_sensor: each detector sensor's position in the group (-1: not in it);
                                 null: every sensor, in order */
  const float* weights;       /* device, the acceptance per charge cell (the group's cells), or null: none */
  double* charge;             /* device, n_events * n_sensors * cells: sum of q w0 x the cell weight */
  double* charge2;            /* same: sum over photons of (the photon's adds to the cell)^2 */
  double* time;               /* device, n_events * n_sensors * delay cells * nt (nt > 0; else null) */
  double* over_q;             /* device, n_events * n_sensors * delay cells * 2: [late, early] q */
  double* over_qt;            /* same: q t */
} LumenGroup;
#define LUMEN_REC_WORDS 20    /* one deposit record (80 bytes): the readout groups' scratch */
typedef struct LumenTallies {
  int32_t n_events;          /* events tallied (>= 1) */
  int32_t n_bins;            /* time-histogram bins per sensor (0: none) */
  float bin0, bin_w;         /* ns: first bin edge and width */
  double* arrival;           /* device, n_events * n_sensor: sum of q w0 (src/lumen/readout/fill.py:216) */
  double* arrival_t;         /* device, same: sum of q w0 time */
  double* arrival2;          /* device, same: sum over photons of (the photon's sum of q w0)^2 */
  double* hist;              /* device, n_events * n_sensor * n_bins, or null */
  double* jac;               /* device, n_events * n_sensor * n_grad: d arrival / d parameter, or null */
  double* health;            /* device, LUMEN_N_HEALTH: the fates summed over photons (times w0) */
  unsigned long long* counts;/* device, LUMEN_N_COUNT */
  /* the readout groups (n_groups 0: none; lumen_b200_trace only): the trace appends a record per sensor deposit to
     `records` (device scratch of rec_capacity * LUMEN_REC_WORDS 32-bit words, 16-byte aligned), then bins them */
  int32_t n_groups;
  int32_t reserved;
  const LumenGroup* groups;  /* host, n_groups */
  double* pe2;               /* device, n_events * n_sensor, or null: per photon (its q x the group's acceptance at its
                                charge cells)^2, the pe moment of src/lumen/readout/fill.py:200 */
  void* records;
  int64_t rec_capacity;
  float* truth;              /* device, n (the call's photons) * LUMEN_TRUTH_WORDS: the analog records (LUMEN_F_TRUTH) */
} LumenTallies;

/* ------------------------------------------------------------------------------------------- entry points */
/* Version of this ABI (LUMEN_B200_ABI_VERSION). */
int32_t lumen_b200_abi_version(void);
/* The last error message of this thread (static storage; "" after success). */
const char* lumen_b200_last_error(void);

/* The kernels the calling thread's last call of an entry point launched (its trace kernels, the wavefront's rounds,
   the moment table's pass, the readout groups' binning): for a caller counting its GPU work. No counterpart in the
   reference (tallymap launches its kernels itself). */
int64_t lumen_b200_last_launches(void);

/* Upload a detector to the current CUDA device; replaces the reference's Navigator.operands / pack.pack device put
   (src/lumen/geometry/navigate.py:140, src/lumen/api.py:842). Unified rows with sigma_alpha > 0 draw Geant4's facet
   path (src/lumen/surfaces/facets.py:372), weighted by its path density from desc->unified; GLISUR rows (polish < 1)
   draw GLISUR's facet paths (facets.py:341-548). */
int32_t lumen_b200_scene_create(const LumenSceneDesc* desc, LumenScene** out);
/* Replace the live and reference parameter pools (host, n_pool floats each; ref may be null: the live pool): the
   reference's packed params and reference (src/lumen/transport/step.py:129 `operands`). */
int32_t lumen_b200_scene_set_pools(LumenScene* scene, const float* pool_live, const float* pool_ref);
int32_t lumen_b200_scene_destroy(LumenScene* scene);

/* Trace photons first_id .. first_id + n - 1 and add their tallies. Replaces runner.trace + runner.rebuild
   (src/lumen/run.py:693, :534): photon i keyed fold_in(key, first_id + i) (src/lumen/run.py:309). Exactly one of
   rows / source is non-null. stream: a cudaStream_t (null: the default stream). */
int32_t lumen_b200_trace(const LumenScene* scene, const LumenRows* rows, const LumenSource* source,
                         uint32_t key0, uint32_t key1, int64_t first_id, int64_t n, const LumenControls* controls,
                         LumenTallies* out, void* stream);

/* The adjoint: replay photons first_id .. first_id + n - 1 from their keys (no stored path) and add
   grads[p] += sum over events e and sensors s of cotangent[e * n_sensor + s] * d arrival[e, s] / d parameter p.
   Replaces the reverse pass of the reference's custom_jvp rule (src/lumen/api.py:748-787). cotangent, grads:
   device; grads has controls->n_grad doubles. */
int32_t lumen_b200_adjoint(const LumenScene* scene, const LumenRows* rows, const LumenSource* source,
                           uint32_t key0, uint32_t key1, int64_t first_id, int64_t n,
                           const LumenControls* controls, const double* cotangent, int32_t n_events,
                           double* grads, void* stream);

/* The words of the fixed device array lumen_b200_trace_static takes its scratch from (64 x 8 bytes). */
#define LUMEN_STATIC_SCRATCH_WORDS 64
/* The slots of its fixed moment table (16 bytes each: 1 MiB): the photons' per-sensor sums past their first four. */
#define LUMEN_STATIC_MOMENT_SLOTS 65536

/* lumen_b200_trace for callers that cannot allocate device memory during a call. Such callers include a framework
   whose pool owns all of the device's memory and forbids other allocations while it runs a step, and a loop that
   must not wait on the allocator. No counterpart in the reference: lumen's loop allocates through JAX.
   Same arguments, outputs and results as lumen_b200_trace; the caller still passes every input and output. The
   controls' variant and blocks_per_sm pick the launch as there, except that the wavefront (whose slot pool is an
   allocation) runs as the persistent shape 0. With LUMEN_F_ASYNC the call returns once its work is enqueued, and a
   step budget that ran out shows in counts[LUMEN_C_ABORTED]; without it the call waits for the stream and reads
   back the abort flag and the record count. The call's own scratch (4 of LUMEN_STATIC_SCRATCH_WORDS words: the
   photon counter, the abort flag, the step count and the readout groups' record count) comes from one fixed array
   in the library's device memory instead of an allocation, and a call whose scratch would not fit that array is
   refused with LUMEN_ERR_ARG. The photons' sums past their first four sensors go to a fixed moment table of
   LUMEN_STATIC_MOMENT_SLOTS slots; a sum that finds it full is squared alone and counted in
   counts[LUMEN_C_MOMENT_LOST]. Every GPU that loads the library holds both arrays until the process exits. The
   first call on a device looks up the arrays' addresses there, with that device current. All calls share the arrays and leave their contents in them; each call clears what
   must start at zero. Calls that overlap on the GPU (other streams, other host threads) race on the arrays: run
   them one after another. */
int32_t lumen_b200_trace_static(const LumenScene* scene, const LumenRows* rows, const LumenSource* source,
                                uint32_t key0, uint32_t key1, int64_t first_id, int64_t n,
                                const LumenControls* controls, LumenTallies* out, void* stream);

/* Per-photon trace record for parity checks: for each photon, out_i[5*i ..] = vertices, deposits, end code
   (0 alive at the guard, 1 ended), first sensor hit (-1 none), last volume; out_f[4*i ..] = sum of q, final
   weight, final time, sum of q * time. Same inputs as lumen_b200_trace; device outputs. */
int32_t lumen_b200_trace_photons(const LumenScene* scene, const LumenRows* rows, const LumenSource* source,
                                 uint32_t key0, uint32_t key1, int64_t first_id, int64_t n,
                                 const LumenControls* controls, int32_t* out_i, float* out_f, void* stream);

/* Navigator query on a fixed ray set (the geometry hot spot, src/lumen/geometry/navigate.py:663, as the step calls
   it through TrackedGeometry.query, src/lumen/build/tracked.py:86): for ray i, out_i[8*i ..] = hit, vol_before,
   vol_after, cls_before, cls_after, srf, zero, sensor; out_f[4*i ..] = t, normal xyz. vol[i] < 0: located first.
   Device inputs: ray (n * 6: origin, direction), vol, srf (n each); t_max a scalar. */
int32_t lumen_b200_query(const LumenScene* scene, const float* ray, const int32_t* vol, const int32_t* srf,
                         float t_max, int64_t n, int32_t* out_i, float* out_f, void* stream);

/* Volume holding each point (src/lumen/geometry/navigate.py:226 `locate`): device pts (n * 3) -> vol (n). */
int32_t lumen_b200_locate(const LumenScene* scene, const float* pts, int64_t n, int32_t* vol, void* stream);

/* lumen_b200_query and lumen_b200_locate in the navigator's own precision on a float64 scene (LUMEN_PREC_FLOAT64): the
   rays (n * 6), t_max, the points (n * 3) and out_f's t are float64 (out_f: n * 4 doubles, the normal widened from
   the float32 the step reads). A float32 scene refuses them with LUMEN_ERR_ARG, as lumen_b200_query and
   lumen_b200_locate are refused on a float64 scene. */
int32_t lumen_b200_query64(const LumenScene* scene, const double* ray, const int32_t* vol, const int32_t* srf,
                           double t_max, int64_t n, int32_t* out_i, double* out_f, void* stream);
int32_t lumen_b200_locate64(const LumenScene* scene, const double* pts, int64_t n, int32_t* vol, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LUMEN_B200_H */
