"""ctypes mirror of the C ABI (include/lumen_b200.h) and the loader of the engine library.

The engine is ``lumen_b200/liblumen_b200.so`` (built in-tree by ``lumen_b200.build``). ``engine()`` loads it and fails
loudly when it is missing: there is no CPU fallback on the product path.
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.environ.get("LUMEN_B200_LIB") or os.path.join(HERE, "liblumen_b200.so")  # a library built elsewhere: env

c_i32p = ctypes.POINTER(ctypes.c_int32)
c_f32p = ctypes.POINTER(ctypes.c_float)
c_i64p = ctypes.POINTER(ctypes.c_int64)
c_f64p = ctypes.POINTER(ctypes.c_double)
c_u64p = ctypes.POINTER(ctypes.c_uint64)

MAX_GRAD = 8
N_COL = 10
N_HEALTH = 11
N_COUNT = 8
C_PHOTONS, C_STEPS, C_DEPOSITS, C_TRUNCATED, C_MULTI, C_ABORTED, C_RECORDS, C_MOMENT_LOST = range(8)  # LUMEN_C_*
ERR_ARG, ERR_CUDA, ERR_SCENE, ERR_STEP_BUDGET, ERR_NO_DEVICE, ERR_NOT_SUPPORTED, ERR_RECORDS = range(1, 8)
MAX_AXES = 4
MAX_GROUPS = 8
REC_WORDS = 20
F_ASYNC = 1
F_REACH = 2
F_JUMP = 4
F_TRUTH = 8
TRUTH_WORDS = 8
N_VARIANT = 4
VARIANT_WAVEFRONT = 3
UNI_NX, UNI_NY = 257, 69
UNI_WORDS = 4 * UNI_NX * UNI_NY + 2 * UNI_NY
HEALTH = ("lost", "abandoned", "escaped", "distance_cut", "absorbed_bulk", "absorbed_surface", "rouletted",
          "reweighted", "truncated", "pushed", "start")  # fmt: skip
COUNTS = ("photons", "steps", "deposits", "truncated", "multi", "aborted", "records", "moment_lost")
FEATURES = ("wavelength", "theta", "cos_incidence", "generation", "x", "y", "z", "rho")  # LUMEN_FEAT_* order
SRC_POINT, SRC_TRACK, SRC_SCINT, SRC_CHERENKOV, SRC_SCINT_MATERIAL = 0, 1, 2, 3, 4
SM_N, SM_SEGMENT, SM_RISES, SM_YIELD, SM_SPEC, SM_TAU, SM_RISE, SM_SHARE, SM_WORDS = 0, 1, 2, 3, 4, 7, 10, 13, 16
EV_F = 12


class LumenSceneDesc(ctypes.Structure):
    _fields_ = [
        ("n_vol", ctypes.c_int32), ("n_kind", ctypes.c_int32), ("n_leaf", ctypes.c_int32),
        ("n_plane", ctypes.c_int32), ("n_prog", ctypes.c_int32), ("n_node", ctypes.c_int32),
        ("n_item", ctypes.c_int32), ("n_cand", ctypes.c_int32),
        ("vol_i", c_i32p), ("vol_f", c_f32p), ("cand", c_i32p), ("node_f", c_f32p), ("node_i", c_i32p),
        ("items", c_i32p), ("kind_i", c_i32p), ("leaf_f", c_f32p), ("leaf_i", c_i32p), ("plane_f", c_f32p),
        ("prog_i", c_i32p), ("reach", ctypes.c_float),
        ("n_cls", ctypes.c_int32), ("n_med", ctypes.c_int32), ("n_row", ctypes.c_int32), ("n_tab", ctypes.c_int32),
        ("n_pool", ctypes.c_int32), ("n_sensor", ctypes.c_int32),
        ("cls_medium", c_i32p), ("row_of", c_i32p), ("med_i", c_i32p), ("row_i", c_i32p), ("tab", c_i32p),
        ("pool", c_f32p), ("unified", c_f32p),
        ("n_comp", ctypes.c_int32), ("n_fnode", ctypes.c_int32), ("comp", c_i32p), ("comp_box", c_f32p),
        ("fnode_f", c_f32p), ("fnode_i", c_i32p),
        ("n_jump", ctypes.c_int32), ("jump_f", c_f32p), ("jump_i", c_i32p), ("n_clear", ctypes.c_int64),
        ("clear", c_f32p),
        ("precision", ctypes.c_int32), ("vol_f64", c_f64p), ("node_f64", c_f64p), ("leaf_f64", c_f64p),
        ("plane_f64", c_f64p),
        ("n_mesh", ctypes.c_int32), ("n_chunk", ctypes.c_int32), ("n_tri", ctypes.c_int32), ("mesh_tri", c_f32p),
        ("mesh_tri64", c_f64p), ("mesh_chunk", c_i32p), ("chunk_box", c_f32p), ("chunk_box64", c_f64p),
        ("n_group", ctypes.c_int32), ("group_i", c_i32p), ("group_r", c_f32p), ("group_r64", c_f64p),
        ("cls_born", c_i32p), ("pair_pre", c_i32p),
    ]  # fmt: skip


class LumenRows(ctypes.Structure):
    _fields_ = [("x", c_f32p), ("y", c_f32p), ("z", c_f32p), ("dx", c_f32p), ("dy", c_f32p), ("dz", c_f32p),
                ("t", c_f32p), ("lam", c_f32p), ("w", c_f32p), ("pol", c_f32p), ("event", c_i32p)]  # fmt: skip


class LumenSource(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("n_events", ctypes.c_int32), ("ev_f", c_f32p), ("ev_first", c_i64p),
                ("ev_w", c_f32p), ("lam0", ctypes.c_float), ("lam1", ctypes.c_float), ("cone_cos", ctypes.c_float),
                ("tau1", ctypes.c_float), ("tau2", ctypes.c_float), ("frac1", ctypes.c_float),
                ("rindex_tab", ctypes.c_int32), ("reserved", ctypes.c_int32), ("mat", ctypes.c_int32 * 16)]  # fmt: skip


class LumenControls(ctypes.Structure):
    _fields_ = [("max_distance", ctypes.c_float), ("roulette", ctypes.c_float), ("max_vertices", ctypes.c_int32),
                ("n_grad", ctypes.c_int32), ("grad_tab", ctypes.c_int32 * MAX_GRAD),
                ("step_budget", ctypes.c_int64), ("flags", ctypes.c_int32), ("variant", ctypes.c_int32),
                ("blocks_per_sm", ctypes.c_int32), ("wave_slots_log2", ctypes.c_int32),
                ("wave_rounds", ctypes.c_int32)]  # fmt: skip


class LumenAxis(ctypes.Structure):
    _fields_ = [("feature", ctypes.c_int32), ("n", ctypes.c_int32), ("knots", ctypes.c_int32),
                ("reserved", ctypes.c_int32), ("values", c_f32p)]  # fmt: skip


class LumenGroup(ctypes.Structure):
    _fields_ = [("n_axes", ctypes.c_int32), ("n_delay", ctypes.c_int32), ("nt", ctypes.c_int32),
                ("weighted", ctypes.c_int32), ("normalise", ctypes.c_int32), ("n_sensors", ctypes.c_int32),
                ("t0", ctypes.c_float), ("dt", ctypes.c_float), ("axes", LumenAxis * MAX_AXES),
                ("index", c_i32p), ("weights", c_f32p), ("charge", c_f64p), ("charge2", c_f64p), ("time", c_f64p),
                ("over_q", c_f64p), ("over_qt", c_f64p)]  # fmt: skip


class LumenTallies(ctypes.Structure):
    _fields_ = [("n_events", ctypes.c_int32), ("n_bins", ctypes.c_int32), ("bin0", ctypes.c_float),
                ("bin_w", ctypes.c_float), ("arrival", c_f64p), ("arrival_t", c_f64p), ("arrival2", c_f64p),
                ("hist", c_f64p), ("jac", c_f64p), ("health", c_f64p), ("counts", c_u64p),
                ("n_groups", ctypes.c_int32), ("reserved", ctypes.c_int32), ("groups", ctypes.POINTER(LumenGroup)),
                ("pe2", c_f64p), ("records", ctypes.c_void_p), ("rec_capacity", ctypes.c_int64),
                ("truth", c_f32p)]  # fmt: skip


def iptr(a):
    return a.ctypes.data_as(c_i32p) if a is not None and a.size else ctypes.cast(None, c_i32p)


def fptr(a):
    return a.ctypes.data_as(c_f32p) if a is not None and a.size else ctypes.cast(None, c_f32p)


def dptr(a):
    return a.ctypes.data_as(c_f64p) if a is not None and a.size else ctypes.cast(None, c_f64p)


def controls(max_distance=0.0, roulette=0.01, max_vertices=1 << 22, grad_tabs=(), step_budget=0, flags=0, variant=0,
             blocks_per_sm=0, wave_slots_log2=0, wave_rounds=0):
    c = LumenControls()
    c.flags, c.variant, c.blocks_per_sm = int(flags), int(variant), int(blocks_per_sm)
    c.wave_slots_log2, c.wave_rounds = int(wave_slots_log2), int(wave_rounds)
    c.max_distance = float(max_distance)
    c.roulette = float(roulette)
    c.max_vertices = int(max_vertices)
    if len(grad_tabs) > MAX_GRAD:
        raise ValueError(f"at most {MAX_GRAD} gradient parameters")
    c.n_grad = len(grad_tabs)
    for i, t in enumerate(grad_tabs):
        c.grad_tab[i] = int(t)
    c.step_budget = int(step_budget)
    return c


ENTRY_POINTS = ("lumen_b200_abi_version", "lumen_b200_last_error", "lumen_b200_last_launches",
                "lumen_b200_scene_create", "lumen_b200_scene_set_pools", "lumen_b200_scene_destroy", "lumen_b200_trace",
                "lumen_b200_adjoint", "lumen_b200_trace_photons", "lumen_b200_query", "lumen_b200_locate", "lumen_b200_trace_static",
                "lumen_b200_query64", "lumen_b200_locate64")  # fmt: skip

_lib = None


def engine():
    """Return the loaded engine library (ctypes); raise if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise RuntimeError(f"the CUDA engine {LIB} is not built: run `python -c 'import __graft_entry__ as g; "
                               "g.build()'` (there is no CPU fallback)")  # fmt: skip
        lib = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        lib.lumen_b200_abi_version.restype = ctypes.c_int32
        lib.lumen_b200_last_error.restype = ctypes.c_char_p
        lib.lumen_b200_last_launches.restype = ctypes.c_int64
        lib.lumen_b200_scene_create.argtypes = [ctypes.POINTER(LumenSceneDesc), ctypes.POINTER(vp)]
        lib.lumen_b200_scene_set_pools.argtypes = [vp, c_f32p, c_f32p]
        lib.lumen_b200_scene_destroy.argtypes = [vp]
        lib.lumen_b200_trace.argtypes = [vp, ctypes.POINTER(LumenRows), ctypes.POINTER(LumenSource), ctypes.c_uint32,
                                         ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64,
                                         ctypes.POINTER(LumenControls), ctypes.POINTER(LumenTallies), vp]  # fmt: skip
        lib.lumen_b200_adjoint.argtypes = [vp, ctypes.POINTER(LumenRows), ctypes.POINTER(LumenSource),
                                           ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64,
                                           ctypes.POINTER(LumenControls), c_f64p, ctypes.c_int32, c_f64p, vp]  # fmt: skip
        lib.lumen_b200_trace_static.argtypes = [vp, ctypes.POINTER(LumenRows), ctypes.POINTER(LumenSource),
                                                ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64,
                                                ctypes.POINTER(LumenControls), ctypes.POINTER(LumenTallies), vp]
        lib.lumen_b200_trace_photons.argtypes = [vp, ctypes.POINTER(LumenRows), ctypes.POINTER(LumenSource),
                                                 ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64,
                                                 ctypes.POINTER(LumenControls), c_i32p, c_f32p, vp]  # fmt: skip
        lib.lumen_b200_query.argtypes = [vp, c_f32p, c_i32p, c_i32p, ctypes.c_float, ctypes.c_int64, c_i32p, c_f32p,
                                         vp]  # fmt: skip
        lib.lumen_b200_locate.argtypes = [vp, c_f32p, ctypes.c_int64, c_i32p, vp]
        lib.lumen_b200_query64.argtypes = [vp, c_f64p, c_i32p, c_i32p, ctypes.c_double, ctypes.c_int64, c_i32p,
                                           c_f64p, vp]  # fmt: skip
        lib.lumen_b200_locate64.argtypes = [vp, c_f64p, ctypes.c_int64, c_i32p, vp]
        for name in ENTRY_POINTS[3:]:
            getattr(lib, name).restype = ctypes.c_int32
        _lib = lib
    return _lib


class EngineError(RuntimeError):
    """A non-zero status of the engine (``code``: LUMEN_ERR_*)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"lumen_b200 status {code}: {msg}")
        self.code = code


class RecordsOverflow(EngineError):
    """The deposit records outgrew the scratch (LUMEN_ERR_RECORDS; src/lumen/run.py:236 RecordsOverflow)."""


class StepBudgetExhausted(EngineError):
    """The call's device step budget ran out before every photon ended (LUMEN_ERR_STEP_BUDGET): the kernel stopped
    handing out photons and returned; the tallies hold the photons that ended before it."""  # noqa: D205, D209


def check(status: int):
    """Raise the engine's error for a non-zero status."""
    if status != 0:
        msg = engine().lumen_b200_last_error().decode(errors="replace")
        cls = {ERR_RECORDS: RecordsOverflow, ERR_STEP_BUDGET: StepBudgetExhausted}.get(status, EngineError)
        raise cls(status, msg)


def key_of_seed(seed: int):
    """Return jax.random.PRNGKey(seed)'s key data for a 32-bit seed: (0, seed) (threefry_seed)."""
    s = int(seed)
    return (s >> 32) & 0xFFFFFFFF, s & 0xFFFFFFFF


def np_f32(a):
    return np.ascontiguousarray(a, np.float32)
