"""ORACLE (test infrastructure): ctypes access to the CPU restatement in ``oracle/liblumen_oracle.so``.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU baseline import this package, and only as the checker
(or the timed CPU baseline). The product path (``lumen_b200``) never does.
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from lumen_b200 import _abi as A

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liblumen_oracle.so")
_lib = None


def build():
    """Compile the restatement (make)."""
    subprocess.run(["make", "-C", HERE, "-s"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        P = ctypes.POINTER
        L.lumen_oracle_trace.argtypes = [P(A.LumenSceneDesc), A.c_f32p, A.c_f32p, P(A.LumenRows), P(A.LumenSource),
                                         ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64,
                                         P(A.LumenControls), P(A.LumenTallies), A.c_i32p, A.c_f32p, ctypes.c_int32]
        L.lumen_oracle_query.argtypes = [P(A.LumenSceneDesc), A.c_f32p, A.c_i32p, A.c_i32p, ctypes.c_float,
                                         ctypes.c_int64, A.c_i32p, A.c_f32p]
        L.lumen_oracle_locate.argtypes = [P(A.LumenSceneDesc), A.c_f32p, ctypes.c_int64, A.c_i32p]
        L.lumen_oracle_query64.argtypes = [P(A.LumenSceneDesc), A.c_f64p, A.c_i32p, A.c_i32p, ctypes.c_double,
                                           ctypes.c_int64, A.c_i32p, A.c_f64p]
        L.lumen_oracle_locate64.argtypes = [P(A.LumenSceneDesc), A.c_f64p, ctypes.c_int64, A.c_i32p]
        L.lumen_oracle_uniforms.argtypes = [ctypes.c_uint32, ctypes.c_uint32, A.c_i64p, ctypes.c_int64,
                                            ctypes.c_int32, ctypes.c_int32, A.c_f32p]
        L.lumen_oracle_threefry.argtypes = [ctypes.c_uint32] * 4 + [P(ctypes.c_uint32)]
        L.lumen_oracle_math.argtypes = [ctypes.c_int32, A.c_f32p, ctypes.c_int64, A.c_f32p]
        L.lumen_oracle_set_rule_020.argtypes = [ctypes.c_int32]
        L.lumen_oracle_fresnel.argtypes = [A.c_f32p, ctypes.c_int64, A.c_f32p]
        L.lumen_oracle_basis.argtypes = [A.c_f32p, ctypes.c_int64, A.c_f32p]
        L.lumen_oracle_facet_path.argtypes = [ctypes.c_float, A.c_f32p, ctypes.c_uint32, ctypes.c_uint32,
                                              ctypes.c_int64, A.c_f32p, A.c_i64p, A.c_f32p, ctypes.c_float, A.c_f32p,
                                              ctypes.c_int32]  # fmt: skip
        L.lumen_oracle_unified.argtypes = [A.c_f32p, ctypes.c_int32, A.c_f32p, ctypes.c_int64, A.c_f32p]
        L.lumen_oracle_glisur.argtypes = [ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float, A.c_f32p,
                                          A.c_f32p, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int64,
                                          A.c_f32p, A.c_i64p]  # fmt: skip
        L.lumen_oracle_mie.argtypes = [ctypes.c_float] * 3 + [A.c_f32p, ctypes.c_uint32, ctypes.c_uint32,
                                                               ctypes.c_int64, A.c_f32p, A.c_f32p]  # fmt: skip
        L.lumen_oracle_mie_logpdf.argtypes = [ctypes.c_float] * 3 + [A.c_f32p, A.c_f32p, ctypes.c_int64, A.c_f32p]
        L.lumen_oracle_wls.argtypes = [A.c_f32p, A.c_f32p, A.c_f32p, ctypes.c_int32, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_float, ctypes.c_int32, ctypes.c_float, ctypes.c_uint32,
                                       ctypes.c_uint32, ctypes.c_int64, A.c_f32p]  # fmt: skip
        L.lumen_oracle_group_index.argtypes = [A.c_f32p, A.c_f32p, ctypes.c_int32, A.c_f32p, ctypes.c_int64, A.c_f32p]
        L.lumen_oracle_source_rows.argtypes = [P(A.LumenSceneDesc), A.c_f32p, A.c_f32p, P(A.LumenSource), ctypes.c_uint32,
                                               ctypes.c_uint32, ctypes.c_int64, ctypes.c_int64, A.c_f32p, A.c_i32p]
        del vp
        _lib = L
    return _lib


def threefry(k0, k1, x0, x1):
    out = (ctypes.c_uint32 * 2)()
    lib().lumen_oracle_threefry(k0, k1, x0, x1, out)
    return int(out[0]), int(out[1])


def uniforms(key, ids, vertex, n):
    ids = np.ascontiguousarray(ids, np.int64)
    out = np.zeros((len(ids), n), np.float32)
    lib().lumen_oracle_uniforms(key[0], key[1], ids.ctypes.data_as(A.c_i64p), len(ids), vertex, n, A.fptr(out))
    return out


MATH = {"exp": 0, "log": 1, "sin2pi": 2, "cos2pi": 3, "acos": 4, "cbrt": 5, "erfinv": 6, "sin": 7, "cos": 8,
        "dipole_cos": 9, "gaussian": 10}  # fmt: skip


class rule_020:
    """Within the block the checker runs lumen 0.2.0's reference weight at a covered draw of a surface that absorbs
    every photon at the reference (kept as it was; lumen 0.2.1 multiplies it by e / (1 - e)): the rule of the
    reference's published tutorial run."""  # noqa: D205, N801

    def __enter__(self):
        self.was = lib().lumen_oracle_set_rule_020(1)
        return self

    def __exit__(self, *exc):
        lib().lumen_oracle_set_rule_020(self.was)


def math(fn, x):
    x = A.np_f32(x)
    out = np.zeros_like(x)
    A.check(0) if False else None
    st = lib().lumen_oracle_math(MATH[fn], A.fptr(x), x.size, A.fptr(out))
    assert st == 0
    return out


def fresnel(cos_i, n1, n2re, n2im):
    b = np.broadcast_arrays(*(np.asarray(v, np.float32) for v in (cos_i, n1, n2re, n2im)))
    inp = np.ascontiguousarray(np.stack([v.ravel() for v in b], 1), np.float32)
    out = np.zeros((len(inp), 8), np.float32)
    lib().lumen_oracle_fresnel(A.fptr(inp), len(inp), A.fptr(out))
    return out


def basis(n):
    n = A.np_f32(n).reshape(-1, 3)
    out = np.zeros((len(n), 6), np.float32)
    lib().lumen_oracle_basis(A.fptr(n), len(n), A.fptr(out))
    return out[:, :3], out[:, 3:]


def group_index(e, n, lam):
    e, n, lam = A.np_f32(e), A.np_f32(n), A.np_f32(lam)
    out = np.zeros_like(lam)
    assert lib().lumen_oracle_group_index(A.fptr(e), A.fptr(n), len(e), A.fptr(lam), lam.size, A.fptr(out)) == 0
    return out


def facet_path(sigma, wi, n, key=(0, 7), *, sig_live=None, one=False):
    """n unified facet paths off a flat surface (normal +z): (last directions (n, 3), paths that hit a loop bound),
    and with ``sig_live`` also the paths' log densities (n, 3): at sig_live, at sigma, d / d sig_live of the first.
    ``one``: single facet reflections instead of paths."""  # noqa: D205, D209
    from lumen_b200 import facets

    wi = A.np_f32(wi)
    out = np.zeros((n, 3), np.float32)
    capped = np.zeros(1, np.int64)
    U = facets.flat() if sig_live is not None else None
    dens = np.zeros((n, 3), np.float32) if U is not None else None
    assert lib().lumen_oracle_facet_path(sigma, A.fptr(wi), key[0], key[1], n, A.fptr(out),
                                         capped.ctypes.data_as(A.c_i64p), A.fptr(U),
                                         0.0 if sig_live is None else sig_live, A.fptr(dens), int(one)) == 0  # fmt: skip
    return (out, int(capped[0])) if U is None else (out, int(capped[0]), dens)


def unified(fn, inp, U=None):
    """The unified tables and density (lumen_oracle_unified): fn 0 log zeta at y; 1 F at (x, y); 2 log p1 at
    (sigma, w0, n, w1). Returns the values with their derivatives, one row per input."""  # noqa: D205, D209
    from lumen_b200 import facets

    U = facets.flat() if U is None else A.np_f32(U)
    width, nout = {0: (1, 2), 1: (2, 3), 2: (10, 2)}[fn]
    inp = A.np_f32(inp).reshape(-1, width)
    out = np.zeros((len(inp), nout), np.float32)
    assert lib().lumen_oracle_unified(A.fptr(U), fn, A.fptr(inp), len(inp), A.fptr(out)) == 0
    return out


def locate(det, pts):
    """The volume holding each point, in the detector's navigator precision (float64 points on a float64 one)."""
    d, keep = det.desc()
    if det.precision == "float64":
        pts = np.ascontiguousarray(np.asarray(pts, np.float64).reshape(-1, 3))
        vol = np.zeros(len(pts), np.int32)
        st = lib().lumen_oracle_locate64(ctypes.byref(d), A.dptr(pts), len(pts), A.iptr(vol))
        assert st == 0, st
        return vol
    pts = A.np_f32(pts).reshape(-1, 3)
    vol = np.zeros(len(pts), np.int32)
    st = lib().lumen_oracle_locate(ctypes.byref(d), A.fptr(pts), len(pts), A.iptr(vol))
    assert st == 0, st
    return vol


def query(det, o, dvec, vol=None, srf=None, t_max=None):
    """The navigator query per ray (the layout of lumen_b200_query): (out_i (n, 8), out_f (n, 4)); in float64
    (rays, t_max and out_f) on a float64 detector (lumen_b200_query64)."""  # noqa: D205, D209
    d, keep = det.desc()
    f64 = det.precision == "float64"
    dt = np.float64 if f64 else np.float32
    o, dvec = np.asarray(o, dt).reshape(-1, 3), np.asarray(dvec, dt).reshape(-1, 3)
    n = len(o)
    ray = np.ascontiguousarray(np.concatenate([o, dvec], 1), dt)
    vol = np.full(n, -1, np.int32) if vol is None else np.ascontiguousarray(vol, np.int32)
    srf = np.full(n, -1, np.int32) if srf is None else np.ascontiguousarray(srf, np.int32)
    out_i = np.zeros((n, 8), np.int32)
    out_f = np.zeros((n, 4), dt)
    tm = det.arrays["reach"] if t_max is None else t_max
    if f64:
        st = lib().lumen_oracle_query64(ctypes.byref(d), A.dptr(ray), A.iptr(vol), A.iptr(srf), ctypes.c_double(tm),
                                        n, A.iptr(out_i), A.dptr(out_f))  # fmt: skip
    else:
        st = lib().lumen_oracle_query(ctypes.byref(d), A.fptr(ray), A.iptr(vol), A.iptr(srf), ctypes.c_float(tm), n,
                                      A.iptr(out_i), A.fptr(out_f))  # fmt: skip
    assert st == 0, st
    return out_i, out_f


class Tallies:
    """Host FP64 tallies in the LumenTallies layout."""

    def __init__(self, n_sensor, n_events=1, n_bins=0, bin0=0.0, bin_w=1.0, n_grad=0):
        S, E = max(n_sensor, 1), max(n_events, 1)
        self.arrival = np.zeros((E, S))
        self.arrival_t = np.zeros((E, S))
        self.arrival2 = np.zeros((E, S))
        self.hist = np.zeros((E, S, n_bins)) if n_bins else None
        self.jac = np.zeros((E, S, n_grad)) if n_grad else None
        self.health = np.zeros(A.N_HEALTH)
        self.counts = np.zeros(A.N_COUNT, np.uint64)
        t = A.LumenTallies()
        t.n_events, t.n_bins, t.bin0, t.bin_w = E, n_bins, bin0, bin_w
        t.arrival, t.arrival_t, t.arrival2 = A.dptr(self.arrival), A.dptr(self.arrival_t), A.dptr(self.arrival2)
        t.hist = A.dptr(self.hist)
        t.jac = A.dptr(self.jac)
        t.health = A.dptr(self.health)
        t.counts = self.counts.ctypes.data_as(A.c_u64p)
        self.c = t


def host_rows(rows: dict):
    """Return (LumenRows over host arrays, keepalive) of a dict of row arrays (x (n,3), d (n,3), t, lam, w, pol?)."""
    keep = {}
    x, d = A.np_f32(rows["x"]).reshape(-1, 3), A.np_f32(rows["d"]).reshape(-1, 3)
    for i, k in enumerate("xyz"):
        keep[k] = np.ascontiguousarray(x[:, i])
        keep["d" + k] = np.ascontiguousarray(d[:, i])
    for k in ("t", "lam", "w"):
        keep[k] = A.np_f32(rows[k])
    r = A.LumenRows()
    for k in ("x", "y", "z", "dx", "dy", "dz", "t", "lam", "w"):
        setattr(r, k, A.fptr(keep[k]))
    if rows.get("pol") is not None:
        keep["pol"] = A.np_f32(rows["pol"]).reshape(-1, 6)
        r.pol = A.fptr(keep["pol"])
    if rows.get("event") is not None:
        keep["event"] = np.ascontiguousarray(rows["event"], np.int32)
        r.event = A.iptr(keep["event"])
    return r, keep


def host_source(src, samples, det=None):
    """Return (LumenSource over host arrays, keepalive) of a lumen_b200.sources.Source's arrays."""
    a = src.arrays(samples, det)
    keep = {"ev_f": A.np_f32(a["ev_f"]), "ev_first": np.ascontiguousarray(a["ev_first"], np.int64),
            "ev_w": A.np_f32(a["ev_w"])}  # fmt: skip
    s = A.LumenSource()
    s.kind, s.n_events = a["kind"], len(keep["ev_w"])
    s.ev_f, s.ev_first, s.ev_w = A.fptr(keep["ev_f"]), keep["ev_first"].ctypes.data_as(A.c_i64p), A.fptr(keep["ev_w"])
    s.lam0, s.lam1, s.cone_cos = a["lam0"], a["lam1"], a["cone_cos"]
    s.tau1, s.tau2, s.frac1 = a["tau1"], a["tau2"], a["frac1"]
    s.rindex_tab = a.get("rindex_tab", -1)
    if "mat" in a:
        s.mat[:] = [int(v) for v in a["mat"]]
    return s, keep


def trace(det, key, n, *, rows=None, source=None, samples=None, first_id=0, pool_live=None, pool_ref=None,
          controls=None, n_events=1, n_bins=0, bin0=0.0, bin_w=1.0, records=False, threads=0, groups=None,
          deposits=0, truth=False):
    """Trace photons first_id .. first_id + n - 1 on the CPU; return (Tallies, (rec_i, rec_f) or None).

    ``groups``: readout groups ({name: Grid or Group}, lumen_b200.readout): their cells in ``Tallies.groups`` (a host
    GroupCells); ``deposits`` > 0: up to that many deposit records, in photon order and the engine's layout, in
    ``Tallies.deposits`` ((deposits, LUMEN_REC_WORDS) uint32); ``truth``: each photon's analog record in
    ``Tallies.truth`` ((n, LUMEN_TRUTH_WORDS) float32; with LUMEN_F_TRUTH in the controls' flags).
    """
    d, keep = det.desc()
    c = controls or A.controls()
    T = Tallies(det.n_sensor, n_events, n_bins, bin0, bin_w, c.n_grad)
    T.groups = T.deposits = T.truth = None
    if truth:
        T.truth = np.zeros((n, A.TRUTH_WORDS), np.float32)
        T.c.truth = A.fptr(T.truth)
    if groups:
        from lumen_b200.readout import GroupCells

        T.groups = GroupCells(det, groups, n_events)
        T.deposits = np.zeros((deposits, A.REC_WORDS), np.uint32) if deposits else None
        T.groups.attach(T.c, T.deposits, deposits)
    rr, rkeep = host_rows(rows) if rows is not None else (None, None)
    ss, skeep = host_source(source, samples or n, det) if source is not None else (None, None)
    live = None if pool_live is None else A.np_f32(pool_live)
    ref = None if pool_ref is None else A.np_f32(pool_ref)
    rec_i = np.zeros((n, 5), np.int32) if records else None
    rec_f = np.zeros((n, 4), np.float32) if records else None
    st = lib().lumen_oracle_trace(ctypes.byref(d), A.fptr(live), A.fptr(ref),
                                  ctypes.byref(rr) if rr is not None else None,
                                  ctypes.byref(ss) if ss is not None else None, key[0], key[1], first_id, n,
                                  ctypes.byref(c), ctypes.byref(T.c), A.iptr(rec_i), A.fptr(rec_f), threads)
    assert st == 0, f"oracle status {st}"
    return T, ((rec_i, rec_f) if records else None)


def source_rows(source, key, n, first_id=0, samples=None, det=None, pool=None, pool_ref=None):
    """The emission rows of a procedural source (n, 15: x, d, t, lam, w0, er, ei) and their events; ``det`` (and
    ``pool``, the live values: default the detector's) for a Cherenkov segment's medium."""  # noqa: D205, D209
    ss, skeep = host_source(source, samples or n, det)
    d, dkeep = det.desc() if det is not None else (None, None)
    pl = None if pool is None else A.np_f32(pool)
    rf = None if pool_ref is None else A.np_f32(pool_ref)
    out_f = np.zeros((n, 15), np.float32)
    ev = np.zeros(n, np.int32)
    st = lib().lumen_oracle_source_rows(ctypes.byref(d) if d is not None else None, A.fptr(pl), A.fptr(rf), ctypes.byref(ss),
                                        key[0], key[1], first_id, n, A.fptr(out_f), A.iptr(ev))  # fmt: skip
    assert st == 0, f"oracle status {st}"
    return out_f, ev


def mie(gf, gb, ratio, wi, n, key=(0, 9)):
    """n G4OpMieHG draws about wi: (directions (n, 3), their log densities (n,))."""
    wi = A.np_f32(wi)
    out = np.zeros((n, 3), np.float32)
    lp = np.zeros(n, np.float32)
    assert lib().lumen_oracle_mie(gf, gb, ratio, A.fptr(wi), key[0], key[1], n, A.fptr(out), A.fptr(lp)) == 0
    return out, lp


def mie_logpdf(gf, gb, ratio, wi, wo):
    """The Mie log density at directions wo (n, 3) about wi and its derivatives in (gf, gb, ratio): (n, 4)."""
    wi, wo = A.np_f32(wi), A.np_f32(wo).reshape(-1, 3)
    out = np.zeros((len(wo), 4), np.float32)
    assert lib().lumen_oracle_mie_logpdf(gf, gb, ratio, A.fptr(wi), A.fptr(wo), len(wo), A.fptr(out)) == 0
    return out


def wls(energy, s_live, s_ref, lam_in, n, *, yield_live=1.0, yield_ref=1.0, tau=0.0, exponential=False, key=(0, 11)):
    """n G4OpWLS emissions of photons absorbed at lam_in: (n, 4) wavelength, delay, weight, reference weight."""
    e, sl, sr = A.np_f32(energy), A.np_f32(s_live), A.np_f32(s_ref)
    out = np.zeros((n, 4), np.float32)
    assert lib().lumen_oracle_wls(A.fptr(e), A.fptr(sl), A.fptr(sr), len(e), yield_live, yield_ref, tau,
                                  int(exponential), lam_in, key[0], key[1], n, A.fptr(out)) == 0  # fmt: skip
    return out


def glisur(kind, polish, wi, er, *, n1=1.0, n2=1.0, e=0.0, key=(0, 13)):
    """GLISUR facet paths off a flat surface (normal +z): kind "metal" or "dielectric", one per row of er (n, 3) (the
    photons' linear states); e the cover's share (0: Geant4's draw). Returns (last directions (n, 3), far (n,),
    path weights (n,), d/dr of the log weights (n,), paths that hit a loop bound)."""  # noqa: D205, D209
    wi, er = A.np_f32(wi), A.np_f32(er).reshape(-1, 3)
    out = np.zeros((len(er), 6), np.float32)
    capped = np.zeros(1, np.int64)
    assert lib().lumen_oracle_glisur(1 if kind == "metal" else 2, polish, n1, n2, A.fptr(wi), A.fptr(er), e, key[0],
                                     key[1], len(er), A.fptr(out), capped.ctypes.data_as(A.c_i64p)) == 0  # fmt: skip
    return out[:, :3], out[:, 3] > 0.5, out[:, 4], out[:, 5], int(capped[0])
