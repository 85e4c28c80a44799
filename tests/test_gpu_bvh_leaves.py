"""BVH leaves of more than one item, as the reference builds them (src/lumen/geometry/bvh.py:18 LEAF_SIZE = 2; every
item of a leaf visited in turn, src/lumen/geometry/navigate.py:440-443 _node).

This package's builder makes a leaf per item, so these tests rebuild a detector's BVHs with the two leaves of every
node whose children are both leaves of consecutive items merged into one leaf of two. The winner of a query does not
depend on the order the items are visited in, and the checker scans the candidate lists without a BVH. Through the
merged BVHs: the query, locate and per-photon kernels (the extended walk over the node arrays, in float32 and float64,
frame groups included) are the checker's bit for bit, and the engine's own trace (the wavefront and the persistent
loop: the float32 walk over the node records) gives the checker's counts and its tallies to their summation order.
"""

import copy

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

pytestmark = pytest.mark.gpu

KEY = A.key_of_seed(0)
NODE0, NODE1 = 7, 8  # vol_i's columns: the volume's daughter BVH, nodes [NODE0, NODE1)


def _two_item_leaves(det):
    """A copy of ``det`` whose BVHs (each volume's and each frame group's) hold two items in a leaf wherever a node's
    two children are leaves of consecutive items: the node becomes that leaf, with its own box."""
    a = dict(det.arrays)
    nf, ni, nf64 = a["node_f"], a["node_i"], a.get("node_f64")
    vol_i, group_i = a["vol_i"].copy(), a["group_i"].copy()
    n = a["n_vol"]
    out_f, out_i, out_f64 = [], [], []

    def emit(nd):
        k = len(out_i)
        out_i.append(None)
        out_f.append(nf[nd])
        if nf64 is not None:
            out_f64.append(nf64[nd])
        cnt = int(ni[nd, 1])
        if cnt > 0:
            row = [0, cnt, int(ni[nd, 2]), 0]
        else:
            lc, rc = nd + 1, int(ni[nd + 1, 0])
            if ni[lc, 1] > 0 and ni[rc, 1] > 0 and ni[rc, 2] == ni[lc, 2] + ni[lc, 1]:
                row = [0, int(ni[lc, 1] + ni[rc, 1]), int(ni[lc, 2]), 0]
            else:
                emit(lc)
                emit(rc)
                row = [0, 0, 0, 0]
        row[0] = len(out_i)  # skip: the node after this subtree
        out_i[k] = row

    trees = [("v", v, int(vol_i[v, NODE0]), int(vol_i[v, NODE1])) for v in range(n + 1)]
    trees += [("g", g, int(group_i[g, 1]), int(group_i[g, 2])) for g in range(len(group_i))]
    for kind, j, n0, n1 in sorted(trees, key=lambda t: (t[2], t[3])):
        start = len(out_i)
        if n0 < n1:
            emit(n0)
            assert int(ni[n0, 0]) == n1, "a range holds one tree"
        if kind == "v":
            vol_i[j, NODE0], vol_i[j, NODE1] = start, len(out_i)
        else:
            group_i[j, 1], group_i[j, 2] = start, len(out_i)
    vol_i[n + 1:, NODE0] = vol_i[n + 1:, NODE1] = len(out_i)
    a["node_f"] = np.asarray(out_f, np.float32).reshape(-1, 6)
    a["node_i"] = np.asarray(out_i, np.int32).reshape(-1, 4)
    if nf64 is not None:
        a["node_f64"] = np.asarray(out_f64, np.float64).reshape(-1, 6)
    a["vol_i"], a["group_i"] = vol_i, group_i
    out = copy.copy(det)
    out.arrays = a
    out.__dict__.pop("_engines", None)
    return out


def _engine(det):
    from lumen_b200 import make as build

    build.build()
    return Engine(det)


def _queries_match(det, n=20000, seed=7):
    f64 = det.precision == "float64"
    rng = np.random.default_rng(seed)
    vf = det.arrays["vol_f64" if f64 else "vol_f"]
    o = rng.uniform(vf[0, 12:15], vf[0, 15:18], (n, 3))
    d = rng.normal(size=(n, 3))
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    if not f64:
        o, d = o.astype(np.float32), d.astype(np.float32)
    eng = _engine(det)
    gi, gf = eng.query(o, d)
    oi, of = oracle.query(det, o, d)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    assert (gi == oi).all(), np.flatnonzero((gi != oi).any(1))[:10]
    u = np.uint64 if f64 else np.uint32
    assert (gf.view(u) == of.view(u)).all()
    assert (eng.locate(o).cpu().numpy() == oracle.locate(det, o)).all()


@pytest.mark.parametrize("which", ["toy", "tank", "wires", "toy64"])
def test_two_item_leaves_queries_bit_exact(which, built):
    det = {"toy": detectors.toy_tank, "tank": detectors.cylinder_tank, "wires": detectors.wire_planes,
           "toy64": lambda: detectors.toy_tank().with_precision("float64")}[which]()  # fmt: skip
    merged = _two_item_leaves(det)
    assert (merged.arrays["node_i"][:, 1] == 2).sum() > 0, "the rebuilt BVHs hold two-item leaves"
    assert len(merged.arrays["node_i"]) < len(det.arrays["node_i"])
    if which == "wires":
        assert merged.arrays["n_group"] > 0  # the frame groups' walk (the extended traversal)
    _queries_match(merged)


def test_two_item_leaves_photons_bit_exact(built):
    """The tank's photons through BVHs of two-item leaves: every per-photon record the checker's bit for bit."""
    tank = _two_item_leaves(detectors.cylinder_tank())
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    n = 1 << 14
    eng = _engine(tank)
    c = A.controls()
    gi, gf = eng.trace_photons(KEY, n, source=DeviceSource(src, n), controls=c)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    _, (oi, of) = oracle.trace(tank, KEY, n, source=src, samples=n, records=True, controls=c)
    bad = np.flatnonzero((gi != oi).any(1) | (gf.view(np.uint32) != of.view(np.uint32)).any(1))
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}"


@pytest.mark.parametrize("variant", [A.VARIANT_WAVEFRONT, 0])
def test_two_item_leaves_traced_tallies_match(variant, built):
    """The engine's own trace (the wavefront and the persistent loop: the float32 walk over the node records) on the
    tank with two-item leaves, and a second event whose photons start elsewhere: the counts are the checker's and the
    FP64 tallies agree to their summation order."""
    tank = _two_item_leaves(detectors.cylinder_tank())
    src = sources.Point(position=[(1.0, -0.5, 2.0), (-3.0, 2.5, -4.0)], n_photons=1.0, lam_range=(300.0, 600.0))
    n = 1 << 15
    c = A.controls(variant=variant)
    eng = _engine(tank)
    ds = DeviceSource(src, n)
    T = DeviceTallies(eng.n_sensor, ds.n_events, 0, 0.0, 1.0, 0)
    eng.trace(KEY, n, source=ds, controls=c, tallies=T)
    O, _ = oracle.trace(tank, KEY, n, source=src, samples=n, controls=c, n_events=ds.n_events)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=1e-9, atol=1e-15)
    np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=1e-9, atol=1e-15)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()
