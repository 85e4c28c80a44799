"""Tessellated meshes (G4TessellatedSolid; src/lumen/geometry/scene.py:33 Mesh, navigate.py:283-332 the watertight
ray-triangle test and the facet rule, navigator_build.py:266 the chunks) in the checker:

- a query's first mesh hit is the first triangle a float64 brute-force search meets (to 1e-9 with the float64
  navigator, 1e-4 in float32), its normal the triangle's against the ray, its volume the mesh's pseudo-volume;
- a ray starting inside a closed mesh enters it at the facet it meets from behind (the facet rule: a mesh holds no
  point), and no point is located in a mesh;
- a reflection leaves the mesh's triangle without meeting it again (a facet edge is a crease: the next facet may be
  met at a zero step);
- the chunks: at most 8 Morton-ordered triangles each, items of the mesh's mother;
- photons conserve their weight among meshes; a mesh that could hold light (a RINDEX), a mesh sensor or a mesh with
  daughters is refused.
"""

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200 import geometry as G
from lumen_b200 import optics as O
from lumen_b200.detector import build


@pytest.fixture(scope="module")
def det():
    return detectors.mesh_tank()


def _brute(det, o, d):
    """The first triangle hit along each ray (float64 Moller-Trumbore over every triangle): (t, triangle)."""
    T = det.arrays["mesh_tri64"][:, :9].reshape(-1, 3, 3)
    e1, e2 = T[:, 1] - T[:, 0], T[:, 2] - T[:, 0]
    ts, ks = [], []
    for oi, di in zip(o, d, strict=True):
        p = np.cross(np.broadcast_to(di, e2.shape), e2)
        dt = np.einsum("ij,ij->i", e1, p)
        s = oi - T[:, 0]
        u = np.einsum("ij,ij->i", s, p) / dt
        q = np.cross(s, e1)
        v = q @ di / dt
        t = np.einsum("ij,ij->i", e2, q) / dt
        t = np.where((u >= 0) & (v >= 0) & (u + v <= 1) & (t > 0), t, np.inf)
        ts.append(t.min())
        ks.append(int(np.argmin(t)))
    return np.asarray(ts), np.asarray(ks)


def _rays(n, seed=0, lo=-1.4, hi=1.4):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    return o, d / np.linalg.norm(d, axis=1, keepdims=True)


@pytest.mark.parametrize("prec", ["float32", "float64"])
def test_first_mesh_hit_is_the_first_triangle(det, prec):
    dp = det.with_precision(prec)
    o, d = _rays(6000)
    if prec == "float32":
        o, d = o.astype(np.float32).astype(np.float64), d.astype(np.float32).astype(np.float64)
    oi, of = oracle.query(dp, o, d)
    nv, n_mesh = int(det.arrays["n_vol"]), int(det.arrays["n_mesh"])
    m = (oi[:, 2] > nv) & (oi[:, 2] <= nv + n_mesh)
    assert m.sum() > 300
    t, k = _brute(det, o[m], d[m])
    N = det.arrays["mesh_tri64"][k, 9:12]
    nd = np.abs(np.einsum("ij,ij->i", N, d[m]))
    tol = (1e-9 if prec == "float64" else 1e-4) / np.maximum(nd, 0.05)
    assert (np.abs(of[m, 0] - t) < tol).all(), np.max(np.abs(of[m, 0] - t) / tol)
    assert (of[m, 0] <= t + 1e-12).all()  # short of the plane, never past it
    ok = nd > 0.05  # away from grazing: the normal is the triangle's, against the ray
    nrm = of[m, 1:4]
    np.testing.assert_allclose(nrm[ok], -np.sign(np.einsum("ij,ij->i", N, d[m]))[ok, None] * N[ok], atol=1e-5)


def test_rays_inside_a_mesh_enter_it_and_points_are_never_in_one(det):
    ball = int(det.arrays["n_vol"]) + 1
    c = np.array([-0.5, 0.2, 0.1])
    rng = np.random.default_rng(2)
    o = c + rng.uniform(-0.2, 0.2, (500, 3))  # inside the icosphere (r 0.4: its inscribed radius > 0.35)
    d = rng.normal(size=(500, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    assert (oracle.locate(det, o) == 0).all()  # the water box holds them: a mesh holds no point
    oi, of = oracle.query(det, o, d)
    assert (oi[:, 2] == ball).all()
    t, _ = _brute(det, o, d)
    np.testing.assert_allclose(of[:, 0], t, atol=1e-5)


def test_a_reflection_leaves_the_triangle(det):
    o, d = _rays(4000, seed=3)
    o32, d32 = o.astype(np.float32), d.astype(np.float32)
    oi, of = oracle.query(det, o32, d32)
    nv = int(det.arrays["n_vol"])
    m = np.flatnonzero((oi[:, 2] > nv) & (oi[:, 1] == 0))
    assert len(m) > 100
    x = o32[m].astype(np.float64) + of[m, :1].astype(np.float64) * d32[m]
    nrm = of[m, 1:4].astype(np.float64)
    r = d32[m] - 2.0 * np.einsum("ij,ij->i", d32[m], nrm)[:, None] * nrm  # the specular direction
    r /= np.linalg.norm(r, axis=1, keepdims=True)
    oi2, of2 = oracle.query(det, x, r, vol=oi[m, 1], srf=oi[m, 5])
    again = (oi2[:, 5] == oi[m, 5]) & (of2[:, 0] <= 1e-6)
    assert not again.any()  # never the same triangle at a zero step
    # a zero-length event at a crease (the next facet, met within the band at the edge) is the reference's facet rule
    assert (of2[:, 0] > 1e-5).mean() > 0.9


def test_chunks(det):
    a = det.arrays
    ch = a["mesh_chunk"]
    assert (ch[:, 1] >= 1).all() and (ch[:, 1] <= G.MESH_CHUNK).all()
    assert (np.diff(ch[:, 0]) == ch[:-1, 1]).all() and ch[-1, 0] + ch[-1, 1] == len(a["mesh_tri"])
    ch0 = int(a["ch0"])
    assert ch0 == a["n_vol"] + 1 + a["n_mesh"]
    vi = a["vol_i"]
    box = vi[0]
    kids = a["cand"][box[5]:box[5] + box[6]]
    assert set(range(ch0, ch0 + len(ch))) <= set(kids.tolist())  # every chunk an item of the box
    assert (vi[ch0:, 2] == vi[a["n_vol"] + 1 + ch[:, 2], 2]).all()  # a chunk has its mesh's class
    c = G.icosphere(1.0, 1).mean(1)
    code = G.morton(c)
    assert len(np.unique(code)) == len(code)


def test_photons_conserve_their_weight(det):
    n = 1 << 14
    for prec in ("float32", "float64"):
        T = oracle.trace(det.with_precision(prec), A.key_of_seed(1), n, source=sources.Point((0.0, 0.5, -0.6), 1.0,
                         lam=400.0), samples=n, controls=A.controls())[0]  # fmt: skip
        assert abs(T.health[:10].sum() - T.health[10]) < 1e-6 * T.health[10]
        assert T.arrival[0].sum() > 0


def test_meshes_are_refused_where_they_cannot_be():
    mats = {"Water": O.Material("Water", rindex=1.33), "Glass": O.Material("Glass", rindex=1.5),
            "Steel": O.Material("Steel")}  # fmt: skip
    for mesh_mat, kw in (("Glass", {}), ("Steel", {"sensors": {"pmt": "M"}})):
        top = G.Volume("World", G.Box(2, 2, 2), "Water")
        top.place(G.Volume("M", G.Mesh(G.box_mesh(0.2, 0.2, 0.2)), mesh_mat), (0, 0, 0), None, name="M")
        with pytest.raises(ValueError):
            build(top, mats, **kw)
    top = G.Volume("World", G.Box(2, 2, 2), "Water")
    m = G.Volume("M", G.Mesh(G.box_mesh(0.5, 0.5, 0.5)), "Steel")
    m.place(G.Volume("K", G.Box(0.1, 0.1, 0.1), "Water"), (0, 0, 0), None, name="K")
    top.place(m, (0, 0, 0), None, name="M")
    with pytest.raises(ValueError):
        build(top, mats)
