"""Detector geometry on the host: solids lowered to quadric / plane leaves, placed volumes, and the navigator arrays.

A solid is lowered, as lumen lowers the GDML solid catalogue (src/lumen/geometry/solids.py, csg_build.py), to *leaves*
(a quadric piece {y^T A y + 2 b.y + c <= 0}, y = x - oq, intersected with a slab of planes {n.(x - og) <= h}) and a
postfix boolean program over them (op 0 pushes a leaf, 1 union, 2 intersection, 3 subtraction). Every solid then runs
the same instructions on different data (src/lumen/geometry/csg.py module docstring). The layout of the flattened
arrays is the C ABI's (include/lumen_b200.h): volume records, daughter lists, a BVH per volume over its daughters'
world boxes (depth-first, skip pointers, one item per leaf), kinds, leaves, planes and programs.

Scope: boxes, tubes (full phi, optional inner radius), spheres (full, or a hemisphere in z), and their unions,
subtractions and intersections with a placement of the second operand; volumes nest in a tree (daughters inside their
mother, siblings disjoint or touching).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

# the navigator's padded world boxes (src/lumen/rules/tolerances.py:83-84)
WORLD_BOX_PAD_REL = 1e-6
WORLD_BOX_PAD_ABS = 1e-9
MAX_LEAVES = 8  # include/lumen_b200.h LUMEN_MAX_LEAVES
MAX_BVH_DEPTH = 24  # include/lumen_b200.h LUMEN_MAX_BVH_DEPTH
MAX_PLANES = 8


# ------------------------------------------------------------------------------------------------------ leaves
@dataclass
class Leaf:
    """One leaf in its solid's frame: optional quadric (A, b, c about oq) and planes n.(x - og) <= h."""

    has_q: bool
    A: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))
    b: np.ndarray = field(default_factory=lambda: np.zeros(3))
    c: float = 0.0
    oq: np.ndarray = field(default_factory=lambda: np.zeros(3))
    og: np.ndarray = field(default_factory=lambda: np.zeros(3))
    N: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    H: np.ndarray = field(default_factory=lambda: np.zeros(0))

    def moved(self, R: np.ndarray, p: np.ndarray) -> Leaf:
        """Return the leaf placed by x' = R x + p (its frame rotated and shifted)."""
        return Leaf(self.has_q, R @ self.A @ R.T, R @ self.b, self.c, R @ self.oq + p, R @ self.og + p,
                    self.N @ R.T, self.H.copy())  # fmt: skip


@dataclass
class Lowered:
    """A solid as leaves, a postfix program over them and a bounding box (lo, hi) in its frame."""

    leaves: list
    program: list  # [(op, arg)]
    lo: np.ndarray
    hi: np.ndarray


class Solid:
    """A solid (local frame, metres); ``lower()`` gives its leaves and program."""

    def lower(self) -> Lowered:  # pragma: no cover - abstract
        raise NotImplementedError


def _slab_planes(hx, hy, hz):
    N = np.array([[1, 0, 0], [-1, 0, 0], [0, 1, 0], [0, -1, 0], [0, 0, 1], [0, 0, -1]], float)
    H = np.array([hx, hx, hy, hy, hz, hz], float)
    return N, H


@dataclass
class Box(Solid):
    """G4Box: half lengths (m)."""

    hx: float
    hy: float
    hz: float

    def lower(self):
        N, H = _slab_planes(self.hx, self.hy, self.hz)
        h = np.array([self.hx, self.hy, self.hz])
        return Lowered([Leaf(False, N=N, H=H)], [(0, 0)], -h, h)


@dataclass
class Tube(Solid):
    """G4Tubs with a full phi range: radii and half length (m)."""

    rmax: float
    dz: float
    rmin: float = 0.0

    def lower(self):
        A = np.diag([1.0, 1.0, 0.0])
        N = np.array([[0, 0, 1.0], [0, 0, -1.0]])
        H = np.array([self.dz, self.dz])
        outer = Leaf(True, A=A, c=-self.rmax**2, N=N, H=H)
        h = np.array([self.rmax, self.rmax, self.dz])
        if self.rmin <= 0.0:
            return Lowered([outer], [(0, 0)], -h, h)
        inner = Leaf(True, A=A.copy(), c=-self.rmin**2)
        return Lowered([outer, inner], [(0, 0), (0, 1), (3, 0)], -h, h)


@dataclass
class Sphere(Solid):
    """G4Sphere with a full phi range; ``hemisphere``: 0 full, +1 the z >= 0 half (theta in [0, pi/2]), -1 z <= 0."""

    rmax: float
    hemisphere: int = 0

    def lower(self):
        A = np.eye(3)
        r = self.rmax
        if self.hemisphere == 0:
            return Lowered([Leaf(True, A=A, c=-r * r)], [(0, 0)], -np.full(3, r), np.full(3, r))
        s = float(np.sign(self.hemisphere))
        leaf = Leaf(True, A=A, c=-r * r, N=np.array([[0.0, 0.0, -s]]), H=np.array([0.0]))
        lo, hi = -np.full(3, r), np.full(3, r)
        if s > 0:
            lo[2] = 0.0
        else:
            hi[2] = 0.0
        return Lowered([leaf], [(0, 0)], lo, hi)


@dataclass
class Boolean(Solid):
    """G4UnionSolid / G4SubtractionSolid / G4IntersectionSolid: ``a op (b placed at (rot, pos) in a's frame)``."""

    op: str  # "union", "subtraction", "intersection"
    a: Solid
    b: Solid
    pos: tuple = (0.0, 0.0, 0.0)
    rot: np.ndarray | None = None

    def lower(self):
        la, lb = self.a.lower(), self.b.lower()
        R = np.eye(3) if self.rot is None else np.asarray(self.rot, float)
        p = np.asarray(self.pos, float)
        moved = [lf.moved(R, p) for lf in lb.leaves]
        k = len(la.leaves)
        prog = list(la.program) + [(op, arg + k) if op == 0 else (op, arg) for op, arg in lb.program]
        prog.append(({"union": 1, "intersection": 2, "subtraction": 3}[self.op], 0))
        blo, bhi = _box_corners(lb.lo, lb.hi, R, p)
        if self.op == "union":
            lo, hi = np.minimum(la.lo, blo), np.maximum(la.hi, bhi)
        elif self.op == "intersection":
            lo, hi = np.maximum(la.lo, blo), np.minimum(la.hi, bhi)
        else:
            lo, hi = la.lo, la.hi
        return Lowered(la.leaves + moved, prog, lo, hi)


def _box_corners(lo, hi, R, t):
    """Return the axis-aligned box of the box (lo, hi) placed by x' = R x + t."""
    c = np.array([[x, y, z] for x in (lo[0], hi[0]) for y in (lo[1], hi[1]) for z in (lo[2], hi[2])])
    w = c @ R.T + t
    return w.min(0), w.max(0)


def rotation(axis: str, degrees: float) -> np.ndarray:
    """Return the rotation matrix about x, y or z by ``degrees``."""
    a = math.radians(degrees)
    c, s = math.cos(a), math.sin(a)
    return {
        "x": np.array([[1, 0, 0], [0, c, -s], [0, s, c]]),
        "y": np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]]),
        "z": np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]]),
    }[axis]


def gdml_rotation(x=0.0, y=0.0, z=0.0) -> np.ndarray:
    """Return the rotation of a GDML physvol ``<rotation x y z>`` (degrees): G4's frame rotation, inverted.

    G4GDMLReadStructure builds rot.rotateX(x).rotateY(y).rotateZ(z) = Rz Ry Rx and places the daughter with its
    inverse: the daughter's local axes in the mother are R = (Rz Ry Rx)^-1.
    """
    Rf = rotation("z", z) @ rotation("y", y) @ rotation("x", x)
    return Rf.T


# ------------------------------------------------------------------------------------------------------ volumes
@dataclass
class Volume:
    """A logical volume: a solid of a material, with placed daughters."""

    name: str
    solid: Solid
    material: str
    daughters: list = field(default_factory=list)

    def place(self, vol: Volume, pos=(0.0, 0.0, 0.0), rot=None, name=None, copy=0):
        """Place ``vol`` inside this volume at ``pos`` (m) with rotation ``rot`` (3x3; daughter local -> mother)."""
        self.daughters.append(Placement(vol, np.asarray(pos, float), np.eye(3) if rot is None else np.asarray(rot, float),
                                        name or f"{vol.name}_{len(self.daughters)}", copy))  # fmt: skip
        return self


@dataclass
class Placement:
    volume: Volume
    pos: np.ndarray
    rot: np.ndarray
    name: str
    copy: int = 0


@dataclass
class Placed:
    """One placed volume (a navigator volume): its path, logical volume, world pose and parent index."""

    name: str
    lv: Volume
    R: np.ndarray
    t: np.ndarray
    parent: int
    depth: int


def flatten(top: Volume, top_name: str = None) -> list:
    """Return the placed volumes of the tree under ``top`` (placed at the origin), depth first: parents first."""
    out = []

    def walk(lv, name, R, t, parent, depth):
        i = len(out)
        out.append(Placed(name, lv, R, t, parent, depth))
        for pl in lv.daughters:
            walk(pl.volume, pl.name, R @ pl.rot, R @ pl.pos + t, i, depth + 1)

    walk(top, top_name or top.name, np.eye(3), np.zeros(3), -1, 0)
    return out


# ------------------------------------------------------------------------------------------------------ BVH
def _bvh(items, lo, hi):
    """Return the BVH over items (their boxes lo[i], hi[i]) as (node_lo, node_hi, skip, count, start, order):
    depth first, a leaf per item, median split on the longest axis of the centroids."""  # noqa: D205
    nodes = []  # [lo, hi, skip, count, start]
    order = []

    def build(ids):
        k = len(nodes)
        nodes.append(None)
        blo, bhi = lo[ids].min(0), hi[ids].max(0)
        if len(ids) == 1:
            nodes[k] = [blo, bhi, 0, 1, len(order)]
            order.append(ids[0])
        else:
            cen = 0.5 * (lo[ids] + hi[ids])
            ax = int(np.argmax(cen.max(0) - cen.min(0)))
            srt = ids[np.argsort(cen[:, ax], kind="stable")]
            m = len(srt) // 2
            build(srt[:m])
            build(srt[m:])
            nodes[k] = [blo, bhi, 0, 0, 0]
        nodes[k][2] = len(nodes)  # skip: the node after this subtree
        return k

    if len(items):
        build(np.asarray(items))
    return nodes, order


def bvh_depth(node_i, n0, n1) -> int:
    """Return the levels of the BVH in nodes [n0, n1) (0: empty)."""
    if n0 >= n1:
        return 0
    depth, todo = 0, [(n0, 1)]
    while todo:
        nd, dp = todo.pop()
        depth = max(depth, dp)
        if node_i[nd, 1] == 0:
            todo += [(nd + 1, dp + 1), (int(node_i[nd + 1, 0]), dp + 1)]
    return depth


# ------------------------------------------------------------------------------------------------ sensor reach
BAND_ULPS_EPS = 8.0 * 2.0**-23  # the navigator's band: BAND_ULPS float32 ulps of the coordinate scale, plus a floor
BAND_FLOOR = 1e-9
K_ON = 4.0


def reach_arrays(arrays) -> dict:
    """Return the arrays that let a bulk step's query stop just past its free path (src/lumen/geometry/reach.py:66
    ``build``): per volume its COMPONENT (the volumes joined to it by crossings without a vertex: a parent and a
    daughter of one class), each component's box (the union of its members' padded world boxes), and a skip-pointer
    tree over every sensor volume's box; the component and sensor boxes padded by the contact tolerance at the scene's
    scale (K_ON bands). The outside has no component (-1).
    """
    vol_i, vol_f = arrays["vol_i"], np.asarray(arrays["vol_f"], np.float64)
    n = int(arrays["n_vol"])
    parent, cls, sensor = vol_i[:n, 1], vol_i[:, 2], vol_i[:n, 3]
    root = list(range(n))

    def find(a):
        while root[a] != a:
            root[a] = root[root[a]]
            a = root[a]
        return a

    for v in range(n):
        p = int(parent[v])
        if p < n and cls[v] == cls[p]:
            ra, rb = find(v), find(p)
            if ra != rb:
                root[rb] = ra
    roots = [find(v) for v in range(n)]
    uniq, comp = np.unique(np.asarray(roots, np.int64), return_inverse=True) if n else (np.zeros(0), np.zeros(0))
    lo_w, hi_w = vol_f[:n, 12:15], vol_f[:n, 15:18]
    scale = float(np.max(np.abs(np.concatenate([lo_w, hi_w])))) if n else 1.0
    pad = K_ON * (BAND_ULPS_EPS * scale + BAND_FLOOR)
    c_lo = np.full((len(uniq), 3), np.inf)
    c_hi = np.full((len(uniq), 3), -np.inf)
    np.minimum.at(c_lo, comp, lo_w)
    np.maximum.at(c_hi, comp, hi_w)
    sv = np.flatnonzero(sensor >= 0)
    f_lo, f_hi = lo_w - pad, hi_w + pad
    nodes, _ = _bvh(sv.astype(np.int64), f_lo, f_hi)
    fnode_f = np.asarray([[*nd[0], *nd[1]] for nd in nodes], np.float32).reshape(-1, 6)
    fnode_i = np.asarray([[nd[2], nd[3], 0, 0] for nd in nodes], np.int32).reshape(-1, 4)
    return dict(comp=np.append(comp, -1).astype(np.int32),
                comp_box=np.concatenate([c_lo - pad, c_hi + pad], 1).astype(np.float32).reshape(-1, 6),
                fnode_f=fnode_f, fnode_i=fnode_i)  # fmt: skip


# ------------------------------------------------------------------------------------------------- the arrays
def pad_box(lo, hi):
    """Return the box padded as the navigator's world boxes (tolerances.py:83-84)."""
    c, h = 0.5 * (lo + hi), 0.5 * (hi - lo)
    pad = WORLD_BOX_PAD_REL * (np.abs(c) + h) + WORLD_BOX_PAD_ABS
    return lo - pad, hi + pad


def navigator_arrays(placed: list, vol_cls, outside_cls: int, vol_sensor, prio=None) -> dict:
    """Return the navigator's flat arrays (include/lumen_b200.h layouts) of the placed volumes."""
    n = len(placed)
    kinds, kind_of = [], {}
    for p in placed:
        key = id(p.lv.solid)
        if key not in kind_of:
            kind_of[key] = len(kinds)
            kinds.append(p.lv.solid.lower())
    # kinds -> leaf / plane / program tables
    kind_i, leaf_f, leaf_i, plane_f, prog_i = [], [], [], [], []
    for low in kinds:
        if len(low.leaves) > MAX_LEAVES:
            raise ValueError(f"a solid of {len(low.leaves)} leaves: at most {MAX_LEAVES}")
        kind_i.append([len(leaf_f), len(low.leaves), len(prog_i), len(low.program)])
        for lf in low.leaves:
            if lf.N.shape[0] > MAX_PLANES:
                raise ValueError(f"a leaf of {lf.N.shape[0]} planes: at most {MAX_PLANES}")
            sa = float(np.max(np.abs(lf.A))) if lf.has_q else 0.0
            leaf_f.append(np.concatenate([lf.og, lf.oq, lf.A.ravel(), lf.b, [lf.c, sa]]))
            leaf_i.append([1 if lf.has_q else 0, len(plane_f), lf.N.shape[0], 0])
            for nn, hh in zip(lf.N, lf.H, strict=True):
                plane_f.append([*nn, hh])
        prog_i.extend([list(x) for x in low.program])
    # volumes
    vol_f = np.zeros((n, 18), np.float64)
    lo_w, hi_w = np.zeros((n, 3)), np.zeros((n, 3))
    for i, p in enumerate(placed):
        low = kinds[kind_of[id(p.lv.solid)]]
        blo, bhi = _box_corners(low.lo, low.hi, p.R, p.t)
        blo, bhi = pad_box(blo, bhi)
        lo_w[i], hi_w[i] = blo, bhi
        vol_f[i, 0:9] = p.R.ravel()
        vol_f[i, 9:12] = p.t
        vol_f[i, 12:15] = blo
        vol_f[i, 15:18] = bhi
    kids = [[] for _ in range(n + 1)]
    for i, p in enumerate(placed):
        kids[p.parent if p.parent >= 0 else n].append(i)
    prio = np.arange(n + 1) if prio is None else np.asarray(prio)
    vol_i = np.zeros((n + 1, 10), np.int32)
    cand, node_f, node_i, items = [], [], [], []
    for v in range(n + 1):
        ks = kids[v]
        vol_i[v, 0] = kind_of[id(placed[v].lv.solid)] if v < n else -1
        vol_i[v, 1] = (placed[v].parent if placed[v].parent >= 0 else n) if v < n else -1
        vol_i[v, 2] = vol_cls[v] if v < n else outside_cls
        vol_i[v, 3] = vol_sensor[v] if v < n else -1
        vol_i[v, 4] = prio[v]
        vol_i[v, 5], vol_i[v, 6] = len(cand), len(ks)
        cand.extend(ks)
        # the daughters' BVH, in the float32 boxes the engine reads
        lo32 = lo_w.astype(np.float32).astype(np.float64)
        hi32 = hi_w.astype(np.float32).astype(np.float64)
        nodes, order = _bvh(np.asarray(ks, np.int64), lo32, hi32)
        base, ibase = len(node_f), len(items)
        vol_i[v, 7] = base
        for nd in nodes:
            node_f.append([*nd[0], *nd[1]])
            node_i.append([base + nd[2], nd[3], ibase + nd[4] if nd[3] else 0, 0])
        items.extend(order)
        vol_i[v, 8] = len(node_f)
    ni_arr = np.asarray(node_i, np.int32).reshape(-1, 4)
    for v in range(n + 1):
        if bvh_depth(ni_arr, vol_i[v, 7], vol_i[v, 8]) > MAX_BVH_DEPTH:
            raise ValueError(f"volume {v}: a daughter BVH deeper than {MAX_BVH_DEPTH} levels")
    allp = np.concatenate([lo_w, hi_w]) if n else np.zeros((1, 3))
    reach = float(np.linalg.norm(allp.max(0) - allp.min(0)))
    return dict(
        n_vol=n, vol_i=vol_i, vol_f=vol_f.astype(np.float32), cand=np.asarray(cand, np.int32),
        node_f=np.asarray(node_f, np.float32).reshape(-1, 6), node_i=np.asarray(node_i, np.int32).reshape(-1, 4),
        items=np.asarray(items, np.int32), kind_i=np.asarray(kind_i, np.int32).reshape(-1, 4),
        leaf_f=np.asarray(leaf_f, np.float32).reshape(-1, 20), leaf_i=np.asarray(leaf_i, np.int32).reshape(-1, 4),
        plane_f=np.asarray(plane_f, np.float32).reshape(-1, 4), prog_i=np.asarray(prog_i, np.int32).reshape(-1, 2),
        reach=reach, names=[p.name for p in placed],
    )  # fmt: skip
