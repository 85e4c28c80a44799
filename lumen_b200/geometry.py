"""Detector geometry on the host: solids lowered to quadric / plane leaves, placed volumes, and the navigator arrays.

A solid is lowered, as lumen lowers the GDML solid catalogue (src/lumen/geometry/solids.py, csg_build.py), to *leaves*
(a quadric piece {y^T A y + 2 b.y + c <= 0}, y = x - oq, intersected with a slab of planes {n.(x - og) <= h}) and a
postfix boolean program over them (op 0 pushes a leaf, 1 union, 2 intersection, 3 subtraction). Every solid then runs
the same instructions on different data (src/lumen/geometry/csg.py module docstring). The layout of the flattened
arrays is the C ABI's (include/lumen_b200.h): volume records, daughter lists, a BVH per volume over its daughters'
world boxes (depth-first, skip pointers, one item per leaf), kinds, leaves, planes and programs.

Scope: the Geant4 solids of the reference's catalogue whose faces are planes, quadrics or tori (solids.py:477-772):
boxes, tubes, cones, spheres (radii, phi and theta ranges), orbs, ellipsoids, elliptical tubes and cones, paraboloids,
hyperboloids, polycones, polyhedra, tori (a torus leaf, leaf_kernels.py:212) and the convex polytopes (trd, para, trap,
tet, planar generic trap); their unions, subtractions and intersections with a placement of the second operand; at
most LUMEN_MAX_LEAVES leaves a solid. Volumes nest in a tree (daughters inside their mother, siblings disjoint or
touching).
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
    """One leaf in its solid's frame: optional quadric (A, b, c about oq) and planes n.(x - og) <= h; or a solid
    torus {(rho - R)^2 + z^2 <= r^2} of ``torus`` = (R, r) in the canonical coordinates u = M (x - og)
    (src/lumen/geometry/solids.py:88 TorusLeaf: M is the inverse of its placement's linear map; no planes)."""  # noqa: D205

    has_q: bool
    A: np.ndarray = field(default_factory=lambda: np.zeros((3, 3)))
    b: np.ndarray = field(default_factory=lambda: np.zeros(3))
    c: float = 0.0
    oq: np.ndarray = field(default_factory=lambda: np.zeros(3))
    og: np.ndarray = field(default_factory=lambda: np.zeros(3))
    N: np.ndarray = field(default_factory=lambda: np.zeros((0, 3)))
    H: np.ndarray = field(default_factory=lambda: np.zeros(0))
    torus: tuple | None = None
    M: np.ndarray = field(default_factory=lambda: np.eye(3))

    def moved(self, R: np.ndarray, p: np.ndarray) -> Leaf:
        """Return the leaf placed by x' = R x + p (its frame rotated and shifted)."""
        return Leaf(self.has_q, R @ self.A @ R.T, R @ self.b, self.c, R @ self.oq + p, R @ self.og + p,
                    self.N @ R.T, self.H.copy(), self.torus, self.M @ R.T)  # fmt: skip


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


FULL_PHI_TOL = 1e-12  # rad: a phi range this close to 2 pi is the full circle (src/lumen/rules/tolerances.py:104)
ANGLE_TOL = 1e-12


def _combine(op: int, la: Lowered, lb: Lowered, lo, hi) -> Lowered:
    """Return ``la op lb`` (1 union, 2 intersection, 3 subtraction), both in one frame, with the box (lo, hi)."""
    k = len(la.leaves)
    prog = list(la.program) + [(o, a + k) if o == 0 else (o, a) for o, a in lb.program] + [(op, 0)]
    return Lowered(la.leaves + lb.leaves, prog, np.asarray(lo, float), np.asarray(hi, float))


def phi_wedge(sphi: float, dphi: float) -> Lowered:
    """Return {phi in [sphi, sphi + dphi]} (dphi < 2 pi) as planes through the z axis: one leaf of two half-spaces
    when dphi <= pi, else the union of the two (src/lumen/geometry/solids.py:290 phi_wedge); its box unbounded."""  # noqa: D205
    ephi = sphi + dphi
    n1 = np.array([math.sin(sphi), -math.cos(sphi), 0.0])
    n2 = np.array([-math.sin(ephi), math.cos(ephi), 0.0])
    big = np.full(3, np.inf)
    if dphi <= math.pi + ANGLE_TOL:
        return Lowered([Leaf(False, N=np.stack([n1, n2]), H=np.zeros(2))], [(0, 0)], -big, big)
    a = Lowered([Leaf(False, N=n1[None], H=np.zeros(1))], [(0, 0)], -big, big)
    b = Lowered([Leaf(False, N=n2[None], H=np.zeros(1))], [(0, 0)], -big, big)
    return _combine(1, a, b, -big, big)


def with_phi(low: Lowered, sphi: float, dphi: float) -> Lowered:
    """Return a solid cut to the phi range [sphi, sphi + dphi] (rad; the full circle: itself)."""
    if not dphi > 0.0:
        raise ValueError(f"phi range {dphi} <= 0: Geant4's constructor aborts (invalid dphi)")
    if dphi >= 2.0 * math.pi - FULL_PHI_TOL:
        return low
    return _combine(2, low, phi_wedge(sphi, dphi), low.lo, low.hi)


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
    """G4Tubs: radii and half length (m), the phi range [sphi, sphi + dphi] (rad)."""

    rmax: float
    dz: float
    rmin: float = 0.0
    sphi: float = 0.0
    dphi: float = 2.0 * math.pi

    def lower(self):
        A = np.diag([1.0, 1.0, 0.0])
        N = np.array([[0, 0, 1.0], [0, 0, -1.0]])
        H = np.array([self.dz, self.dz])
        outer = Leaf(True, A=A, c=-self.rmax**2, N=N, H=H)
        h = np.array([self.rmax, self.rmax, self.dz])
        if self.rmin <= 0.0:
            low = Lowered([outer], [(0, 0)], -h, h)
        else:
            inner = Leaf(True, A=A.copy(), c=-self.rmin**2)
            low = Lowered([outer, inner], [(0, 0), (0, 1), (3, 0)], -h, h)
        return with_phi(low, self.sphi, self.dphi)


@dataclass
class Torus(Solid):
    """G4Torus (src/lumen/geometry/solids.py:697 g4_torus): swept radius ``rtor``, tube radii ``rmin`` and ``rmax``
    (m), the phi range [sphi, sphi + dphi] (rad)."""  # noqa: D205

    rmax: float
    rtor: float
    rmin: float = 0.0
    sphi: float = 0.0
    dphi: float = 2.0 * math.pi

    def lower(self):
        if not (0.0 <= self.rmin < self.rmax <= self.rtor):
            raise ValueError(f"Torus: 0 <= rmin < rmax <= rtor, got {self.rmin}, {self.rmax}, {self.rtor}")
        big = self.rtor + self.rmax
        h = np.array([big, big, self.rmax])
        outer = Leaf(False, torus=(float(self.rtor), float(self.rmax)))
        low = Lowered([outer], [(0, 0)], -h, h)
        if self.rmin > 0.0:
            low = _combine(3, low, Lowered([Leaf(False, torus=(float(self.rtor), float(self.rmin)))], [(0, 0)], -h, h),
                           -h, h)  # fmt: skip
        return with_phi(low, self.sphi, self.dphi)


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


# --------------------------------------------------------------------- the rest of the Geant4 catalogue (solids.py)
CYLINDER_REL = 1e-15  # a frustum whose radii agree to this (relative) is a cylinder (tolerances.py:106)
Z_TOL = 1e-15  # m: polycone / polyhedra sections thinner than this are dropped (tolerances.py:107)
DEGENERATE_FACE = 1e-14  # a face normal this small (relative to the size squared) has collapsed (tolerances.py:111)
VERTEX_TOL = 1e-9  # relative: a vertex beyond a face plane by more than this is not convex (tolerances.py:112)
G4CONS_ZERO_RMIN = 1e-6  # m: G4Cons's inner radius standing in for a zero one opposite a non-zero one (1e3 kRadTolerance)
FULL = 2.0 * math.pi


def _one(leaf: Leaf, lo, hi) -> Lowered:
    return Lowered([leaf], [(0, 0)], np.asarray(lo, float), np.asarray(hi, float))


def _unbounded(leaf: Leaf) -> Lowered:
    return _one(leaf, np.full(3, -np.inf), np.full(3, np.inf))


def _planes_leaf(planes, origin=(0.0, 0.0, 0.0)) -> Leaf:
    """The intersection of the half-spaces [(n, h)] (n . x <= h, absolute offsets) as a plane leaf at ``origin``."""
    o = np.asarray(origin, float)
    N = np.asarray([n for n, _ in planes], float).reshape(-1, 3)
    H = np.asarray([h - float(np.dot(n, o)) for n, h in planes], float)
    return Leaf(False, og=o.copy(), oq=o.copy(), N=N, H=H)


def _frustum(z_lo, r_lo, z_hi, r_hi, caps=True, one_nappe=True) -> Leaf:
    """The solid of revolution about z whose radius runs affinely from r_lo at z_lo to r_hi at z_hi (z_lo < z_hi):
    a G4Cons, or one section of a G4Polycone. Taken about the slab's middle m, with the slope s and the middle
    radius r_m, its surface is x^2 + y^2 = (r_m + s z)^2: the quadric x^2 + y^2 - s^2 z^2 - 2 r_m s z - r_m^2 <= 0,
    which holds two nappes meeting at the apex; ``one_nappe`` keeps the one of positive radius (the plane
    r_m + s z >= 0). Equal radii make it the cylinder x^2 + y^2 <= r^2. ``caps``: the slab's planes."""  # noqa: D205
    half = 0.5 * (z_hi - z_lo)
    centre = np.array([0.0, 0.0, 0.5 * (z_lo + z_hi)])
    normals, offsets = ([(0.0, 0.0, 1.0), (0.0, 0.0, -1.0)], [half, half]) if caps else ([], [])
    if abs(r_hi - r_lo) < CYLINDER_REL * max(1.0, abs(r_lo)):
        quad = dict(A=np.diag([1.0, 1.0, 0.0]), c=-(r_lo * r_lo))
    else:
        slope, r_m = (r_hi - r_lo) / (z_hi - z_lo), 0.5 * (r_lo + r_hi)
        quad = dict(A=np.diag([1.0, 1.0, -(slope * slope)]), b=np.array([0.0, 0.0, -(r_m * slope)]), c=-(r_m * r_m))
        if one_nappe:
            normals.append((0.0, 0.0, -slope))
            offsets.append(r_m)
    return Leaf(True, oq=centre, og=centre.copy(), N=np.asarray(normals, float).reshape(-1, 3),
                H=np.asarray(offsets, float), **quad)  # fmt: skip


def _cone_theta(theta, up=True) -> Leaf:
    """The solid cone of half-angle theta < pi / 2 about +z (up) or -z, apex at the origin."""
    t2 = math.tan(theta) ** 2
    return Leaf(True, A=np.diag([1.0, 1.0, -t2]), N=np.array([[0.0, 0.0, -1.0 if up else 1.0]]), H=np.zeros(1))


def _halfspace(n, h) -> Leaf:
    return Leaf(False, N=np.asarray([n], float), H=np.array([float(h)]))


def convex_polytope(verts, faces) -> Lowered:
    """The convex polytope of vertices and faces (index lists, any orientation), one plane leaf at the centroid; a
    vertex set that is not convex is refused (solids.py:332 polytope_from_faces)."""
    V = np.asarray(verts, float)
    cen = V.mean(0)
    planes = []
    for fc in faces:
        P = V[list(fc)]
        nrm = np.cross(P[2] - P[0], P[3] - P[1]) if len(P) >= 4 else np.cross(P[1] - P[0], P[2] - P[0])
        ln = float(np.linalg.norm(nrm))
        if ln < DEGENERATE_FACE * max(1.0, float(np.abs(V).max()) ** 2):
            continue  # a collapsed face
        nrm = nrm / ln
        h = float(np.dot(nrm, P.mean(0)))
        if np.dot(nrm, cen) > h:
            nrm, h = -nrm, -h
        planes.append((nrm, h))
    tol = VERTEX_TOL * max(1.0, float(np.abs(V).max()))
    if any(float(np.max(V @ n - h)) > tol for n, h in planes):
        raise ValueError("convex_polytope: the vertices are not convex in position (a concave base or a twisted face)")
    if len(planes) > MAX_PLANES:
        raise ValueError(f"convex_polytope: {len(planes)} faces, at most {MAX_PLANES}")
    return _one(_planes_leaf(planes, cen), V.min(0), V.max(0))


HEX_FACES = [(0, 1, 3, 2), (4, 5, 7, 6), (0, 1, 5, 4), (2, 3, 7, 6), (0, 2, 6, 4), (1, 3, 7, 5)]


@dataclass
class Cons(Solid):
    """G4Cons: inner and outer radii at -dz and +dz, half length dz (m), phi range (solids.py:509 g4_cone)."""

    rmin1: float
    rmax1: float
    rmin2: float
    rmax2: float
    dz: float
    sphi: float = 0.0
    dphi: float = FULL

    def lower(self):
        r1, r2 = self.rmin1, self.rmin2
        if r1 == 0.0 and r2 > 0.0:
            r1 = G4CONS_ZERO_RMIN
        if r2 == 0.0 and r1 > 0.0:
            r2 = G4CONS_ZERO_RMIN
        big = max(self.rmax1, self.rmax2)
        lo, hi = (-big, -big, -self.dz), (big, big, self.dz)
        low = _one(_frustum(-self.dz, self.rmax1, self.dz, self.rmax2), lo, hi)
        if r1 > 0.0 or r2 > 0.0:
            low = _combine(3, low, _unbounded(_frustum(-self.dz, r1, self.dz, r2, caps=False)), lo, hi)
        return with_phi(low, self.sphi, self.dphi)


@dataclass
class SphereShell(Solid):
    """G4Sphere: radii rmin, rmax (m), phi range [sphi, sphi + dphi] and theta range [stheta, stheta + dtheta]
    (rad; solids.py:626 g4_sphere, :600 _theta_cut)."""  # noqa: D205

    rmax: float
    rmin: float = 0.0
    sphi: float = 0.0
    dphi: float = FULL
    stheta: float = 0.0
    dtheta: float = math.pi

    def lower(self):
        r = self.rmax
        lo, hi = (-r, -r, -r), (r, r, r)
        low = _one(Leaf(True, A=np.eye(3), c=-r * r), lo, hi)
        if self.rmin > 0.0:
            low = _combine(3, low, _unbounded(Leaf(True, A=np.eye(3), c=-self.rmin**2)), lo, hi)
        low = with_phi(low, self.sphi, self.dphi)
        ts, te, h = self.stheta, self.stheta + self.dtheta, 0.5 * math.pi
        if ts > ANGLE_TOL:  # theta < ts removed
            if abs(ts - h) < ANGLE_TOL:
                low = _combine(3, low, _unbounded(_halfspace((0, 0, -1), 0.0)), lo, hi)
            elif ts < h:
                low = _combine(3, low, _unbounded(_cone_theta(ts, up=True)), lo, hi)
            else:
                low = _combine(2, low, _unbounded(_cone_theta(math.pi - ts, up=False)), lo, hi)
        if te < math.pi - ANGLE_TOL:  # theta <= te kept
            if abs(te - h) < ANGLE_TOL:
                low = _combine(2, low, _unbounded(_halfspace((0, 0, -1), 0.0)), lo, hi)
            elif te < h:
                low = _combine(2, low, _unbounded(_cone_theta(te, up=True)), lo, hi)
            else:
                low = _combine(3, low, _unbounded(_cone_theta(math.pi - te, up=False)), lo, hi)
        return low


@dataclass
class Orb(Solid):
    """G4Orb of radius r (m)."""

    r: float

    def lower(self):
        return _one(Leaf(True, A=np.eye(3), c=-self.r**2), (-self.r,) * 3, (self.r,) * 3)


@dataclass
class Ellipsoid(Solid):
    """G4Ellipsoid of semi-axes ax, by, cz (m) cut to [zcut1, zcut2] (both 0: no cut; clamped to [-cz, cz])."""

    ax: float
    by: float
    cz: float
    zcut1: float = 0.0
    zcut2: float = 0.0

    def lower(self):
        a, b, c = self.ax, self.by, self.cz
        lo, hi = (-c, c) if (self.zcut1 == 0.0 and self.zcut2 == 0.0) else (max(self.zcut1, -c), min(self.zcut2, c))
        N, H = [], []
        if hi < c:
            N, H = [*N, [0, 0, 1.0]], [*H, hi]
        if lo > -c:
            N, H = [*N, [0, 0, -1.0]], [*H, -lo]
        leaf = Leaf(True, A=np.diag([1 / a**2, 1 / b**2, 1 / c**2]), c=-1.0, N=np.asarray(N, float).reshape(-1, 3),
                    H=np.asarray(H, float))  # fmt: skip
        return _one(leaf, (-a, -b, lo), (a, b, hi))


@dataclass
class EllipticalTube(Solid):
    """G4EllipticalTube of semi-axes dx, dy and half length dz (m)."""

    dx: float
    dy: float
    dz: float

    def lower(self):
        leaf = Leaf(True, A=np.diag([1 / self.dx**2, 1 / self.dy**2, 0.0]), c=-1.0,
                    N=np.array([[0, 0, 1.0], [0, 0, -1.0]]), H=np.array([self.dz, self.dz]))  # fmt: skip
        return _one(leaf, (-self.dx, -self.dy, -self.dz), (self.dx, self.dy, self.dz))


@dataclass
class EllipticalCone(Solid):
    """G4EllipticalCone: (x / dx)^2 + (y / dy)^2 <= (zmax - z)^2, |z| <= min(zcut, zmax) (dx, dy unitless)."""

    dx: float
    dy: float
    zmax: float
    zcut: float

    def lower(self):
        zm, zt = self.zmax, min(self.zcut, self.zmax)
        leaf = Leaf(True, A=np.diag([1 / self.dx**2, 1 / self.dy**2, -1.0]), b=np.array([0.0, 0.0, zm]), c=-zm * zm,
                    N=np.array([[0, 0, 1.0], [0, 0, -1.0], [0, 0, 1.0]]), H=np.array([zt, zt, zm]))  # fmt: skip
        rx, ry = self.dx * (zm + zt), self.dy * (zm + zt)
        return _one(leaf, (-rx, -ry, -zt), (rx, ry, zt))


@dataclass
class Paraboloid(Solid):
    """G4Paraboloid of radii rlo at -dz and rhi at +dz (m): rho^2 <= k1 z + k2."""

    rlo: float
    rhi: float
    dz: float

    def lower(self):
        k1 = (self.rhi**2 - self.rlo**2) / (2.0 * self.dz)
        k2 = 0.5 * (self.rhi**2 + self.rlo**2)
        leaf = Leaf(True, A=np.diag([1.0, 1.0, 0.0]), b=np.array([0.0, 0.0, -0.5 * k1]), c=-k2,
                    N=np.array([[0, 0, 1.0], [0, 0, -1.0]]), H=np.array([self.dz, self.dz]))  # fmt: skip
        return _one(leaf, (-self.rhi, -self.rhi, -self.dz), (self.rhi, self.rhi, self.dz))


@dataclass
class Hype(Solid):
    """G4Hype: rho^2 <= rmax^2 + tan^2(outst) z^2 and >= rmin^2 + tan^2(inst) z^2, |z| <= dz (m, rad)."""

    rmin: float
    rmax: float
    inst: float
    outst: float
    dz: float

    def lower(self):
        to2, ti2 = math.tan(self.outst) ** 2, math.tan(self.inst) ** 2
        big = math.sqrt(self.rmax**2 + to2 * self.dz**2)
        lo, hi = (-big, -big, -self.dz), (big, big, self.dz)
        low = _one(Leaf(True, A=np.diag([1.0, 1.0, -to2]), c=-self.rmax**2, N=np.array([[0, 0, 1.0], [0, 0, -1.0]]),
                        H=np.array([self.dz, self.dz])), lo, hi)  # fmt: skip
        if self.rmin > 0.0 or self.inst > 0.0:
            low = _combine(3, low, _unbounded(Leaf(True, A=np.diag([1.0, 1.0, -ti2]), c=-self.rmin**2)), lo, hi)
        return low


def _profile(zplanes, rel=1e-12):
    """A G4Polycone / G4Polyhedra profile as arrays (z, inner, outer) from its z-planes [(rmin, rmax, z)], with every
    interior plane dropped that lies on the straight line of its kept neighbours for both radii, z strictly between
    them: Geant4 builds the solid from G4ReduciblePolygon after RemoveRedundantVertices, so such a plane is no
    section boundary (the tolerance is ``rel`` of the profile's scale there)."""  # noqa: D205
    arr = np.asarray(zplanes, float).reshape(-1, 3)
    inner, outer, z = arr[:, 0], arr[:, 1], arr[:, 2]
    kept = [0]
    for i in range(1, len(z) - 1):
        a, c = kept[-1], i + 1
        between = (z[i] - z[a]) * (z[c] - z[i]) > 0
        if between:
            t = (z[i] - z[a]) / (z[c] - z[a])
            scale = rel * max(1.0, abs(z[a]), abs(z[c]), abs(outer[a]), abs(outer[c]))
            if all(abs(r[a] + t * (r[c] - r[a]) - r[i]) <= scale for r in (inner, outer)):
                continue
        kept.append(i)
    if len(z) > 1:
        kept.append(len(z) - 1)
    return z[kept], inner[kept], outer[kept]


def _slabs(z, inner, outer):
    """The profile's sections between consecutive z-planes, each as (z_lo, z_hi, inner_lo, inner_hi, outer_lo,
    outer_hi) with z_lo below z_hi; a section thinner than Z_TOL (a radius step at one z) bounds nothing."""  # noqa: D205
    for i in range(len(z) - 1):
        lo, hi = (i, i + 1) if z[i] <= z[i + 1] else (i + 1, i)
        if z[hi] - z[lo] < Z_TOL:
            continue
        yield z[lo], z[hi], inner[lo], inner[hi], outer[lo], outer[hi]


def _union_all(parts, lo, hi) -> Lowered:
    if not parts:
        raise ValueError("a solid with no part: every section is thinner than the z tolerance")
    out = parts[0]
    for p in parts[1:]:
        out = _combine(1, out, p, lo, hi)
    return Lowered(out.leaves, out.program, np.asarray(lo, float), np.asarray(hi, float))


@dataclass
class Polycone(Solid):
    """G4Polycone of z-planes [(rmin, rmax, z)] (m) and phi range (dphi <= 0: the full circle; solids.py:556)."""

    zplanes: tuple
    sphi: float = 0.0
    dphi: float = FULL

    def lower(self):
        z, inner, outer = _profile(self.zplanes)
        r = float(outer.max())
        lo, hi = (-r, -r, float(z.min())), (r, r, float(z.max()))
        parts = []
        for z0, z1, i0, i1, o0, o1 in _slabs(z, inner, outer):
            part = _one(_frustum(z0, o0, z1, o1), lo, hi)
            if i0 > 0 or i1 > 0:  # the bore: the inner frustum taken out, unbounded across the slab's planes
                part = _combine(3, part, _unbounded(_frustum(z0, i0, z1, i1, caps=False)), lo, hi)
            parts.append(part)
        return with_phi(_union_all(parts, lo, hi), self.sphi, FULL if self.dphi <= 0.0 else self.dphi)


@dataclass
class Polyhedra(Solid):
    """G4Polyhedra of z-planes [(rmin, rmax, z)] whose radii are the distances to the sides (apothems), ``nsides``
    sides over the phi range (dphi <= 0: the full circle; solids.py:588)."""  # noqa: D205

    zplanes: tuple
    nsides: int
    sphi: float = 0.0
    dphi: float = FULL

    def _section(self, z_lo, a_lo, z_hi, a_hi, caps):
        """One section as a plane leaf: side k (its outward normal at the middle of its phi step) keeps the points
        whose distance from the axis along that normal is within the apothem, affine in z from a_lo to a_hi."""  # noqa: D205
        span = FULL if self.dphi <= 0.0 else self.dphi
        slope = (a_hi - a_lo) / (z_hi - z_lo)
        mids = self.sphi + (np.arange(self.nsides) + 0.5) * (span / self.nsides)
        normals = np.column_stack([np.cos(mids), np.sin(mids), np.full(self.nsides, -slope)])
        planes = [(nv, a_lo - slope * z_lo) for nv in normals]
        if caps:
            planes += [((0.0, 0.0, 1.0), z_hi), ((0.0, 0.0, -1.0), -z_lo)]
        return _planes_leaf(planes, (0.0, 0.0, 0.5 * (z_lo + z_hi)))

    def lower(self):
        z, inner, outer = _profile(self.zplanes)
        full = self.dphi >= FULL - FULL_PHI_TOL or self.dphi <= 0.0
        step = (FULL if self.dphi <= 0 else self.dphi) / self.nsides
        r = float(outer.max()) / math.cos(0.5 * min(step, math.pi - 1e-6))  # the corners lie beyond the apothem
        lo, hi = (-r, -r, float(z.min())), (r, r, float(z.max()))
        parts = []
        for z0, z1, i0, i1, o0, o1 in _slabs(z, inner, outer):
            part = _one(self._section(z0, o0, z1, o1, True), lo, hi)
            if i0 > 0 or i1 > 0:
                part = _combine(3, part, _unbounded(self._section(z0, i0, z1, i1, False)), lo, hi)
            parts.append(part)
        low = _union_all(parts, lo, hi)
        return low if full else _combine(2, low, phi_wedge(self.sphi, self.dphi), lo, hi)


@dataclass
class Trd(Solid):
    """G4Trd: half lengths dx1, dy1 at -dz and dx2, dy2 at +dz (m)."""

    dx1: float
    dx2: float
    dy1: float
    dy2: float
    dz: float

    def lower(self):
        a, b, c, d, z = self.dx1, self.dx2, self.dy1, self.dy2, self.dz
        verts = [(-a, -c, -z), (a, -c, -z), (-a, c, -z), (a, c, -z), (-b, -d, z), (b, -d, z), (-b, d, z), (b, d, z)]
        return convex_polytope(verts, HEX_FACES)


@dataclass
class Para(Solid):
    """G4Para: half lengths dx, dy, dz (m) and the angles alpha, theta, phi (rad)."""

    dx: float
    dy: float
    dz: float
    alpha: float
    theta: float
    phi: float

    def lower(self):
        ta, tt = math.tan(self.alpha), math.tan(self.theta)
        verts = []
        for sz in (-1, 1):
            for sy in (-1, 1):
                for sx in (-1, 1):
                    Z, Y = sz * self.dz, sy * self.dy
                    verts.append((sx * self.dx + Y * ta + Z * tt * math.cos(self.phi), Y + Z * tt * math.sin(self.phi), Z))
        return convex_polytope(verts, HEX_FACES)


@dataclass
class Trap(Solid):
    """G4Trap: half length dz, the axis's theta and phi, and at -dz / +dz the half lengths dy1 (dx1, dx2 at -/+dy1)
    and the angle alpha1, dy2 (dx3, dx4) and alpha2 (m, rad)."""  # noqa: D205

    dz: float
    theta: float
    phi: float
    dy1: float
    dx1: float
    dx2: float
    alpha1: float
    dy2: float
    dx3: float
    dx4: float
    alpha2: float

    def lower(self):
        dz, tth = self.dz, math.tan(self.theta)
        cph, sph = math.cos(self.phi), math.sin(self.phi)
        t1, t2 = math.tan(self.alpha1), math.tan(self.alpha2)
        verts = []
        for s, dy, xa, xb, t in ((-1, self.dy1, self.dx1, self.dx2, t1), (1, self.dy2, self.dx3, self.dx4, t2)):
            cx, cy = s * dz * tth * cph, s * dz * tth * sph
            verts += [(cx - dy * t - xa, cy - dy, s * dz), (cx - dy * t + xa, cy - dy, s * dz),
                      (cx + dy * t - xb, cy + dy, s * dz), (cx + dy * t + xb, cy + dy, s * dz)]  # fmt: skip
        return convex_polytope(verts, HEX_FACES)


@dataclass
class Tet(Solid):
    """G4Tet of four vertices (m)."""

    v1: tuple
    v2: tuple
    v3: tuple
    v4: tuple

    def lower(self):
        return convex_polytope([self.v1, self.v2, self.v3, self.v4], [(0, 1, 2), (0, 1, 3), (0, 2, 3), (1, 2, 3)])


@dataclass
class GenericTrap(Solid):
    """G4GenericTrap with planar faces: eight (x, y) vertices, 0..3 at -dz and 4..7 at +dz (m); a twisted face is
    refused."""  # noqa: D205

    verts_xy: tuple
    dz: float

    def lower(self):
        xy = np.asarray(self.verts_xy, float).reshape(8, 2)
        zcol = np.repeat([-self.dz, self.dz], 4)[:, None]
        V = np.hstack([xy, zcol])  # rows 0..3 the -dz face, 4..7 the +dz face, in the same order
        low_ring = np.arange(4)
        nxt = np.roll(low_ring, -1)
        sides = np.stack([low_ring, nxt, nxt + 4, low_ring + 4], 1)  # each side: an edge below and the one above it
        for quad in sides:
            p = V[quad]
            # four points are coplanar when the volume they span is 0: a twisted side is a hyperbolic paraboloid
            vol = abs(np.linalg.det(np.stack([p[1] - p[0], p[2] - p[0], p[3] - p[0]])))
            scale = max(np.linalg.norm(p - p[0], axis=1).max(), 1e-300) ** 3
            if vol > 1e-9 * scale:
                raise NotImplementedError("GenericTrap with a twisted (non-planar) face")
        return convex_polytope(V, [tuple(low_ring), tuple(low_ring + 4), *map(tuple, sides)])


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
class Mesh(Solid):
    """G4TessellatedSolid (src/lumen/geometry/scene.py:33 Mesh): a closed triangle surface, ``tris`` (n, 3, 3) m in its
    definition frame, each triangle's normal (V1 - V0) x (V2 - V0) outward. An opaque free-form part: the navigator
    uses only its first facet hit and that facet's normal (a facet met from either side is an entry into it; no point
    is inside it), so its material holds no photon (no RINDEX) and it has no daughters and is no sensor."""  # noqa: D205

    def __init__(self, tris):
        self.tris = np.asarray(tris, float).reshape(-1, 3, 3)
        if not len(self.tris):
            raise ValueError("Mesh: no triangles")

    def lower(self):
        raise ValueError("a Mesh is not a CSG solid: it is placed as triangle chunks (navigator_arrays)")


def icosphere(radius: float, subdiv: int = 2) -> np.ndarray:
    """Return the triangles (n, 3, 3) of a sphere of ``radius`` tessellated from an icosahedron by ``subdiv`` 4-way
    splits (20 x 4^subdiv triangles, vertices on the sphere), wound so that (V1 - V0) x (V2 - V0) points out."""  # noqa: D205
    p = (1.0 + math.sqrt(5.0)) / 2.0
    V = [(-1, p, 0), (1, p, 0), (-1, -p, 0), (1, -p, 0), (0, -1, p), (0, 1, p), (0, -1, -p), (0, 1, -p),
         (p, 0, -1), (p, 0, 1), (-p, 0, -1), (-p, 0, 1)]  # fmt: skip
    F = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10),
         (8, 6, 7), (9, 8, 1)]  # fmt: skip
    T = np.asarray([[V[i] for i in f] for f in F], np.float64)
    T /= np.linalg.norm(T, axis=2, keepdims=True)
    for _ in range(subdiv):
        a, b, c = T[:, 0], T[:, 1], T[:, 2]
        ab, bc, ca = [x / np.linalg.norm(x, axis=1, keepdims=True) for x in (a + b, b + c, c + a)]
        T = np.concatenate([np.stack(s, 1) for s in ((a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca))])
    n = np.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    flip = np.einsum("ij,ij->i", n, T.mean(1)) < 0
    T[flip] = T[flip][:, ::-1]
    return radius * T


def box_mesh(hx: float, hy: float, hz: float) -> np.ndarray:
    """Return the 12 triangles of a box of half lengths (hx, hy, hz), wound outward."""
    c = np.array([[sx * hx, sy * hy, sz * hz] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)])
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    T = np.asarray([[c[q[0]], c[q[1]], c[q[2]]] for q in quads] + [[c[q[0]], c[q[2]], c[q[3]]] for q in quads])
    n = np.cross(T[:, 1] - T[:, 0], T[:, 2] - T[:, 0])
    flip = np.einsum("ij,ij->i", n, T.mean(1)) < 0
    T[flip] = T[flip][:, ::-1]
    return T


MESH_CHUNK = 8  # triangles per chunk (one BVH item: src/lumen/geometry/navigator_build.py:46)
MORTON_BITS = 10  # the chunks' order: triangles sorted along a Morton curve of this many bits per axis
MESH_PARALLEL = 1e-6  # a mesh hit's t comes from its plane where |n . d| is above this (tolerances.py:135)


def morton(c) -> np.ndarray:
    """Return the Morton codes (MORTON_BITS bits per axis, interleaved z y x from the top bit) of points c (n, 3),
    quantised in their own bounding box."""  # noqa: D205, D209
    c = np.asarray(c, np.float64)
    lo, hi = c.min(0), c.max(0)
    q = np.clip(((c - lo) / np.maximum(hi - lo, 1e-300) * (1 << MORTON_BITS)).astype(np.int64), 0, (1 << MORTON_BITS) - 1)
    code = np.zeros(len(c), np.int64)
    for b in range(MORTON_BITS - 1, -1, -1):
        for a in range(3):
            code = (code << 1) | ((q[:, a] >> b) & 1)
    return code


def mesh_chunks(meshes):
    """Return the chunk arrays of placed meshes [(world triangles (n, 3, 3), mother)]: the triangles Morton-ordered
    per mesh (its centroids), cut into chunks of MESH_CHUNK consecutive triangles; per triangle V0, V1, V2 and the unit
    normal (float64), per chunk (first triangle, count, mesh) and its box padded as the reference's chunks
    (navigator_build.py:346: WORLD_BOX_PAD_REL (|lo| + |hi|) + WORLD_BOX_PAD_ABS)."""  # noqa: D205, D209
    tri, chunk, mother = [], [], []
    for m, (T, mo) in enumerate(meshes):
        T = np.asarray(T, np.float64)[np.argsort(morton(T.mean(1)), kind="stable")]
        k0 = sum(len(x) for x in tri)
        for s in range(0, len(T), MESH_CHUNK):
            chunk.append([k0 + s, min(MESH_CHUNK, len(T) - s), m, 0])
            mother.append(mo)
        tri.append(T)
    V = np.concatenate(tri) if tri else np.zeros((0, 3, 3))
    nrm = np.cross(V[:, 1] - V[:, 0], V[:, 2] - V[:, 0])
    nrm = nrm / np.maximum(np.linalg.norm(nrm, axis=1, keepdims=True), 1e-30)
    ch = np.asarray(chunk, np.int64).reshape(-1, 4)
    lo = np.asarray([V[s:s + c].reshape(-1, 3).min(0) for s, c, _, _ in ch]).reshape(-1, 3)
    hi = np.asarray([V[s:s + c].reshape(-1, 3).max(0) for s, c, _, _ in ch]).reshape(-1, 3)
    pad = WORLD_BOX_PAD_REL * (np.abs(lo) + np.abs(hi)) + WORLD_BOX_PAD_ABS
    tri_f = np.concatenate([V.reshape(-1, 9), nrm], 1) if len(V) else np.zeros((0, 12))
    return dict(tri=tri_f, chunk=ch, mother=np.asarray(mother, np.int64), lo=lo - pad, hi=hi + pad)


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
    cb = np.asarray(arrays.get("chunk_box64", np.zeros((0, 6))), np.float64)
    if len(cb):  # a mesh chunk's box bounds the query like a sensor's (reach.py:102: a mesh box on the segment)
        sv = np.concatenate([sv, n + np.arange(len(cb))])
        f_lo, f_hi = np.concatenate([f_lo, cb[:, :3] - pad]), np.concatenate([f_hi, cb[:, 3:] + pad])
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


MIN_GROUP = 8  # a rotation shared by at least this many daughters (or by all) may be a frame group (bvh.py:20)
GROUP_GAIN = 4.0  # ... when their world boxes' surface areas are at least this times their own boxes' (bvh.py:21)
MAX_GROUPS_PER_VOLUME = 64  # frame groups in one volume (the engine walks them in turn)


def _area(lo, hi):
    d = np.maximum(np.asarray(hi) - np.asarray(lo), 0.0)
    return 2.0 * (d[..., 0] * d[..., 1] + d[..., 1] * d[..., 2] + d[..., 0] * d[..., 2])


def frame_groups(ks, placed, low, lo_w, hi_w, n):
    """Return (the candidates left to the world-frame BVH, [(R, members)]): the daughters of one volume sharing a
    rotation R other than the identity, at least MIN_GROUP of them (or all its daughters), whose world boxes' summed
    surface area is at least GROUP_GAIN times their own boxes' (src/lumen/geometry/navigator_build.py:11, bvh.py
    frame_groups_all): each such set gets a BVH in R's frame (diagonal wire planes)."""  # noqa: D205, D209
    units = [k for k in ks if k < n]
    by = {}
    for k in units:
        by.setdefault(tuple(np.round(placed[k].R.ravel(), 12)), []).append(k)
    groups, taken = [], set()
    for mem in by.values():
        R = placed[mem[0]].R
        if np.allclose(R, np.eye(3), atol=1e-12) or not (len(mem) >= MIN_GROUP or len(mem) == len(units)):
            continue
        own = sum(float(_area(low[k].lo, low[k].hi)) for k in mem)
        if float(_area(lo_w[mem], hi_w[mem]).sum()) < GROUP_GAIN * own:
            continue
        groups.append((R, mem))
        taken.update(mem)
        if len(groups) == MAX_GROUPS_PER_VOLUME:  # the engine's bound (LUMEN_MAX_GROUPS_PER_VOLUME)
            break
    return [k for k in ks if k not in taken], groups


def group_boxes(R, mem, placed, low):
    """Return the members' boxes (lo, hi) in the group frame x_g = R^T x_w, padded as the world boxes."""
    lo, hi = np.zeros((len(mem), 3)), np.zeros((len(mem), 3))
    for j, k in enumerate(mem):
        M, tt = R.T @ placed[k].R, R.T @ placed[k].t
        c = np.array([[(low[k].hi if (q >> a) & 1 else low[k].lo)[a] for a in range(3)] for q in range(8)]) @ M.T + tt
        lo[j], hi[j] = pad_box(c.min(0), c.max(0))
    return lo, hi


def _node_boxes64(node_i, items, lo, hi, n0=0, n1=None, out=None) -> np.ndarray:
    """Return the BVH nodes' boxes in float64 over the float32 BVH's topology (depth-first with skips: a node's left
    child follows it, its right child is the left child's skip): a leaf the union of its items' float64 boxes, an inner
    node the union of its children's, bottom-up."""
    out = np.zeros((len(node_i), 6)) if out is None else out
    for k in range((len(node_i) if n1 is None else n1) - 1, n0 - 1, -1):
        cnt, st = int(node_i[k, 1]), int(node_i[k, 2])
        if cnt > 0:
            it = items[st:st + cnt]
            out[k, :3], out[k, 3:] = lo[it].min(0), hi[it].max(0)
        else:
            lc = k + 1
            rc = int(node_i[lc, 0])
            out[k, :3] = np.minimum(out[lc, :3], out[rc, :3])
            out[k, 3:] = np.maximum(out[lc, 3:], out[rc, 3:])
    return out


def _convex_leaf(low: Lowered) -> bool:
    """Whether a lowered solid is one convex leaf (planes, and a quadric whose matrix is positive semidefinite)."""
    if len(low.leaves) != 1 or len(low.program) != 1 or low.leaves[0].torus is not None:
        return False
    lf = low.leaves[0]
    return (not lf.has_q) or float(np.min(np.linalg.eigvalsh(0.5 * (lf.A + lf.A.T)))) >= -1e-12


def _leaf_holds(lf: Leaf, x: np.ndarray) -> np.ndarray:
    """Whether points x (n, 3; the solid's frame) lie in leaf lf (float64)."""
    ok = np.all((x - lf.og) @ lf.N.T <= lf.H, axis=1) if len(lf.N) else np.ones(len(x), bool)
    if lf.has_q:
        y = x - lf.oq
        ok &= np.einsum("ni,ij,nj->n", y, lf.A, y) + 2.0 * (y @ lf.b) + lf.c <= 0.0
    return ok


def _proved_inside(inner: Placed, outer: Placed, low_in: Lowered, low_out: Lowered, tol: float) -> bool:
    """Whether ``inner``'s solid is proved to lie inside ``outer``'s: its box shrunk by ``tol`` has every corner in
    ``outer``'s solid and that solid is one convex leaf (so the corners' hull, the box, is inside it). No sampling: what
    is not proved is not assumed (src/lumen/geometry/ownership.py:11)."""  # noqa: D205, D209
    if not _convex_leaf(low_out):
        return False
    lo, hi = np.minimum(low_in.lo + tol, low_in.hi - tol), np.maximum(low_in.hi - tol, low_in.lo + tol)
    c = np.array([[(hi if (k >> a) & 1 else lo)[a] for a in range(3)] for k in range(8)])
    w = c @ inner.R.T + inner.t
    return bool(_leaf_holds(low_out.leaves[0], (w - outer.t) @ outer.R).all())


def _leaf_interval(lf: Leaf, lo, hi) -> int:
    """Return leaf lf's membership over the box [lo, hi] (its solid's frame) by interval bounds: -1 out everywhere,
    1 in everywhere, 0 not proved either way (a torus is never proved)."""
    if lf.torus is not None:
        return 0
    c, r = 0.5 * (lo + hi), 0.5 * (hi - lo)
    ins = True
    for nn, hh in zip(lf.N, lf.H, strict=True):  # n . (x - og) <= h: exact bounds of a linear form
        m, s = float(nn @ (c - lf.og)) - hh, float(np.abs(nn) @ r)
        if m - s > 0.0:
            return -1
        ins = ins and m + s <= 0.0
    if lf.has_q:  # y^T A y + 2 b . y + c over y in [lo - oq, hi - oq]: interval arithmetic, term by term
        ylo, yhi = lo - lf.oq, hi - lf.oq
        fl, fh = float(lf.c), float(lf.c)
        for i in range(3):
            for j in range(3):
                a = float(lf.A[i, j])
                if a == 0.0:
                    continue
                if i == j:
                    sq = [ylo[i] * ylo[i], yhi[i] * yhi[i]]
                    pl, ph = (0.0 if ylo[i] <= 0.0 <= yhi[i] else min(sq)), max(sq)
                else:
                    pr = [ylo[i] * ylo[j], ylo[i] * yhi[j], yhi[i] * ylo[j], yhi[i] * yhi[j]]
                    pl, ph = min(pr), max(pr)
                fl += min(a * pl, a * ph)
                fh += max(a * pl, a * ph)
            bl, bh = 2.0 * float(lf.b[i]) * ylo[i], 2.0 * float(lf.b[i]) * yhi[i]
            fl += min(bl, bh)
            fh += max(bl, bh)
        if fl > 0.0:
            return -1
        ins = ins and fh <= 0.0
    return 1 if ins else 0


def _solid_interval(low: Lowered, lo, hi) -> int:
    """Return a lowered solid's membership over the box [lo, hi] (its frame): its program in three-valued logic."""
    st = []
    for op, arg in low.program:
        if op == 0:
            st.append(_leaf_interval(low.leaves[arg], lo, hi))
            continue
        b, a = st.pop(), st.pop()
        if op == 1:  # union
            st.append(1 if (a == 1 or b == 1) else (-1 if (a == -1 and b == -1) else 0))
        elif op == 2:  # intersection
            st.append(-1 if (a == -1 or b == -1) else (1 if (a == 1 and b == 1) else 0))
        else:  # subtraction a - b
            st.append(-1 if (a == -1 or b == 1) else (1 if (a == 1 and b == -1) else 0))
    return st[-1]


def _local_box(p: Placed, lo, hi):
    """Return the box (in placement p's frame) enclosing the world box [lo, hi]."""
    c, r = 0.5 * (lo + hi) - p.t, 0.5 * (hi - lo)
    cl, rl = c @ p.R, r @ np.abs(p.R)
    return cl - rl, cl + rl


def _proved_apart(pa: Placed, pb: Placed, la: Lowered, lb: Lowered, depth: int = 7) -> bool:
    """Whether solids a and b share no point: in a's frame, the region a's box shares with the box of b's box
    corners is empty, or every cell of its bisection (down to ``depth`` levels) is proved outside one of them by
    interval bounds (``relation`` in src/lumen/geometry/ownership.py: interval bounds over bisected boxes, never
    sampling)."""  # noqa: D205, D209
    cb = np.array([[(lb.hi if (q >> a) & 1 else lb.lo)[a] for a in range(3)] for q in range(8)]) @ pb.R.T + pb.t
    ca = (cb - pa.t) @ pa.R  # b's box corners in a's frame
    rlo, rhi = np.maximum(la.lo, ca.min(0)), np.minimum(la.hi, ca.max(0))
    if np.any(rlo >= rhi):
        return True
    todo = [(rlo, rhi, 0)]
    while todo:
        clo, chi, dp = todo.pop()
        if _solid_interval(la, clo, chi) == -1 or _solid_interval(lb, *_local_box(pb, *_world_box(pa, clo, chi))) == -1:
            continue
        if dp >= depth:
            return False
        ax = int(np.argmax(chi - clo))
        mid = 0.5 * (clo[ax] + chi[ax])
        h1, l2 = chi.copy(), clo.copy()
        h1[ax], l2[ax] = mid, mid
        todo += [(clo, h1, dp + 1), (l2, chi, dp + 1)]
    return True


def _world_box(p: Placed, lo, hi):
    """Return the world box enclosing the box [lo, hi] of placement p's frame."""
    c, r = 0.5 * (lo + hi), 0.5 * (hi - lo)
    return p.R @ c + p.t - np.abs(p.R) @ r, p.R @ c + p.t + np.abs(p.R) @ r


def _proved_within(pv: Placed, pm: Placed, lv: Lowered, lm: Lowered, tol: float, depth: int = 7) -> bool:
    """Whether solid v (its box shrunk by ``tol``) lies inside solid m: the corner proof for a convex m, else every
    cell of a bisection of v's box is proved outside v or inside m by interval bounds (src/lumen/geometry/ownership.py
    :679 _clips: the unit's box shrunk by the contact tolerance, then the containment proof)."""  # noqa: D205, D209
    if _proved_inside(pv, pm, lv, lm, tol):
        return True
    lo, hi = np.minimum(lv.lo + tol, lv.hi - tol), np.maximum(lv.hi - tol, lv.lo + tol)
    todo = [(lo, hi, 0)]
    while todo:
        clo, chi, dp = todo.pop()
        if _solid_interval(lv, clo, chi) == -1 or _solid_interval(lm, *_local_box(pm, *_world_box(pv, clo, chi))) == 1:
            continue
        if dp >= depth:
            return False
        ax = int(np.argmax(chi - clo))
        mid = 0.5 * (clo[ax] + chi[ax])
        h1, l2 = chi.copy(), clo.copy()
        h1[ax], l2[ax] = mid, mid
        todo += [(clo, h1, dp + 1), (l2, chi, dp + 1)]
    return True


def clips_of(placed: list, kinds: list, kind_of: dict, tol: float) -> list:
    """Return per volume the ancestors it is not proved to lie inside (src/lumen/geometry/ownership.py:679 _clips):
    its mother and those of its mother's clips, each a candidate whose face is the volume's exit."""  # noqa: D205, D209
    low = [kinds[kind_of[id(p.lv.solid)]] for p in placed]
    clips = [[] for _ in placed]
    for v, p in enumerate(placed):  # parents first (the walk's order)
        if p.parent < 0:
            continue
        for m in [p.parent, *clips[p.parent]]:
            if not _proved_within(p, placed[m], low[v], low[m], tol):
                clips[v].append(m)
    return clips


def ownership(placed: list, kinds: list, kind_of: dict, lo_w, hi_w, tol: float):
    """Return (prio, owners) of the placed volumes (src/lumen/geometry/ownership.py:744 resolve, without protrusion
    clips): one owner per point, level by level. Among siblings the rule's order puts a volume proved inside a sibling
    ahead of it, else keeps the placement order; ``prio`` is the depth-first order of the tree with each mother's
    daughters in that order (lower first). ``owners[v]``: the siblings ahead of v whose world boxes meet v's deeper
    than the contact tolerance, and those of v's ancestors' siblings ahead of them that meet v (a candidate entered as a
    daughter: where it holds a point, the point is not v's)."""  # noqa: D205, D209
    n = len(placed)
    kids = [[] for _ in range(n + 1)]
    for i, p in enumerate(placed):
        kids[p.parent if p.parent >= 0 else n].append(i)
    low = [kinds[kind_of[id(p.lv.solid)]] for p in placed]
    lo_w, hi_w = np.asarray(lo_w, np.float64), np.asarray(hi_w, np.float64)

    def meets(a, bs):  # the siblings bs whose boxes meet a's deeper than the contact tolerance
        bs = np.asarray(bs, np.int64)
        if not len(bs):
            return bs
        d = np.minimum(hi_w[bs], hi_w[a]) - np.maximum(lo_w[bs], lo_w[a])
        return bs[(d > tol).all(1)]

    linked = {}  # (a, b) -> the solids may share a point (boxes meet, not proved apart)

    def link(a, b):
        k = (min(a, b), max(a, b))
        if k not in linked:
            linked[k] = not _proved_apart(placed[a], placed[b], low[a], low[b])
        return linked[k]

    order_of = {}
    for ks in kids:
        n_in = {a: 0 for a in ks}
        for a in ks:  # how many siblings a is proved inside (only a sibling whose box meets a's can hold it)
            for b in meets(a, [b for b in ks if b != a]):
                n_in[a] += _proved_inside(placed[a], placed[int(b)], low[a], low[int(b)], tol)
        for r, a in enumerate(sorted(ks, key=lambda a: (-n_in[a], a))):
            order_of[a] = r
    prio = np.zeros(n + 1, np.int64)
    count = 0

    def walk(v):
        nonlocal count
        for a in sorted(kids[v], key=lambda a: order_of[a]):
            prio[a] = count
            count += 1
            walk(a)

    walk(n)
    prio[n] = count
    owners = [[] for _ in range(n)]
    for ks in kids:
        for a in ks:
            for b in meets(a, [b for b in ks if b != a and order_of[b] < order_of[a]]):
                if link(a, int(b)):
                    owners[a].append(int(b))
    for v in range(n):  # below a non-owner: the owners of an ancestor that may meet v too
        u = placed[v].parent
        while u >= 0:
            for b in meets(v, [b for b in owners[u] if b not in owners[v]]):
                if link(v, int(b)):
                    owners[v].append(int(b))
            u = placed[u].parent
    return prio, owners


def navigator_arrays(placed: list, vol_cls, outside_cls: int, vol_sensor, prio=None, meshes=(), mesh_cls=(),
                     use_frame_groups=True) -> dict:
    """Return the navigator's flat arrays (include/lumen_b200.h layouts) of the placed volumes and ``meshes``
    [(world triangles, mother)] of classes ``mesh_cls``: navigator ids 0 .. n - 1 the volumes, n the outside, n + 1 + k
    mesh k's pseudo-volume, CH0 + c (CH0 = n + 1 + meshes) chunk c, an item of its mesh's mother; every id has a
    vol_i row (a mesh's and its chunks' carry its class, mother and rank)."""  # noqa: D205, D209
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
            if lf.torus is not None:  # typ 2: M at the quadric's A, R and r after it
                leaf_f.append(np.concatenate([lf.og, lf.og, lf.M.ravel(), [lf.torus[0], lf.torus[1], 0.0, 0.0, 0.0]]))
                leaf_i.append([2, len(plane_f), 0, 0])
                continue
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
    nm = len(meshes)
    mc = mesh_chunks(meshes)
    nch = len(mc["chunk"])
    ch0 = n + 1 + nm
    kids = [[] for _ in range(n + 1)]
    for i, p in enumerate(placed):
        kids[p.parent if p.parent >= 0 else n].append(i)
    for c in range(nch):  # each chunk: an item of its mesh's mother (Geant4: not of the volumes below it)
        kids[int(mc["mother"][c])].append(ch0 + c)
    scale = float(np.max(np.abs(np.concatenate([lo_w, hi_w])))) if n else 1.0
    tol = K_ON * (BAND_ULPS_EPS * scale + BAND_FLOOR)  # the contact tolerance: a contact is no overlap
    size = np.ones(n, np.int64)
    for v in range(n - 1, -1, -1):  # the walk is depth first: a subtree is its root and the size - 1 volumes after it
        if placed[v].parent >= 0:
            size[placed[v].parent] += size[v]
    own_prio, owners = ownership(placed, kinds, kind_of, lo_w, hi_w, tol)
    clips = clips_of(placed, kinds, kind_of, tol)
    for v in range(n):  # an owner is a candidate of its non-owner, an ancestor v reaches out of too (its face an
        kids[v].extend(owners[v])  # exit: src/lumen/geometry/navigator_build.py:442)
        kids[v].extend(clips[v])
    prio = own_prio if prio is None else np.asarray(prio)
    prio = np.concatenate([prio[:n + 1], n + 1 + np.arange(nm)])
    # boxes per navigator id (the volumes', then zero for the outside and the meshes, then the chunks')
    lo_w = np.concatenate([lo_w, np.zeros((1 + nm, 3)), mc["lo"]])
    hi_w = np.concatenate([hi_w, np.zeros((1 + nm, 3)), mc["hi"]])
    vol_i = np.zeros((ch0 + nch, 10), np.int32)
    cand, node_f, node_i, items = [], [], [], []
    fgroups = []  # (volume, first node, end node, R, members' group-frame boxes lo, hi)
    low_all = [kinds[kind_of[id(p.lv.solid)]] for p in placed]
    for v in range(n + 1, ch0 + nch):  # the meshes' and their chunks' rows: class, mother, rank; no solid, no BVH
        k = v - n - 1 if v < ch0 else int(mc["chunk"][v - ch0, 2])
        vol_i[v, 0] = -1
        vol_i[v, 1] = int(meshes[k][1]) if int(meshes[k][1]) >= 0 else n
        vol_i[v, 2] = mesh_cls[k]
        vol_i[v, 3] = -1
        vol_i[v, 4] = prio[n + 1 + k]
    for v in range(n + 1):
        ks = kids[v]
        vol_i[v, 0] = kind_of[id(placed[v].lv.solid)] if v < n else -1
        vol_i[v, 1] = (placed[v].parent if placed[v].parent >= 0 else n) if v < n else -1
        vol_i[v, 2] = vol_cls[v] if v < n else outside_cls
        vol_i[v, 3] = vol_sensor[v] if v < n else -1
        vol_i[v, 4] = prio[v]
        vol_i[v, 5], vol_i[v, 6] = len(cand), len(ks)
        vol_i[v, 9] = size[v] if v < n else 1  # the volumes of its subtree (an ancestor of w: v < w < v + size)
        cand.extend(ks)
        # the daughters' BVH, in the float32 boxes the engine reads (the frame groups' own BVHs after it)
        lo32 = lo_w.astype(np.float32).astype(np.float64)
        hi32 = hi_w.astype(np.float32).astype(np.float64)
        wks, grp = frame_groups(ks, placed, low_all, lo_w, hi_w, n) if use_frame_groups and v < n + 1 else (ks, [])
        nodes, order = _bvh(np.asarray(wks, np.int64), lo32, hi32)
        base, ibase = len(node_f), len(items)
        vol_i[v, 7] = base
        for nd in nodes:
            node_f.append([*nd[0], *nd[1]])
            node_i.append([base + nd[2], nd[3], ibase + nd[4] if nd[3] else 0, 0])
        items.extend(order)
        vol_i[v, 8] = len(node_f)
        for R, mem in grp:  # a frame group: its BVH over the members' boxes in the group frame
            glo, ghi = group_boxes(R, mem, placed, low_all)
            gl, gh = np.zeros_like(lo_w), np.zeros_like(hi_w)
            gl[mem], gh[mem] = glo, ghi
            gnodes, gorder = _bvh(np.asarray(mem, np.int64), gl.astype(np.float32).astype(np.float64),
                                  gh.astype(np.float32).astype(np.float64))  # fmt: skip
            gb, gib = len(node_f), len(items)
            for nd in gnodes:
                node_f.append([*nd[0], *nd[1]])
                node_i.append([gb + nd[2], nd[3], gib + nd[4] if nd[3] else 0, 0])
            items.extend(gorder)
            fgroups.append((v, gb, len(node_f), R, gl, gh))
    ni_arr = np.asarray(node_i, np.int32).reshape(-1, 4)
    for _, g0, g1, _, _, _ in fgroups:
        if bvh_depth(ni_arr, g0, g1) > MAX_BVH_DEPTH:
            raise ValueError(f"a frame group's BVH deeper than {MAX_BVH_DEPTH} levels")
    for v in range(n + 1):
        if bvh_depth(ni_arr, vol_i[v, 7], vol_i[v, 8]) > MAX_BVH_DEPTH:
            raise ValueError(f"volume {v}: a daughter BVH deeper than {MAX_BVH_DEPTH} levels")
    for v in range(n + 1, ch0 + nch):
        vol_i[v, 5], vol_i[v, 7], vol_i[v, 8] = len(cand), len(node_f), len(node_f)
    allp = np.concatenate([lo_w[:n], hi_w[:n], mc["lo"], mc["hi"]]) if n else np.zeros((1, 3))
    reach = float(np.linalg.norm(allp.max(0) - allp.min(0)))
    items_a = np.asarray(items, np.int64)
    node64 = _node_boxes64(ni_arr, items_a, lo_w, hi_w)
    for _, g0, g1, _, gl, gh in fgroups:  # a group's nodes over its members' group-frame boxes
        _node_boxes64(ni_arr, items_a, gl, gh, g0, g1, node64)
    return dict(
        n_vol=n, vol_i=vol_i, vol_f=vol_f.astype(np.float32), cand=np.asarray(cand, np.int32),
        # the float64 navigator's arrays (LUMEN_PREC_FLOAT64): the same geometry in float64, the BVH's topology shared
        vol_f64=vol_f.copy(), leaf_f64=np.asarray(leaf_f, np.float64).reshape(-1, 20),
        plane_f64=np.asarray(plane_f, np.float64).reshape(-1, 4),
        node_f64=node64,
        # frame groups: per group (volume, first node, end node, 0) and its frame R (row-major, x_g = R^T x_w)
        n_group=len(fgroups), group_i=np.asarray([[g[0], g[1], g[2], 0] for g in fgroups], np.int32).reshape(-1, 4),
        group_r=np.asarray([g[3].ravel() for g in fgroups], np.float32).reshape(-1, 9),
        group_r64=np.asarray([g[3].ravel() for g in fgroups], np.float64).reshape(-1, 9),
        node_f=np.asarray(node_f, np.float32).reshape(-1, 6), node_i=np.asarray(node_i, np.int32).reshape(-1, 4),
        items=np.asarray(items, np.int32), kind_i=np.asarray(kind_i, np.int32).reshape(-1, 4),
        leaf_f=np.asarray(leaf_f, np.float32).reshape(-1, 20), leaf_i=np.asarray(leaf_i, np.int32).reshape(-1, 4),
        plane_f=np.asarray(plane_f, np.float32).reshape(-1, 4), prog_i=np.asarray(prog_i, np.int32).reshape(-1, 2),
        reach=reach, names=[p.name for p in placed],
        # the meshes: triangles (V0, V1, V2, unit normal), chunks (first triangle, count, mesh, 0) and their boxes
        n_mesh=nm, ch0=ch0, mesh_tri=mc["tri"].astype(np.float32), mesh_tri64=mc["tri"].copy(),
        mesh_chunk=mc["chunk"].astype(np.int32), chunk_box=np.concatenate([mc["lo"], mc["hi"]], 1).astype(np.float32),
        chunk_box64=np.concatenate([mc["lo"], mc["hi"]], 1),
    )  # fmt: skip
