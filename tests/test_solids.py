"""The Geant4 solid catalogue (src/lumen/geometry/solids.py:477-772) lowered to quadric, plane and torus leaves: the
checker's locate against each solid's own membership written from its definition (float64), at random points of a
placed, rotated copy, away from its surface (the membership the same at the point and 1e-4 either side of it on
every axis); the torus's first crossings against the roots of its quartic."""

import math

import numpy as np
import pytest
from scipy.spatial import Delaunay

import oracle
from lumen_b200 import geometry as G
from lumen_b200 import optics as O
from lumen_b200.detector import build

POS = np.array([0.2, -0.1, 0.3])
ROT = G.rotation("x", 30.0) @ G.rotation("z", 20.0)


def _placed(solid):
    top = G.Volume("World", G.Box(3, 3, 3), "Water")
    top.place(G.Volume("S", solid, "Glass"), POS, ROT, name="S")
    return build(top, {"Water": O.Material("Water", rindex=1.33), "Glass": O.Material("Glass", rindex=1.5)})


def _phi_in(x, y, s, d):
    return (d >= 2 * math.pi - 1e-12) | (np.mod(np.arctan2(y, x) - s, 2 * math.pi) <= d)


def _hull(verts):
    h = Delaunay(np.asarray(verts, float))
    return lambda p: h.find_simplex(p) >= 0


def _zlin(z, zs, vs):
    return np.interp(z, zs, vs)


CASES = {
    "cons": (G.Cons(0.1, 0.3, 0.05, 0.2, 0.4, 0.3, 4.0), lambda p: (
        (np.abs(p[:, 2]) <= 0.4) & (np.hypot(p[:, 0], p[:, 1]) <= _zlin(p[:, 2], [-0.4, 0.4], [0.3, 0.2]))
        & (np.hypot(p[:, 0], p[:, 1]) >= _zlin(p[:, 2], [-0.4, 0.4], [0.1, 0.05])) & _phi_in(p[:, 0], p[:, 1], 0.3, 4.0))),
    "sphere": (G.SphereShell(0.5, 0.2, 0.5, 2.0, 0.3, 1.5), lambda p: (
        (np.linalg.norm(p, axis=1) <= 0.5) & (np.linalg.norm(p, axis=1) >= 0.2) & _phi_in(p[:, 0], p[:, 1], 0.5, 2.0)
        & (np.arccos(np.clip(p[:, 2] / np.linalg.norm(p, axis=1), -1, 1)) >= 0.3)
        & (np.arccos(np.clip(p[:, 2] / np.linalg.norm(p, axis=1), -1, 1)) <= 1.8))),
    "sphere_wide": (G.SphereShell(0.5, 0.0, 1.0, 5.0, 1.2, 1.4), lambda p: (
        (np.linalg.norm(p, axis=1) <= 0.5) & _phi_in(p[:, 0], p[:, 1], 1.0, 5.0)
        & (np.arccos(np.clip(p[:, 2] / np.linalg.norm(p, axis=1), -1, 1)) >= 1.2)
        & (np.arccos(np.clip(p[:, 2] / np.linalg.norm(p, axis=1), -1, 1)) <= 2.6))),
    "orb": (G.Orb(0.3), lambda p: np.linalg.norm(p, axis=1) <= 0.3),
    "ellipsoid": (G.Ellipsoid(0.3, 0.2, 0.4, -0.2, 0.3), lambda p: (
        ((p[:, 0] / 0.3) ** 2 + (p[:, 1] / 0.2) ** 2 + (p[:, 2] / 0.4) ** 2 <= 1) & (p[:, 2] >= -0.2) & (p[:, 2] <= 0.3))),
    "eltube": (G.EllipticalTube(0.3, 0.2, 0.4), lambda p: (
        ((p[:, 0] / 0.3) ** 2 + (p[:, 1] / 0.2) ** 2 <= 1) & (np.abs(p[:, 2]) <= 0.4))),
    "elcone": (G.EllipticalCone(0.5, 0.3, 0.6, 0.4), lambda p: (
        ((p[:, 0] / 0.5) ** 2 + (p[:, 1] / 0.3) ** 2 <= (0.6 - p[:, 2]) ** 2) & (np.abs(p[:, 2]) <= 0.4))),
    "paraboloid": (G.Paraboloid(0.1, 0.3, 0.3), lambda p: (
        (p[:, 0] ** 2 + p[:, 1] ** 2 <= (0.09 - 0.01) / 0.6 * p[:, 2] + 0.05) & (np.abs(p[:, 2]) <= 0.3))),
    "hype": (G.Hype(0.1, 0.3, 0.3, 0.5, 0.4), lambda p: (
        (p[:, 0] ** 2 + p[:, 1] ** 2 <= 0.09 + math.tan(0.5) ** 2 * p[:, 2] ** 2)
        & (p[:, 0] ** 2 + p[:, 1] ** 2 >= 0.01 + math.tan(0.3) ** 2 * p[:, 2] ** 2) & (np.abs(p[:, 2]) <= 0.4))),
    "polycone": (G.Polycone(((0.0, 0.2, -0.3), (0.05, 0.3, 0.0), (0.0, 0.1, 0.3)), 0.2, 5.0), lambda p: (
        (np.abs(p[:, 2]) <= 0.3) & _phi_in(p[:, 0], p[:, 1], 0.2, 5.0)
        & (np.hypot(p[:, 0], p[:, 1]) <= _zlin(p[:, 2], [-0.3, 0.0, 0.3], [0.2, 0.3, 0.1]))
        & (np.hypot(p[:, 0], p[:, 1]) >= _zlin(p[:, 2], [-0.3, 0.0, 0.3], [0.0, 0.05, 0.0])))),
    "trd": (G.Trd(0.2, 0.1, 0.3, 0.2, 0.4), _hull([(-0.2, -0.3, -0.4), (0.2, -0.3, -0.4), (-0.2, 0.3, -0.4),
                                                   (0.2, 0.3, -0.4), (-0.1, -0.2, 0.4), (0.1, -0.2, 0.4),
                                                   (-0.1, 0.2, 0.4), (0.1, 0.2, 0.4)])),
    "tet": (G.Tet((0, 0, 0), (0.3, 0, 0), (0, 0.3, 0), (0, 0, 0.3)),
            _hull([(0, 0, 0), (0.3, 0, 0), (0, 0.3, 0), (0, 0, 0.3)])),
    "torus": (G.Torus(0.2, 0.5, 0.1, 0.5, 4.5), lambda p: (
        ((np.hypot(p[:, 0], p[:, 1]) - 0.5) ** 2 + p[:, 2] ** 2 <= 0.04)
        & ((np.hypot(p[:, 0], p[:, 1]) - 0.5) ** 2 + p[:, 2] ** 2 >= 0.01) & _phi_in(p[:, 0], p[:, 1], 0.5, 4.5))),
    "para": (G.Para(0.2, 0.3, 0.4, 0.2, 0.3, 0.5), _hull([
        (sx * 0.2 + sy * 0.3 * math.tan(0.2) + sz * 0.4 * math.tan(0.3) * math.cos(0.5),
         sy * 0.3 + sz * 0.4 * math.tan(0.3) * math.sin(0.5), sz * 0.4)
        for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)])),
    "trap": (G.Trap(0.4, 0.2, 0.3, 0.3, 0.2, 0.26, 0.1, 0.2, 0.15, 0.19, 0.1), _hull([
        (s * 0.4 * math.tan(0.2) * math.cos(0.3) + sy * dy * math.tan(0.1) + sx * (xa if sy < 0 else xb),
         s * 0.4 * math.tan(0.2) * math.sin(0.3) + sy * dy, s * 0.4)
        for s, dy, xa, xb in ((-1, 0.3, 0.2, 0.26), (1, 0.2, 0.15, 0.19)) for sy in (-1, 1) for sx in (-1, 1)])),
    "generic_trap": (G.GenericTrap(((-0.2, -0.2), (0.2, -0.2), (0.2, 0.2), (-0.2, 0.2), (-0.1, -0.1), (0.1, -0.1),
                                    (0.1, 0.1), (-0.1, 0.1)), 0.3),
                     _hull([(x, y, -0.3) for x in (-0.2, 0.2) for y in (-0.2, 0.2)]
                           + [(x, y, 0.3) for x in (-0.1, 0.1) for y in (-0.1, 0.1)])),
    "tube_phi": (G.Tube(0.4, 0.3, 0.1, 1.0, 2.0), lambda p: (
        (np.abs(p[:, 2]) <= 0.3) & (np.hypot(p[:, 0], p[:, 1]) <= 0.4) & (np.hypot(p[:, 0], p[:, 1]) >= 0.1)
        & _phi_in(p[:, 0], p[:, 1], 1.0, 2.0))),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_locate_matches_the_solid(name):
    solid, member = CASES[name]
    det = _placed(solid)
    rng = np.random.default_rng(3)
    low = solid.lower()
    pl = rng.uniform(low.lo - 0.1, low.hi + 0.1, (40000, 3))  # the solid's frame, about its box
    pw = pl @ ROT.T + POS
    pl = (pw.astype(np.float32).astype(np.float64) - POS) @ ROT
    m = member(pl)
    sure = m.copy() == m
    for a in range(3):
        for s in (-1e-4, 1e-4):
            q = pl.copy()
            q[:, a] += s
            sure &= member(q) == m
    v = oracle.locate(det, pw.astype(np.float32))
    assert m[sure].sum() > 500 and (~m[sure]).sum() > 500
    bad = np.flatnonzero(((v == 1) != m) & sure)
    assert len(bad) == 0, f"{name}: {len(bad)} points differ, first {pl[bad[:3]]}"


def test_a_twisted_trap_is_refused():
    with pytest.raises(ValueError):  # its x-faces' slopes differ at the two ends: not planar
        G.Trap(0.4, 0.2, 0.3, 0.3, 0.2, 0.25, 0.1, 0.2, 0.15, 0.2, 0.1).lower()


def test_torus_first_crossings_are_the_quartic_roots():
    R, r = 0.8, 0.25
    det = _placed(G.Torus(rmax=r, rtor=R))
    rng = np.random.default_rng(1)
    o = rng.uniform(-1.5, 1.5, (1500, 3))
    d = rng.normal(size=(1500, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    oi, of = oracle.query(det, o, d)
    ol, dl = (o - POS) @ ROT, d @ ROT
    pp = np.polynomial.polynomial
    hits = 0
    for i in range(len(o)):
        a, b = ol[i], dl[i]
        sq = lambda k: pp.polymul([a[k], b[k]], [a[k], b[k]])  # noqa: E731
        xy = pp.polyadd(sq(0), sq(1))
        q = pp.polyadd(pp.polyadd(xy, sq(2)), [R * R - r * r])
        rts = np.roots(pp.polysub(pp.polymul(q, q), 4 * R * R * xy)[::-1])
        rts = rts[(np.abs(rts.imag) < 1e-7) & (rts.real > 1e-6)].real
        t_world = float(np.min((np.sign(d[i]) * 3 - o[i]) / d[i]))
        want = min(rts.min() if len(rts) else t_world, t_world)
        hits += bool(len(rts)) and rts.min() < t_world
        assert abs(of[i, 0] - want) < 2e-5 * (1 + want), (i, of[i, 0], want)
    assert hits > 150
