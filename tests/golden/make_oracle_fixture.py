"""Golden navigator data from the reference's own float64 geometry referee (run where the reference is mounted).

    python tests/golden/make_oracle_fixture.py /path/to/lumen    # writes tests/golden/oracle_<detector>.npz

For the benchmark detectors (the 2000-PMT cylinder tank, the LAr CSG box) and the solids box, the detector
description of ``lumen_b200.detectors`` is rebuilt as the reference's own ``lumen.geometry.scene.Scene`` with the
reference's solid constructors (``lumen.geometry.solids.g4_*``: Geant4's solids as the reference lowers them, the
booleans as its ``Op`` / ``Xf`` nodes), and ``lumen.compare.oracle.Oracle`` (src/lumen/compare/oracle.py:208) labels
4000 points and takes the first visible change along 800 rays from random starts, as the reference's own navigator
tests do (tests/unit/test_navigator.py:43-59, tests/unit/nav_toys.py:268 ``_agree``). The labels are (medium, sensor):
the medium an index into the fixture's material names (the outside: -1), the sensor this build's sensor index (each
sensor placement is a definition of its own in the Scene, so that the referee reports that index).

The reference's modules are imported under the numpy-backed ``jax`` stub of ``make_golden.py``; the referee is host
numpy in float64 and needs nothing else of JAX. Beside each fixture, ``refscene_<detector>.json.gz`` holds the same Scene
as the reference flattens it (``lumen_b200.reference.export_scene``): the navigator rebuilt from the reference's own
leaves is checked against the referee too.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

N_POINTS, N_RAYS, T_START = 4000, 800, 1e-9  # T_START: the referee's start (tests/unit/nav_toys.py:15 T_ORC)


def capture(make):
    """Run a ``lumen_b200.detectors`` builder and return (its top Volume, materials, sensors spec, Detector)."""
    from lumen_b200 import detector as D

    seen = {}
    real = D.build

    def spy(top, materials, **kw):
        seen.update(top=top, materials=materials, kw=kw)
        return real(top, materials, **kw)

    D.build = spy
    try:
        det = make()
    finally:
        D.build = real
    return seen["top"], seen["materials"], seen["kw"].get("sensors", {}), det


def ref_solid(s):
    """The reference's solid node of one of this build's solids (the same Geant4 solid, the reference's lowering)."""
    from lumen.geometry import solids as so

    from lumen_b200 import geometry as G

    two_pi = 2.0 * np.pi
    if isinstance(s, G.Box):
        return so.g4_box(2 * s.hx, 2 * s.hy, 2 * s.hz)
    if isinstance(s, G.Tube):
        return so.g4_tube(s.rmin, s.rmax, 2 * s.dz, s.sphi, s.dphi)
    if isinstance(s, G.Sphere):
        theta = (0.0, np.pi) if s.hemisphere == 0 else ((0.0, 0.5 * np.pi) if s.hemisphere > 0 else (0.5 * np.pi,
                                                                                                      0.5 * np.pi))
        return so.g4_sphere(0.0, s.rmax, (0.0, two_pi), theta)
    if isinstance(s, G.SphereShell):
        return so.g4_sphere(s.rmin, s.rmax, (s.sphi, s.dphi), (s.stheta, s.dtheta))
    if isinstance(s, G.Torus):
        return so.g4_torus(s.rmin, s.rmax, s.rtor, s.sphi, s.dphi)
    if isinstance(s, G.Cons):
        return so.g4_cone(s.rmin1, s.rmax1, s.rmin2, s.rmax2, 2 * s.dz, (s.sphi, s.dphi))
    if isinstance(s, G.Orb):
        return so.g4_orb(s.r)
    if isinstance(s, G.Ellipsoid):
        return so.g4_ellipsoid(s.ax, s.by, s.cz, s.zcut1, s.zcut2)
    if isinstance(s, G.EllipticalTube):
        return so.g4_eltube(s.dx, s.dy, s.dz)
    if isinstance(s, G.EllipticalCone):
        return so.g4_elcone(s.dx, s.dy, s.zmax, s.zcut)
    if isinstance(s, G.Paraboloid):
        return so.g4_paraboloid(s.rlo, s.rhi, s.dz)
    if isinstance(s, G.Hype):
        return so.g4_hype(s.rmin, s.rmax, s.inst, s.outst, 2 * s.dz)
    if isinstance(s, G.Polycone):
        return so.g4_polycone(s.sphi, s.dphi, s.zplanes)
    if isinstance(s, G.Polyhedra):
        return so.g4_polyhedra(s.sphi, s.dphi, s.nsides, s.zplanes)
    if isinstance(s, G.Trd):
        return so.g4_trd(2 * s.dx1, 2 * s.dx2, 2 * s.dy1, 2 * s.dy2, 2 * s.dz)
    if isinstance(s, G.Para):
        return so.g4_para(2 * s.dx, 2 * s.dy, 2 * s.dz, s.alpha, s.theta, s.phi)
    if isinstance(s, G.Trap):
        return so.g4_trap(2 * s.dz, s.theta, s.phi, (2 * s.dy1, 2 * s.dx1, 2 * s.dx2, s.alpha1),
                          (2 * s.dy2, 2 * s.dx3, 2 * s.dx4, s.alpha2))  # fmt: skip
    if isinstance(s, G.Tet):
        return so.g4_tet(s.v1, s.v2, s.v3, s.v4)
    if isinstance(s, G.Boolean):
        op = {"union": "union", "intersection": "inter", "subtraction": "sub"}[s.op]
        R = np.eye(3) if s.rot is None else np.asarray(s.rot, float)
        return so.Op(op, ref_solid(s.a), so.Xf(R, np.asarray(s.pos, float), ref_solid(s.b)))
    raise NotImplementedError(f"no reference solid for {type(s).__name__}")


def ref_scene(top, materials, sensors):
    """The reference's Scene of a Volume tree; returns (scene, material names). Each placement of a sensor volume is
    a definition of its own whose label carries this build's sensor index (placements in depth-first order)."""  # noqa: D205
    from lumen.geometry import scene as sc

    from lumen_b200 import geometry as G

    mats = sorted(materials)
    med = {m: i for i, m in enumerate(mats)}
    sensor_lv = set(sensors.values())
    defs = {}
    placed = G.flatten(top)
    sensor_of = {}  # id(placement) -> sensor index, in the flattened order the detector numbers its sensors by
    k = 0

    def walk(lv):
        nonlocal k
        for pl in lv.daughters:
            if pl.volume.name in sensor_lv:
                sensor_of[id(pl)] = k
                k += 1
            walk(pl.volume)

    walk(top)
    assert k == sum(1 for p in placed if p.lv.name in sensor_lv)

    def define(lv, sensor=-1, tag=""):
        name = lv.name + tag
        if name in defs:
            return name
        d = sc.Definition(name, sc.Member(ref_solid(lv.solid), sc.Label(med[lv.material], sensor, lv.name)),
                          origin=lv.name)  # fmt: skip
        defs[name] = d
        for pl in lv.daughters:
            s = sensor_of.get(id(pl), -1)
            child = define(pl.volume, s, f"#{s}" if s >= 0 else "")
            d.placements.append(sc.Placement(child, R=np.asarray(pl.rot, float), t=np.asarray(pl.pos, float),
                                             name=pl.name))  # fmt: skip
        return name

    root = define(top)
    return sc.Scene(defs, root, sc.Label(-1, -1, "outside")), mats


def box_of(top):
    low = top.solid.lower()
    return np.asarray(low.lo, float), np.asarray(low.hi, float)


def dump(name, make, seed):
    from lumen.compare.oracle import Oracle

    top, materials, sensors, det = capture(make)
    scene, mats = ref_scene(top, materials, sensors)
    orc = Oracle(scene)
    lo, hi = box_of(top)
    rng = np.random.default_rng(seed)
    X = rng.uniform(lo, hi, (N_POINTS, 3))
    med, sen = orc.label(X)
    O_ = rng.uniform(lo + 0.02 * (hi - lo), hi - 0.02 * (hi - lo), (N_RAYS, 3)).astype(np.float32).astype(float)
    D_ = rng.normal(size=(N_RAYS, 3))
    D_ /= np.linalg.norm(D_, axis=1, keepdims=True)
    D_ = D_.astype(np.float32).astype(float)
    tmax = float(2.0 * np.linalg.norm(hi - lo))
    hit = np.zeros(N_RAYS, bool)
    t = np.zeros(N_RAYS)
    amed = np.zeros(N_RAYS, np.int64)
    asen = np.zeros(N_RAYS, np.int64)
    bmed = np.zeros(N_RAYS, np.int64)
    amb = np.zeros(N_RAYS, bool)
    for i in range(N_RAYS):
        r = orc.query(O_[i], D_[i], T_START, tmax, push=0.0)
        hit[i], t[i] = r["hit"], r["t"]
        amed[i], asen[i] = r["after"]
        bmed[i] = r["before"][0]
        amb[i] = r["ambiguous"]
    placements = [(p.name, p.lv.material) for p in G_flatten(top)]
    np.savez_compressed(os.path.join(HERE, f"oracle_{name}.npz"), X=X, med=np.asarray(med, np.int64),
                        sen=np.asarray(sen, np.int64), O=O_, D=D_, tmax=tmax, hit=hit, t=t, after_med=amed,
                        after_sen=asen, before_med=bmed, ambiguous=amb, materials=np.asarray(mats),
                        place_names=np.asarray([p[0] for p in placements]),
                        place_mats=np.asarray([p[1] for p in placements]))  # fmt: skip
    from lumen_b200 import reference

    solids, volumes = reference.export_scene(scene)  # the same Scene, flattened by the reference for lumen_b200.reference
    reference.save({"solids": solids, "volumes": volumes}, os.path.join(HERE, f"refscene_{name}.json.gz"))
    print(f"{name}: {len(scene.definitions)} definitions, {int(hit.sum())}/{N_RAYS} rays hit, "
          f"{int((sen >= 0).sum())} points in sensors")


def G_flatten(top):
    from lumen_b200 import geometry as G

    return G.flatten(top)


def main(ref_root):
    from make_golden import install_stub, register_lumen

    install_stub()
    register_lumen(os.path.join(ref_root, "src"))
    from lumen_b200 import detectors

    dump("cylinder_tank", detectors.cylinder_tank, 1)
    dump("lar_box", detectors.lar_box, 2)
    dump("solids_box", detectors.solids_box, 3)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <path of the lumen source tree (the directory holding src/lumen)>")
    main(sys.argv[1])
