"""The navigator against the reference's own float64 geometry referee on the benchmark detectors.

``tests/golden/make_oracle_fixture.py`` rebuilt the 2000-PMT cylinder tank, the LAr CSG box and the solids box as the
reference's ``Scene`` with the reference's solid constructors and recorded ``lumen.compare.oracle.Oracle``'s labels
of 4000 points and first visible changes along 800 rays (src/lumen/compare/oracle.py:208). Here the checker's
navigator (the CPU restatement the engine is bit-exact with) locates the same points and queries the same rays, at
the reference's own thresholds (tests/unit/test_navigator.py:43-59): at most 2 of 4000 points labelled otherwise, and
at most 0.2 % of the rays disagreeing on hit, t (within 2e-5 (1 + t), nav_toys.py:268 ``_agree``) or the label after.
A label is (material, sensor); the GPU's answers are compared to the same data in ``tests/test_gpu_parity.py``.
"""

import os

import numpy as np
import pytest

import oracle
from lumen_b200 import detectors

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MAKERS = {"cylinder_tank": detectors.cylinder_tank, "lar_box": detectors.lar_box, "solids_box": detectors.solids_box}


def load(name):
    f = np.load(os.path.join(GOLD, f"oracle_{name}.npz"))
    return {k: f[k] for k in f.files}


def labels_of(det, g, vol):
    """(material index in the fixture's list, sensor) of navigator volumes (-1, -1: the outside)."""
    mats = list(g["materials"])
    by_name = dict(zip(g["place_names"], g["place_mats"], strict=True))
    med_of = np.array([mats.index(by_name[nm]) for nm in det.names] + [-1])
    sen_of = np.concatenate([det.arrays["vol_i"].reshape(-1, 10)[: len(det.names), 3], [-1]])
    v = np.asarray(vol, np.int64)
    return med_of[v], sen_of[v]


def compare(det, g, locate_fn, query_fn):
    """Locate and query mismatch counts against the fixture: (bad points, bad rays, rays)."""
    med, sen = labels_of(det, g, locate_fn(g["X"]))
    bad_pts = int(np.sum((med != g["med"]) | (sen != g["sen"])))
    vol0 = locate_fn(g["O"])
    oi, of = query_fn(g["O"], g["D"], vol0, float(g["tmax"]))
    hit = oi[:, 0].astype(bool)
    t = of[:, 0].astype(np.float64)
    amed, asen = labels_of(det, g, oi[:, 2])
    ok = hit == g["hit"]
    both = ok & hit
    ok[both] &= np.abs(t[both] - g["t"][both]) <= 2e-5 * (1.0 + np.abs(g["t"][both]))
    ok[both] &= (amed[both] == g["after_med"][both]) & (asen[both] == g["after_sen"][both])
    return bad_pts, int(np.sum(~ok)), len(ok)


@pytest.mark.parametrize("name", list(MAKERS))
def test_checker_navigator_matches_the_reference_referee(name):
    det = MAKERS[name]()
    g = load(name)
    bad_pts, bad_rays, n = compare(det, g, lambda x: oracle.locate(det, x),
                                   lambda o, d, v, tm: oracle.query(det, o, d, v, None, tm))  # fmt: skip
    assert bad_pts <= 2, (name, bad_pts)
    assert bad_rays <= 0.002 * n, (name, bad_rays, n)


def test_fixtures_exercise_the_detectors():
    """The data are not vacuous: points in sensors and in the solids, rays that hit sensors and walls."""
    for name in MAKERS:
        g = load(name)
        assert len(g["X"]) == 4000 and len(g["O"]) == 800
        assert g["hit"].sum() > 600
        assert len(np.unique(g["med"])) >= 2
    assert (load("cylinder_tank")["after_sen"] >= 0).sum() > 20  # rays ending on PMTs


@pytest.mark.parametrize("name", list(MAKERS))
def test_navigator_of_the_reference_leaves_matches_the_referee(name):
    """The same Scene as the reference flattens it (tests/golden/refscene_<detector>.json.gz: its ``solids.Compiled``
    leaves, one origin a solid, shared planes; its instance poses), rebuilt by ``lumen_b200.reference`` into this
    package's navigator arrays: the checker's labels and first changes against the referee's, at the same thresholds.
    This pins the converter's reading of every solid of the catalogue the three detectors hold (boxes, tubes, spheres,
    cones, tori, polycones, polyhedra, the convex polytopes and the booleans with placed operands)."""
    from lumen_b200 import reference

    x = reference.load_scene(os.path.join(GOLD, f"refscene_{name}.json.gz"))
    det = reference.scene_detector(x["solids"], x["volumes"])
    g = load(name)
    lab = np.asarray([v["label"] for v in x["volumes"]] + [[-1, -1]], np.int64)

    def labels(vol):
        v = np.asarray(vol, np.int64)
        return lab[v, 0], lab[v, 1]

    med, sen = labels(oracle.locate(det, g["X"]))
    bad_pts = int(np.sum((med != g["med"]) | (sen != g["sen"])))
    vol0 = oracle.locate(det, g["O"])
    oi, of = oracle.query(det, g["O"], g["D"], vol0, None, float(g["tmax"]))
    hit = oi[:, 0].astype(bool)
    t = of[:, 0].astype(np.float64)
    amed, asen = labels(oi[:, 2])
    ok = hit == g["hit"]
    both = ok & hit
    ok[both] &= np.abs(t[both] - g["t"][both]) <= 2e-5 * (1.0 + np.abs(g["t"][both]))
    ok[both] &= (amed[both] == g["after_med"][both]) & (asen[both] == g["after_sen"][both])
    assert bad_pts <= 2, (name, bad_pts)
    assert int(np.sum(~ok)) <= 0.002 * len(ok), (name, int(np.sum(~ok)))
