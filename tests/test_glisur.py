"""GLISUR facet paths (the checker's restatement of src/lumen/surfaces/facets.py:341-548 and
src/lumen/transport/surface_event.py:137): the facet draw M = n + r s, s uniform in the unit ball, r = 1 - polish.

- The dielectric path (each facet reflects or refracts with the Fresnel share of the photon's state, the media and
  normal swapped after a refraction that points back) against Geant4 11.3.0's G4OpBoundaryProcess on one flat
  interface: tests/golden/g4_glisur_dielectric.npz holds the reference's Geant4 histograms (tests/data/g4_boundary,
  extracted by tests/golden/make_g4_fixture.py) of the random-linear cases, compared by the reference's two-sample
  chi2 (tests/unit/test_g4_boundary.py:109 of the reference).
- The step draws the facets from the defensive cover (the shell of the ball with share 0.01) and weights the path by
  its exact density over the cover's: the weighted cover draws reproduce the exact draws' moments, and the path's
  score in r has mean 0 under the exact draw.
"""

import math
import os

import numpy as np
import pytest
from scipy import stats

import oracle

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "g4_glisur_dielectric.npz"))
P_MIN = 0.0027 / 400
Z_MAX = 4.0


def _random_linear(wi, n, seed):
    s = np.array([0.0, 1.0, 0.0])
    p = np.cross(np.asarray(wi, np.float64), s)
    phi = np.random.default_rng(seed).uniform(0.0, 2.0 * math.pi, n)[:, None]
    return (np.cos(phi) * p + np.sin(phi) * s).astype(np.float32)


def _wi(theta_deg):
    t = math.radians(theta_deg)
    return np.array([math.sin(t), 0.0, -math.cos(t)], np.float32)


@pytest.mark.parametrize("i", range(len(GOLD["names"])))
def test_glisur_dielectric_path_is_geant4s(i):
    wi = _wi(float(GOLD[f"c{i}_theta"]))
    n = 1 << 18
    wo, far, w, _, capped = oracle.glisur("dielectric", float(GOLD[f"c{i}_value"]), wi, _random_linear(wi, n, 7 + i),
                                          n1=float(GOLD[f"c{i}_n1"]), n2=float(GOLD[f"c{i}_n2"]), key=(0, 200 + i))
    assert capped == 0
    h = np.histogram2d(wo[:, 2], np.abs(np.arctan2(wo[:, 1], wo[:, 0])),
                       bins=[GOLD[f"c{i}_edges_z"], GOLD[f"c{i}_edges_phi"]])[0]  # fmt: skip
    g4, ours = np.ravel(GOLD[f"c{i}_hist"]).astype(np.float64), np.ravel(h)
    n1, n2 = g4.sum(), ours.sum()
    use = (g4 + ours) > 0
    c2 = float(np.sum((g4[use] / n1 - ours[use] / n2) ** 2 / ((g4[use] + ours[use]) / (n1 * n2))))
    assert stats.chi2.sf(c2, int(use.sum()) - 1) > P_MIN, (GOLD["names"][i], c2)
    # far: the path ends beyond the surface exactly where its last direction points there
    np.testing.assert_array_equal(far, wo[:, 2] < 0.0)


@pytest.mark.parametrize(("kind", "polish", "theta", "n1", "n2"),
                         [("metal", 0.3, 40.0, 1.0, 1.0), ("metal", 0.9, 75.0, 1.0, 1.0),
                          ("dielectric", 0.3, 60.0, 1.0, 1.67), ("dielectric", 0.6, 30.0, 1.5, 1.0)])  # fmt: skip
def test_cover_weights_reproduce_the_exact_draw(kind, polish, theta, n1, n2):
    wi = _wi(theta)
    n = 1 << 19
    er = _random_linear(wi, n, 3)
    wo_c, far_c, w_c, _, cap = oracle.glisur(kind, polish, wi, er, n1=n1, n2=n2, e=0.01, key=(1, 1))
    wo_x, far_x, w_x, dl, cap2 = oracle.glisur(kind, polish, wi, er, n1=n1, n2=n2, e=0.0, key=(2, 2))
    assert cap == 0 and cap2 == 0
    for f_c, f_x in ((wo_c[:, 2], wo_x[:, 2]), (wo_c[:, 2] ** 2, wo_x[:, 2] ** 2), (wo_c[:, 0], wo_x[:, 0]),
                     (far_c.astype(np.float64), far_x.astype(np.float64))):  # fmt: skip
        a = w_c.astype(np.float64) * f_c
        b = w_x.astype(np.float64) * f_x
        se = math.sqrt(a.var() / n + b.var() / n)
        assert abs(a.mean() - b.mean()) < Z_MAX * se + 1e-7, (a.mean(), b.mean(), se)
    sc = dl.astype(np.float64)[w_x > 0]  # the score of the exact path density in r has mean 0 under its draw
    assert abs(sc.mean()) < Z_MAX * sc.std() / math.sqrt(len(sc))


@pytest.mark.parametrize(("kind", "polish", "theta", "n1", "n2"),
                         [("metal", 0.3, 40.0, 1.0, 1.0), ("metal", 0.8, 70.0, 1.0, 1.0),
                          ("dielectric", 0.5, 50.0, 1.0, 1.5)])  # fmt: skip
def test_cover_score_matches_independent_differences(kind, polish, theta, n1, n2):
    """d/dpolish of path expectations: the cover draw's weight times the exact path density's score (the step's
    estimator) against central differences of independent exact draws at polish +- 0.02."""
    wi = _wi(theta)
    n = 1 << 21
    er = _random_linear(wi, n, 1)

    def feats(wo, far):
        return np.stack([wo[:, 2].astype(np.float64), wo[:, 0].astype(np.float64) ** 2, far.astype(np.float64)], 1)

    wo, far, w, dl, _ = oracle.glisur(kind, polish, wi, er, n1=n1, n2=n2, e=0.01, key=(3, 3))
    g = feats(wo, far) * (w.astype(np.float64) * -dl.astype(np.float64))[:, None]  # d r / d polish = -1
    h = 0.02
    fp = feats(*oracle.glisur(kind, polish + h, wi, er, n1=n1, n2=n2, key=(4, 4))[:2])
    fm = feats(*oracle.glisur(kind, polish - h, wi, er, n1=n1, n2=n2, key=(5, 5))[:2])
    fd = (fp.mean(0) - fm.mean(0)) / (2 * h)
    se = np.sqrt(g.var(0) / n + (fp.var(0) + fm.var(0)) / n / (2 * h) ** 2)
    assert (np.abs(g.mean(0) - fd) < Z_MAX * se + 2e-3).all(), (g.mean(0), fd, se)


def test_glisur_tank_balances_and_differentiates():
    """Through the step: every photon's weight ends in one fate, and the Jacobian in the walls' R matches
    common-random-number differences. (Polish is checked above at the surface: moving r moves the edge of the facet
    ball's support, so a reweighted path's weight jumps where a facet crosses it and common-random-number differences
    of whole traces in polish are not smooth; the path score is.)"""
    from lumen_b200 import _abi as A
    from lumen_b200 import detectors, sources

    det = detectors.glisur_tank()
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam=400.0)
    n = 1 << 13
    names = ["surfaces/Wall/R"]
    c = A.controls(grad_tabs=[det.params_index[k] for k in names])
    T, _ = oracle.trace(det, A.key_of_seed(0), n, source=src, samples=n, controls=c)
    h = T.health
    assert abs(h[:10].sum() - h[10]) < 1e-6 * h[10]
    for i, name in enumerate(names):
        off, k = det.arrays["tab"][det.params_index[name]]
        v0 = float(det.pool[off + k])
        dv = 0.0025 * v0
        arr = [oracle.trace(det, A.key_of_seed(0), n, source=src, samples=n, pool_live=det.pool_with({name: v}),
                            pool_ref=det.pool)[0].arrival[0] for v in (v0 + dv, v0 - dv)]  # fmt: skip
        fd = (arr[0] - arr[1]) / (2 * dv)
        scale = np.max(np.abs(fd))
        np.testing.assert_allclose(T.jac[0][:, i], fd, atol=3e-3 * scale + 1e-12, rtol=3e-3, err_msg=name)
