"""The unified facet path (GLOSSY) against Geant4 11.3.0's G4OpBoundaryProcess on one flat interface.

tests/golden/g4_unified_metal.npz holds the reference's Geant4 histograms (tests/data/g4_boundary, made by its
tools/g4ref/boundary.cc; extracted by tests/golden/make_g4_fixture.py): a unified ground dielectric_metal surface with
R = 1 and SPECULARLOBECONSTANT 1, 10^6 photons along one direction, the last direction's histogram in (dz, |phi|).
The checker's facet path (Geant4's GetFacetNormal loop as the reference restates it, src/lumen/surfaces/facets.py)
draws 2^20 paths; the two histograms are compared by the reference's two-sample chi2 on pooled counts
(tests/unit/test_g4_boundary.py:48), at the reference's suite-wide level.
"""

import math
import os

import numpy as np
import pytest
from scipy import stats

import oracle

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "g4_unified_metal.npz"))
P_MIN = 0.0027 / 400  # Z_MAX = 3 two-sided, shared by the reference's 400 statistical assertions


def _chi2_p(g4, ours):
    g4, ours = np.ravel(g4).astype(np.float64), np.ravel(ours).astype(np.float64)
    n1, n2 = g4.sum(), ours.sum()
    use = (g4 + ours) > 0
    c2 = float(np.sum((g4[use] / n1 - ours[use] / n2) ** 2 / ((g4[use] + ours[use]) / (n1 * n2))))
    return float(stats.chi2.sf(c2, int(use.sum()) - 1)), c2, int(use.sum()) - 1


@pytest.mark.parametrize("i", range(len(GOLD["names"])))
def test_unified_facet_path_is_geant4s(i):
    theta = math.radians(float(GOLD[f"c{i}_theta_deg"]))
    sigma = float(GOLD[f"c{i}_sigma"])
    wi = np.array([math.sin(theta), 0.0, -math.cos(theta)], np.float32)
    wo, capped = oracle.facet_path(sigma, wi, 1 << 20, key=(0, 100 + i))
    assert capped == 0
    h = np.histogram2d(wo[:, 2], np.abs(np.arctan2(wo[:, 1], wo[:, 0])),
                       bins=[GOLD[f"c{i}_edges_z"], GOLD[f"c{i}_edges_phi"]])[0]  # fmt: skip
    pv, c2, dof = _chi2_p(GOLD[f"c{i}_hist"], h)
    assert pv > P_MIN, (str(GOLD["names"][i]), c2, dof)
