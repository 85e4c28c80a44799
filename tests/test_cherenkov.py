"""The Cherenkov segment source (src/lumen/sources/cherenkov.py:33 cone, :65 CherenkovSegment) in the checker.

- Every photon leaves on the cone cos theta = 1 / (beta n(lam)) about the segment, n the medium's RINDEX table read
  linearly in energy (Geant4's RINDEX law) at the photon's wavelength;
- the wavelength is drawn ~ 1 / lam^2 over the table's span: 1 / lam uniform (chi2 at the reference's suite level);
- the weights sum to Frank-Tamm's photon number 2 pi alpha z^2 L int (1 - 1 / (beta n)^2)_+ d(1 / lam) (a numerical
  integral of the table, per metre; z-test);
- the start is uniform along the segment, the time the charge's passage there, the polarisation Geant4's (in the plane
  of the axis and the photon, perpendicular to the photon);
- below threshold (beta n <= 1 everywhere) the segment gives no light; through a trace every weight ends in a fate.
"""

import math

import numpy as np
from scipy import stats

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors
from lumen_b200.sources import HC, CherenkovSegment

P_MIN = 0.0027 / 400
ALPHA = 1.0 / 137.035999084
E_TAB = np.array([1.5, 2.5, 3.5, 5.0])
N_TAB = np.array([1.332, 1.336, 1.345, 1.366])  # the tutorial tank's water


def _index(lam):
    return np.interp(HC / lam, E_TAB, N_TAB)


def _rows(src, n, det):
    f, ev = oracle.source_rows(src, A.key_of_seed(3), n, det=det)
    return f.astype(np.float64), ev


def test_cone_wavelengths_and_weights():
    det = detectors.toy_tank()
    axis = np.array([0.3, -0.2, 0.9])
    axis /= np.linalg.norm(axis)
    src = CherenkovSegment("Water", start=(0.01, 0.02, -0.1), direction=axis, length=0.2, beta=0.95, charge=1.0,
                           time=1.5)  # fmt: skip
    n = 1 << 18
    f, _ = _rows(src, n, det)
    x, d, t, lam, w, er = f[:, 0:3], f[:, 3:6], f[:, 6], f[:, 7], f[:, 8], f[:, 9:12]
    lam_min, lam_max = HC / E_TAB.max(), HC / E_TAB.min()
    assert lam.min() >= lam_min * (1 - 1e-6) and lam.max() <= lam_max * (1 + 1e-6)
    nl = _index(lam)
    emits = 0.95 * nl > 1.0
    assert emits.all()
    np.testing.assert_allclose(d @ axis, 1.0 / (0.95 * nl), atol=2e-6)  # the cone
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=1e-6)
    u = (1.0 / lam - 1.0 / lam_max) / (1.0 / lam_min - 1.0 / lam_max)  # ~ 1 / lam^2: 1 / lam uniform
    h = np.histogram(u, np.linspace(0.0, 1.0, 51))[0]
    assert stats.chisquare(h).pvalue > P_MIN
    along = (x - np.array([0.01, 0.02, -0.1])) @ axis  # uniform along the segment; on its axis
    np.testing.assert_allclose(np.linalg.norm(x - np.array([0.01, 0.02, -0.1]) - along[:, None] * axis, axis=1), 0.0,
                               atol=1e-6)  # fmt: skip
    assert stats.kstest(along / 0.2, "uniform").pvalue > P_MIN
    np.testing.assert_allclose(t, 1.5 + along / (0.95 * 0.299792458), rtol=1e-5)
    np.testing.assert_allclose(np.sum(er * d, 1), 0.0, atol=2e-6)  # polarisation: perpendicular to the photon,
    np.testing.assert_allclose(np.einsum("ni,ni->n", er, np.cross(axis, d)), 0.0, atol=2e-6)  # in the axis plane
    zq = 1.0 / lam_min - 1.0 / lam_max
    w_want = 2 * math.pi * ALPHA * 0.2 * (1.0 - 1.0 / (0.95 * nl) ** 2) * zq / n * 1e9
    np.testing.assert_allclose(w, w_want, rtol=2e-5)
    inv = np.linspace(1.0 / lam_max, 1.0 / lam_min, 200001)  # Frank-Tamm: photons of the segment
    g = np.maximum(1.0 - 1.0 / (0.95 * _index(1.0 / inv)) ** 2, 0.0)
    total = 2 * math.pi * ALPHA * 0.2 * np.trapezoid(g, inv) * 1e9
    assert abs(w.sum() - total) < 4.0 * w.std() * math.sqrt(n)


def test_below_threshold_gives_no_light():
    det = detectors.toy_tank()
    src = CherenkovSegment("Water", direction=(0.0, 0.0, 1.0), length=0.1, beta=0.7)  # beta n < 0.96
    f, _ = _rows(src, 4096, det)
    np.testing.assert_array_equal(f[:, 8], 0.0)
    np.testing.assert_allclose(f[:, 3:6], np.broadcast_to([0.0, 0.0, 1.0], (4096, 3)), atol=1e-7)


def test_segments_are_events_and_a_trace_balances():
    det = detectors.toy_tank()
    # the second segment's cone (41 degrees about +x) crosses the PMT at (0.25, 0, -0.48)
    src = CherenkovSegment("Water", start=[(0.0, 0.0, -0.2), (-0.36, 0.0, 0.0)], direction=[(0, 0, 1), (1, 0, 0)],
                           length=[0.3, 0.12], beta=[0.99, 0.999], charge=[1.0, 2.0])  # fmt: skip
    n = 1 << 14
    f, ev = _rows(src, n, det)
    assert (ev[: n // 2] == 0).all() and (ev[n // 2:] == 1).all()
    T, _ = oracle.trace(det, A.key_of_seed(3), n, source=src, samples=n, n_events=2)
    h = T.health
    assert abs(h[:10].sum() - h[10]) < 1e-6 * h[10]
    np.testing.assert_allclose(h[10], f[:, 8].astype(np.float64).sum(), rtol=1e-6)  # the start is the rows' light
    assert T.arrival.sum() > 0
