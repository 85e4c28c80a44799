"""A material's scintillation light (src/lumen/sources/scintillation.py: flash :69, shares :48, ScintillationPoint
:172, ScintillationSegment :182) in the checker.

- The light: the weights sum to the yield times the energy (Birks-quenched along a segment, :42 visible_energy);
- the components share it as the yields say (25 / 75 here), each with its own spectrum (the weighted wavelengths follow
  the share-mixed spectra, chi2), delay (Exp(tau) plus Exp(tau rise / (tau + rise)), Geant4's finite-rise profile: the
  weighted mean delay) and isotropic directions;
- a component of share 0 at the reference is drawn under the defensive mixture and weighted to the live shares
  (unbiased: the live means are recovered);
- a segment's photons start uniformly along it at the charge's passage; a trace balances every weight.
"""

import math

import numpy as np
from scipy import stats

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors
from lumen_b200.detectors import SCINT_COMPONENTS
from lumen_b200.sources import HC, ScintillationPoint, ScintillationSegment

P_MIN = 0.0027 / 400
Z_MAX = 4.0


def _rows(src, n, det, pool=None):
    f, ev = oracle.source_rows(src, A.key_of_seed(7), n, det=det, pool=pool)
    return f.astype(np.float64), ev


def _mixture_cdf(energy, shares):
    """The share-mixed spectra's mass up to energy: Geant4's sampler per component, uniform in energy within each knot
    interval with the interval's trapezoid mass (a piecewise-linear CDF)."""  # noqa: D205, D209
    out = np.zeros_like(energy)
    for c, f in zip(SCINT_COMPONENTS, shares):
        e, s = (np.asarray(x, np.float64) for x in c["spectrum"])
        m = 0.5 * (s[1:] + s[:-1]) * np.diff(e)
        out += f * np.interp(energy, e, np.concatenate([[0.0], np.cumsum(m)]) / m.sum())
    return out


def _check_light(f, n, shares, total):
    w, lam, t = f[:, 8], f[:, 7], f[:, 6]
    assert abs(w.sum() - total) <= Z_MAX * w.std() * math.sqrt(n) + 1e-6 * total, (w.sum(), total)
    mean_delay = sum(s * (c["tau"] + c["tau"] * c["rise"] / (c["tau"] + c["rise"])) for c, s in zip(SCINT_COMPONENTS, shares))
    wm = (w * t).sum() / w.sum()
    sem = math.sqrt(np.sum((w * (t - wm)) ** 2)) / w.sum()
    assert abs(wm - mean_delay) < Z_MAX * sem, (wm, mean_delay)
    edges = np.linspace(2.5, 3.3, 33)
    e = HC / lam
    h = np.histogram(e, edges, weights=w / w.sum() * n)[0]
    want = np.diff(_mixture_cdf(edges, shares)) * n
    h2 = np.histogram(e, edges, weights=(w / w.sum() * n) ** 2)[0]
    use = want > 20
    c2 = float(np.sum((h[use] - want[use]) ** 2 / np.maximum(h2[use], 1e-12)))
    assert stats.chi2.sf(c2, int(use.sum())) > P_MIN, c2


def test_point_light_components_and_directions():
    det = detectors.scintillating_tank()
    n = 1 << 18
    f, _ = _rows(ScintillationPoint("Scint", position=(0.1, -0.2, 0.05), energy=2.0, time=0.0), n, det)
    np.testing.assert_array_equal(f[:, 0:3], np.broadcast_to(np.float32([0.1, -0.2, 0.05]), (n, 3)))
    d = f[:, 3:6]
    np.testing.assert_allclose(np.linalg.norm(d, axis=1), 1.0, atol=2e-6)
    assert stats.kstest((d[:, 2] + 1.0) / 2.0, "uniform").pvalue > P_MIN
    assert abs(d[:, 0].mean()) < Z_MAX / math.sqrt(3 * n) and abs(d[:, 1].mean()) < Z_MAX / math.sqrt(3 * n)
    _check_light(f, n, (0.25, 0.75), 2000.0)


def test_reference_share_zero_is_covered():
    det = detectors.scintillating_tank()
    n = 1 << 18
    live = det.pool_with({"media/Scint/scint_share1": 0.25, "media/Scint/scint_share2": 0.75})
    ref = det.pool_with({"media/Scint/scint_share1": 1.0, "media/Scint/scint_share2": 0.0})
    src = ScintillationPoint("Scint", position=(0.0, 0.0, 0.0), energy=1.0)
    T, _ = oracle.trace(det, A.key_of_seed(7), 4096, source=src, samples=4096, pool_live=live, pool_ref=ref)
    assert abs(T.health[:10].sum() - T.health[10]) < 1e-6 * T.health[10]
    # drawn at the reference shares (1, 0) under the defensive mixture, weighted to the live (0.25, 0.75)
    f, _ = oracle.source_rows(src, A.key_of_seed(7), n, det=det, pool=live, pool_ref=ref)
    w = f[:, 8].astype(np.float64)
    pos = w[w > 0]  # 0: a draw in a covered interval without mass; the slow component's rare draws weigh the most
    assert np.unique(np.round(pos / pos.min(), 3)).size == 2 and (w == 0).any()
    _check_light(f.astype(np.float64), n, (0.25, 0.75), 1000.0)


def test_segment_birks_and_passage():
    det = detectors.scintillating_tank()
    n = 1 << 17
    a, b = np.array([-0.2, 0.0, 0.1]), np.array([0.2, 0.1, -0.1])
    L = float(np.linalg.norm(b - a))
    src = ScintillationSegment("Scint", start=a, end=b, t_start=1.0, t_end=3.0, energy=4.0, birks=0.1)
    f, _ = _rows(src, n, det)
    x, t = f[:, 0:3], f[:, 6]
    u = (x - a) @ (b - a) / L**2
    np.testing.assert_allclose(np.linalg.norm(x - a - u[:, None] * (b - a), axis=1), 0.0, atol=2e-6)
    assert stats.kstest(u, "uniform").pvalue > P_MIN
    assert (t >= 1.0 + 2.0 * u - 1e-4).all()  # the passage, then the delay
    _check_light(np.column_stack([f[:, :6], t - (1.0 + 2.0 * u), f[:, 7:]]), n, (0.25, 0.75),
                 1000.0 * 4.0 / (1.0 + 0.1 * 4.0 / L))  # fmt: skip


def test_trace_balances_with_two_deposits():
    det = detectors.scintillating_tank()
    src = ScintillationPoint("Scint", position=[(0.0, 0.0, 0.0), (0.2, 0.1, -0.3)], energy=[1.0, 0.5])
    n = 1 << 14
    T, _ = oracle.trace(det, A.key_of_seed(7), n, source=src, samples=n, n_events=2)
    h = T.health
    assert abs(h[:10].sum() - h[10]) < 1e-6 * h[10]
    assert T.arrival[0].sum() > 0 and T.arrival[1].sum() > 0
