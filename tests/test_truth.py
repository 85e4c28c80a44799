"""Truth rows (src/lumen/readout/truth.py, the analog photon of src/lumen/transport/step.py:625-660) in the checker.

- The detection draw's threefry (numpy, lumen_b200.truth) is the checker's, bit for bit;
- the analog law: each photon's analog is absorbed at most once, at a crossing with the probability of its reached
  share, so per sensor the absorbed photons estimate the arrivals (their expected detections) whatever the roulette
  (it keeps an open analog fate) and for rows standing for k <= 1 photons (z-tests);
- the expected values of a run with truth rows are the same in law as without (the roulette's keep keeps its total);
- a record's cathode point lies on its sensor's surface, its wavelength is the photon's, its scale 1 / A_n.
"""

import math

import numpy as np
import pytest
from scipy import stats

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200 import truth as TR

P_MIN = 0.0027 / 400
Z = 4.0
KEY = A.key_of_seed(11)


def test_threefry_is_the_checkers():
    rng = np.random.default_rng(0)
    k0, k1, x0, x1 = (rng.integers(0, 2**32, 64, dtype=np.uint64).astype(np.uint32) for _ in range(4))
    a, b = TR.threefry(k0, k1, x0, x1)
    for i in range(64):
        assert (int(a[i]), int(b[i])) == oracle.threefry(int(k0[i]), int(k1[i]), int(x0[i]), int(x1[i]))
    ids = np.arange(1000)
    want = oracle.uniforms(KEY, ids, 0, 3)  # vertex 0 of each photon key
    vk = TR.fold_in(TR.fold_in(KEY, ids.astype(np.uint32)), np.zeros(1000, np.uint32))
    for i in range(3):
        np.testing.assert_array_equal(TR.uniform(vk, i), want[:, i])


def _run(det, src, n, flags=0, roulette=0.01):
    c = A.controls(roulette=roulette, flags=flags)
    return oracle.trace(det, KEY, n, source=src, samples=n, controls=c, truth=bool(flags & A.F_TRUTH))[0]


@pytest.mark.parametrize(("roulette", "k"), [(0.01, 1.0), (1.0, 1.0), (0.01, 0.5)])
def test_absorbed_photons_estimate_the_arrivals(roulette, k):
    det = detectors.toy_tank()
    n = 1 << 17
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=k * n, lam=400.0)
    T = _run(det, src, n, A.F_TRUTH, roulette)
    sensor = T.truth[:, 0].view(np.int32)
    counts = np.bincount(sensor[sensor >= 0], minlength=det.n_sensor)
    arr = T.arrival[0]
    assert counts.sum() > 1000
    # each analog absorption is Bernoulli with a small probability: the count per sensor ~ Poisson(arrival)
    z = (counts - arr) / np.sqrt(np.maximum(arr, 1.0))
    assert np.abs(z).max() < Z, (counts, arr)
    assert abs(T.health[:10].sum() - T.health[10]) < 1e-6 * T.health[10]


def test_expected_values_unchanged_in_law():
    det = detectors.toy_tank()
    n = 1 << 17
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=float(n), lam=400.0)
    out = []
    for flags in (0, A.F_TRUTH):
        T = _run(det, src, n, flags, roulette=0.05)
        var = np.maximum(T.arrival2[0] - T.arrival[0] ** 2 / n, 0.0) * n / (n - 1)
        out.append((T.arrival[0], var))
    (a0, v0), (a1, v1) = out
    c2 = float(np.sum((a1 - a0) ** 2 / (v0 + v1)))
    assert stats.chi2.sf(c2, len(a0)) > P_MIN, c2


def test_record_fields():
    det = detectors.readout_tank()  # photocathodes read per normal incidence on the "pmt" group
    n = 1 << 15
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=float(n), lam_range=(330.0, 480.0))
    T = _run(det, src, n, A.F_TRUTH)
    tr = T.truth
    sensor = tr[:, 0].view(np.int32)
    hit = sensor >= 0
    assert hit.sum() > 100
    vol = tr[hit, 7].view(np.int32)
    np.testing.assert_array_equal(det.arrays["vol_i"][vol, 3], sensor[hit])  # the volume entered is the sensor's
    vf = np.asarray(det.arrays["vol_f"], np.float64)[vol]
    loc = np.einsum("nij,ni->nj", vf[:, 0:9].reshape(-1, 3, 3), tr[hit, 4:7].astype(np.float64) - vf[:, 9:12])
    on_face = np.abs(np.abs(loc[:, 2]) - 0.01) < 1e-5  # the PMT discs: r 0.05, half height 0.01
    on_side = np.abs(np.hypot(loc[:, 0], loc[:, 1]) - 0.05) < 1e-5
    assert (on_face | on_side).all()
    assert (tr[hit, 1] > 0).all() and ((tr[hit, 2] >= 330.0) & (tr[hit, 2] <= 540.0)).all()  # WLS: up to 539 nm
    pmt = np.isin(sensor[hit], det.groups["pmt"])
    assert (tr[hit, 3][pmt] > 1.0).all() and (tr[hit, 3][~pmt] == 1.0).all()  # 1 / A_n of the photocathodes
    assert (sensor[~hit] == -1).all()


def test_detection_thinning_and_sum_by():
    det = detectors.toy_tank()
    n = 1 << 16
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=float(n), lam=400.0)
    T = _run(det, src, n, A.F_TRUTH)
    from lumen_b200.readout import Axis, Grid, Group

    g = Group(Grid(axes=(Axis("wavelength", "wavelength", knots=(300.0, 500.0)),)), None, np.array([0.3, 0.3]), 0.5)
    hits = TR.rows(TR.Truth(keep="absorbed"), det, T.truth, KEY, 0, None, {"pmt": g})
    absorbed = int((T.truth[:, 0].view(np.int32) >= 0).sum())
    assert len(hits.photon) == absorbed and (hits.label == -1).all()
    p = 0.5 * 0.3  # efficiency x the acceptance at 400 nm
    det_n = int(hits.detected.sum())
    assert abs(det_n - p * absorbed) < Z * math.sqrt(absorbed * p * (1 - p))
    only = TR.rows(TR.Truth(), det, T.truth, KEY, 0, None, {"pmt": g})
    np.testing.assert_array_equal(only.photon, hits.photon[hits.detected])
    s = only.sum_by(("sensor",))
    assert int(s["n"].sum()) == det_n and (np.diff(s["sensor"]) > 0).all()
