"""The Mie and WLS channels of a bulk medium (the checker's restatement of src/lumen/media/phase.py:113-191,
spectra.py and emission.py:127-162).

- Mie (G4OpMieHG): the draw follows its density (chi2 in the cosine against the density integrated along it), the
  density integrates to 1 and gives the mixture's mean cosine r g_f - (1 - r) g_b (the lobe contract,
  tests/unit/lobe_contract.py of the reference), the score in each constant has mean 0 under the draw, and the
  derivatives match central differences.
- WLS (G4OpWLS): no emission above the absorbed energy, the emitted energies follow the spectrum truncated there (its
  exact inverse CDF), the weight is the yield times Geant4's chance that one of 100 draws lands below the absorbed
  energy, 0 below the spectrum, the delays are the profile's.
- Through the step: every photon's weight ends in one fate, and the Jacobian in the channels' lengths and constants
  matches +-0.5 % common-random-number differences.
"""

import math

import numpy as np
import pytest
from scipy import stats

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources

P_MIN = 0.0027 / 400  # the reference's suite-wide chi2 level
Z_MAX = 4.0
HC = 1239.84198433200208
WI = np.array([0.0, 0.6, 0.8], np.float32)


def _cos_density(gf, gb, r, n_fine=20001):
    """The density of mu = wo . wi on [-1, 1] (2 pi p per steradian) on a fine grid, from the checker's logpdf."""
    mu = np.linspace(-1.0, 1.0, n_fine)
    t1 = np.cross(WI, [1.0, 0.0, 0.0])
    t1 /= np.linalg.norm(t1)
    ang = np.arccos(mu)
    W = np.cos(ang)[:, None] * WI + np.sin(ang)[:, None] * t1
    return mu, 2.0 * math.pi * np.exp(oracle.mie_logpdf(gf, gb, r, WI, W)[:, 0].astype(np.float64))


@pytest.mark.parametrize(("gf", "gb", "r"), [(0.9, 0.3, 0.8), (0.5, 0.0, 1.0), (-0.3, 0.6, 0.4), (0.0, 0.0, 0.5)])
def test_mie_draw_follows_its_density(gf, gb, r):
    wo, lp = oracle.mie(gf, gb, r, WI, 1 << 20)
    mu = wo.astype(np.float64) @ WI.astype(np.float64)
    assert np.abs(np.linalg.norm(wo, axis=1) - 1.0).max() < 1e-5
    f, p = _cos_density(gf, gb, r)
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (p[1:] + p[:-1]) * np.diff(f))])
    assert abs(cdf[-1] - 1.0) < 1e-3
    edges = np.linspace(-1.0, 1.0, 101)
    expected = np.diff(np.interp(edges, f, cdf)) * len(mu) / cdf[-1]
    h = np.histogram(mu, edges)[0]
    use = expected > 5
    c2 = float(np.sum((h[use] - expected[use]) ** 2 / expected[use]))
    assert stats.chi2.sf(c2, int(use.sum()) - 1) > P_MIN, c2
    sem = mu.std() / math.sqrt(len(mu))
    assert abs(mu.mean() - (r * gf - (1.0 - r) * gb)) < Z_MAX * sem


@pytest.mark.parametrize(("gf", "gb", "r"), [(0.9, 0.3, 0.8), (-0.3, 0.6, 0.4)])
def test_mie_scores_and_derivatives(gf, gb, r):
    wo, _ = oracle.mie(gf, gb, r, WI, 1 << 19, key=(5, 5))
    d = oracle.mie_logpdf(gf, gb, r, WI, wo).astype(np.float64)
    for k in range(3):  # the score of each constant has mean 0 under the draw
        sc = d[:, 1 + k]
        assert abs(sc.mean()) < Z_MAX * sc.std() / math.sqrt(len(sc)), k
    x = wo[:2000]
    h = 1e-3
    for k, args in enumerate([(gf, gb, r)] * 3):
        up, dn = list(args), list(args)
        up[k] += h
        dn[k] -= h
        fd = (oracle.mie_logpdf(*up, WI, x)[:, 0].astype(np.float64) - oracle.mie_logpdf(*dn, WI, x)[:, 0]) / (2 * h)
        np.testing.assert_allclose(d[:2000, 1 + k], fd, rtol=2e-2, atol=2e-2)


E_SPEC = np.array([2.3, 2.5, 2.7, 2.9, 3.1, 3.2], np.float32)
S_SPEC = np.array([0.0, 0.4, 1.0, 0.7, 0.1, 0.0], np.float32)


def _trapezoid_cdf(E):
    """The spectrum's mass up to energy E (float64): Geant4's sampler, uniform in energy within each interval."""
    e, s = E_SPEC.astype(np.float64), S_SPEC.astype(np.float64)
    mass = 0.5 * (s[1:] + s[:-1]) * np.diff(e)
    c = np.concatenate([[0.0], np.cumsum(mass)]) / mass.sum()
    return np.interp(E, e, c)


@pytest.mark.parametrize("lam_in", [360.0, 420.0, 480.0])
def test_wls_emission_is_the_truncated_spectrum(lam_in):
    E_in = HC / lam_in
    out = oracle.wls(E_SPEC, S_SPEC, S_SPEC, lam_in, 1 << 19, yield_live=0.9, yield_ref=0.9, tau=2.0, exponential=True)
    E = HC / out[:, 0].astype(np.float64)
    assert E.max() <= E_in * (1 + 1e-6)
    F = _trapezoid_cdf(E_in)
    edges = np.linspace(E_SPEC[0], min(E_in, E_SPEC[-1]), 41)
    expected = np.diff(_trapezoid_cdf(edges)) / F * len(E)
    h = np.histogram(E, edges)[0]
    use = expected > 5
    c2 = float(np.sum((h[use] - expected[use]) ** 2 / expected[use]))
    assert stats.chi2.sf(c2, int(use.sum()) - 1) > P_MIN, c2
    kept = 1.0 - (1.0 - F) ** 100  # one of G4OpWLS's 100 draws finds an energy at or below the absorbed one
    np.testing.assert_allclose(out[:, 2], 0.9 * kept, rtol=2e-6)
    np.testing.assert_array_equal(out[:, 2], out[:, 3])  # live = reference: the weight is the reference's
    d = out[:, 1].astype(np.float64)
    assert abs(d.mean() - 2.0) < Z_MAX * d.std() / math.sqrt(len(d))  # the exponential profile's mean


def test_wls_below_the_spectrum_and_delta_profile():
    out = oracle.wls(E_SPEC, S_SPEC, S_SPEC, 700.0, 1024, tau=3.5, exponential=False)
    np.testing.assert_array_equal(out[:, 2], 0.0)  # an absorbed energy below the spectrum re-emits nothing
    np.testing.assert_array_equal(out[:, 1], np.float32(3.5))  # the delta profile: the time constant
    live = S_SPEC * np.array([1.0, 1.2, 1.0, 0.8, 1.0, 1.0], np.float32)
    out = oracle.wls(E_SPEC, live, S_SPEC, 400.0, 1 << 18, yield_live=0.8, yield_ref=0.9)
    w = out[:, 2].astype(np.float64)  # drawn at the reference, weighted to the live spectrum: unbiased for its mean
    assert abs(w.mean() / 0.8 - (1.0 - (1.0 - _live_cdf(live, HC / 400.0)) ** 100)) < Z_MAX * w.std() / 0.8 / 512


def _live_cdf(s, E):
    e = E_SPEC.astype(np.float64)
    s = np.asarray(s, np.float64)
    mass = 0.5 * (s[1:] + s[:-1]) * np.diff(e)
    c = np.concatenate([[0.0], np.cumsum(mass)]) / mass.sum()
    return float(np.interp(E, e, c))


def test_scintillator_cube_balances_and_differentiates():
    det = detectors.scintillator_cube()
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam_range=(330.0, 480.0))
    n = 1 << 13
    names = ["media/LAB/mie", "media/LAB/wls", "media/LAB/mie_g_forward", "media/LAB/wls_yield", "media/LAB/rayleigh"]
    c = A.controls(grad_tabs=[det.params_index[k] for k in names])
    T, _ = oracle.trace(det, A.key_of_seed(0), n, source=src, samples=n, controls=c)
    h = T.health
    assert abs(h[:10].sum() - h[10]) < 1e-6 * h[10]  # every photon's weight ends in one fate
    assert T.arrival.sum() > 0
    for i, name in enumerate(names):  # a parameter: every value of its table moving together (d / d value)
        off, k = det.arrays["tab"][det.params_index[name]]
        vals = det.pool[off + k:off + 2 * k].astype(np.float64)
        dv = 0.005 * float(np.abs(vals).min())
        arr = [oracle.trace(det, A.key_of_seed(0), n, source=src, samples=n, pool_live=det.pool_with({name: v}),
                            pool_ref=det.pool)[0].arrival[0] for v in (vals + dv, vals - dv)]  # fmt: skip
        fd = (arr[0] - arr[1]) / (2 * dv)
        scale = np.max(np.abs(fd))
        np.testing.assert_allclose(T.jac[0][:, i], fd, atol=3e-3 * scale + 1e-12, rtol=3e-3, err_msg=name)
