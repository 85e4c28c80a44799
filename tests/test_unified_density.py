"""The unified facet lobe's density: the tables, one facet reflection's log density and its derivative in sigma.

- The tables (lumen_b200.facets) against the reference's own (tests/golden/unified_tables.npz, sampled from
  src/lumen/surfaces/facets.py:127 ``unified_tables`` by tests/golden/make_unified_fixture.py).
- The checker's Hermite reads against the float64 quadrature at each cell's midpoint and a random point in it, to the
  errors the reference states for its tables (src/lumen/rules/choices.py:25-33; tests/unit/test_unified_tables.py:25
  of the reference), and the quadrature itself against scipy's adaptive quadrature at a few points.
- One reflection's density p1(wo | wi) = D(h) / (4 F V . h) integrates to 1 over the sphere (the lobe contract,
  tests/unit/lobe_contract.py:64 of the reference), its score has mean 0 under the facet draw (for one facet and for
  whole paths: the premise of reweighting) and its derivative in sigma matches central differences.
- Through the step: the Jacobian in a ground wall's sigma_alpha against common-random-number differences.
"""

import math
import os

import numpy as np
import pytest
from scipy import integrate

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, facets, sources

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "unified_tables.npz"))
DF_MAX, DLZ_MAX = 5e-7, 1.4e-6  # the reference's stated table errors (4.7e-7, 1.3e-6)
Z_MAX = 4.0


def _wi(theta_deg):
    t = math.radians(theta_deg)
    return np.array([math.sin(t), 0.0, -math.cos(t)], np.float32)


def test_tables_match_the_references():
    T = facets.tables()
    assert tuple(GOLD["shape"]) == T["F"].shape == (facets.NX, facets.NY)
    i, j = GOLD["i"], GOLD["j"]
    # the values and the x derivatives agree bit for bit; the y derivatives (differences of float64 quadratures
    # 2e-5 apart in log sigma) to their rounding
    np.testing.assert_array_equal(T["F"][i, j], GOLD["F"])
    np.testing.assert_array_equal(T["lz"], GOLD["lz"])
    np.testing.assert_allclose(T["Fx"][i, j], GOLD["Fx"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(T["Fy"][i, j], GOLD["Fy"], rtol=0, atol=1e-8)
    np.testing.assert_allclose(T["Fxy"][i, j], GOLD["Fxy"], rtol=0, atol=3e-8)
    np.testing.assert_allclose(T["lzy"], GOLD["lzy"], rtol=0, atol=1e-8)


def test_quadrature_matches_adaptive_quadrature():
    for sigma in (0.003, 0.05, 0.25, 0.7, 1.0):
        fm = min(1.0, 4.0 * sigma)

        def g(a, s=sigma, f=fm):
            return math.exp(-a * a / (2 * s * s)) * min(math.sin(a), f)

        z = integrate.quad(g, 0.0, 0.5 * math.pi, points=[math.asin(fm)], limit=400, epsabs=0, epsrel=1e-12)[0]
        assert facets.norm_z(sigma) == pytest.approx(z, rel=1e-9)
        for theta in (5.0, 40.0, 80.0, 89.5):
            t = math.radians(theta)
            cot = math.cos(t) / math.sin(t)

            def away(a, c=cot, s=sigma, f=fm):
                return g(a, s, f) * math.acos(max(-1.0, min(1.0, c * math.cos(a) / math.sin(a)))) / math.pi

            ak = math.atan(cot)
            a_away = integrate.quad(away, ak, 0.5 * math.pi, points=[max(ak, math.asin(fm))], limit=400,
                                    epsabs=0, epsrel=1e-11)[0]  # fmt: skip
            x = math.atan2(math.cos(t), sigma * math.sin(t)) / (0.5 * math.pi)
            assert facets.facing(np.array([x]), sigma)[0] == pytest.approx(1.0 - a_away / z, abs=1e-9)


def test_hermite_reads_match_the_quadrature_over_the_span():
    rng = np.random.default_rng(1)
    cells = np.arange(facets.J_LO, facets.J_HI)
    ys = (facets.Y0 + facets.DY * np.concatenate([cells + 0.5, cells + rng.uniform(0.05, 0.95, cells.size)]))
    ys = ys.astype(np.float32)
    xs = np.concatenate([(np.arange(128) + 0.5) / 128, rng.uniform(0.0, 1.0, 128)]).astype(np.float32)
    X, Y = np.meshgrid(xs, ys)
    F = oracle.unified(1, np.stack([X.ravel(), Y.ravel()], 1))[:, 0].reshape(X.shape)
    lz = oracle.unified(0, ys)[:, 0]
    x64 = xs.astype(np.float64)
    df = max(float(np.abs(F[k] - facets.facing(x64, math.exp(float(y)))).max()) for k, y in enumerate(ys))
    dlz = max(abs(float(lz[k]) - math.log(facets.norm_z(math.exp(float(y))) / math.exp(2.0 * float(y))))
              for k, y in enumerate(ys))  # fmt: skip
    assert df <= DF_MAX and dlz <= DLZ_MAX, (df, dlz)


def _grid(axis, na=1500, nphi=720):
    """Directions about ``axis`` (polar angle pi u^2, dense near it) and their solid angles."""
    u = (np.arange(na) + 0.5) / na
    a, da = np.pi * u**2, 2.0 * np.pi * u / na
    phi = (np.arange(nphi) + 0.5) / nphi * 2.0 * np.pi
    ref = np.array([1.0, 0.0, 0.0]) if abs(axis[0]) < 0.9 else np.array([0.0, 1.0, 0.0])
    e1 = np.cross(axis, ref)
    e1 /= np.linalg.norm(e1)
    e2 = np.cross(axis, e1)
    AA, PP = np.meshgrid(a, phi, indexing="ij")
    W = np.cos(AA)[..., None] * axis + np.sin(AA)[..., None] * (np.cos(PP)[..., None] * e1 + np.sin(PP)[..., None] * e2)
    return W.reshape(-1, 3), (np.sin(AA) * da[:, None] * (2.0 * np.pi / nphi)).ravel()


def _logpdf_in(sigma, wi, W):
    n = len(W)
    return np.concatenate([np.full((n, 1), sigma), np.tile(wi, (n, 1)), np.tile([0.0, 0.0, 1.0], (n, 1)), W], 1)


@pytest.mark.parametrize(("sigma", "theta"), [(0.1, 30.0), (0.3, 60.0), (0.05, 80.0), (0.9, 45.0), (0.01, 20.0)])
def test_one_reflection_density_integrates_to_one(sigma, theta):
    wi = _wi(theta)
    W, dw = _grid(wi.astype(np.float64) * np.array([1.0, 1.0, -1.0]))
    lp = oracle.unified(2, _logpdf_in(sigma, wi, W))[:, 0].astype(np.float64)
    assert abs(float(np.sum(np.exp(lp) * dw)) - 1.0) < 3e-3


@pytest.mark.parametrize(("sigma", "theta"), [(0.1, 30.0), (0.3, 60.0), (0.05, 80.0), (0.9, 45.0), (0.25, 10.0)])
def test_score_has_mean_zero_under_the_draw(sigma, theta):
    for one in (True, False):
        _, capped, dens = oracle.facet_path(sigma, _wi(theta), 1 << 19, key=(3, 17), sig_live=sigma, one=one)
        assert capped == 0
        np.testing.assert_array_equal(dens[:, 0], dens[:, 1])  # live = drawn width: the weight is exactly 1
        sc = dens[:, 2].astype(np.float64)
        z = sc.mean() / (sc.std(ddof=1) / math.sqrt(len(sc)))
        assert abs(z) < Z_MAX, (one, sc.mean(), z)


@pytest.mark.parametrize(("sigma", "theta"), [(0.9, 45.0), (0.6, 70.0), (0.2, 40.0), (0.02, 60.0)])
def test_sigma_derivative_matches_differences(sigma, theta):
    rng = np.random.default_rng(0)
    W = rng.normal(size=(4000, 3))
    W /= np.linalg.norm(W, axis=1, keepdims=True)
    inp = _logpdf_in(sigma, _wi(theta), W)
    out = oracle.unified(2, inp)
    on = out[:, 0] > 0.5 * -69.0
    h = 1e-3 * sigma
    up, dn = inp.copy(), inp.copy()
    up[:, 0] += h
    dn[:, 0] -= h
    fd = (oracle.unified(2, up)[:, 0].astype(np.float64) - oracle.unified(2, dn)[:, 0]) / (2.0 * h)
    rel = np.abs(fd - out[:, 1])[on] / np.maximum(np.abs(fd[on]), 1.0)
    assert np.median(rel) < 1e-3 and np.quantile(rel, 0.98) < 2e-2


def test_ground_wall_sigma_jacobian_matches_differences():
    """d arrivals / d sigma_alpha of a ground wall through the tracing, against +-0.25 % common-random-number runs.

    The narrow lobe's log density has a large third derivative in sigma (alpha^2 / sigma^5 in its tails): at +-1 % the
    differences' own O(h^2) error reaches 3e-3 of the largest derivative, falling fourfold per halving of h.
    """
    det = detectors.cylinder_tank(n_pmt=200, wall_finish="ground", sigma_alpha=0.1, wall_r=0.9)
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    name = "surfaces/BlackSheet/sigma_alpha"
    n = 1 << 13
    c = A.controls(grad_tabs=[det.params_index[name]])
    T, _ = oracle.trace(det, A.key_of_seed(0), n, source=src, samples=n, controls=c)
    off, k = det.arrays["tab"][det.params_index[name]]
    v0 = float(det.pool[off + k])
    h = 0.0025 * v0
    arr = [oracle.trace(det, A.key_of_seed(0), n, source=src, samples=n, pool_live=det.pool_with({name: v}),
                        pool_ref=det.pool)[0].arrival[0] for v in (v0 + h, v0 - h)]  # fmt: skip
    fd = (arr[0] - arr[1]) / (2 * h)
    scale = np.max(np.abs(fd))
    assert scale > 0
    np.testing.assert_allclose(T.jac[0][:, 0], fd, atol=2e-3 * scale, rtol=2e-3)
