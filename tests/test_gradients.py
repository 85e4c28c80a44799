"""Derivatives of the arrivals: forward tangents of the reweighting estimator along each path, checked

- against central finite differences with common random numbers (the reference held at the nominal values, the live
  values moved +-1 %: every draw identical, the weights live / reference; src/lumen/api.py:935-941's check), and
- against the closed-form derivatives of the specular sensor sphere (tests/physics/test_toys.py:135-146 of the
  reference: d Q / d R and d Q / d L exact).
"""

import math

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from tests.test_oracle import sensor_sphere

KEY = A.key_of_seed(0)


def _fd_vs_jac(det, src, names, n, rel=0.01):
    c = A.controls(grad_tabs=[det.params_index[k] for k in names])
    T, _ = oracle.trace(det, KEY, n, source=src, samples=n, controls=c)
    jac = T.jac[0]
    for i, name in enumerate(names):
        off, k = det.arrays["tab"][det.params_index[name]]
        v0 = float(det.pool[off + k])
        h = rel * v0
        up = oracle.trace(det, KEY, n, source=src, samples=n, pool_live=det.pool_with({name: v0 + h}),
                          pool_ref=det.pool)[0].arrival[0]  # fmt: skip
        dn = oracle.trace(det, KEY, n, source=src, samples=n, pool_live=det.pool_with({name: v0 - h}),
                          pool_ref=det.pool)[0].arrival[0]  # fmt: skip
        fd = (up - dn) / (2 * h)
        scale = np.max(np.abs(fd)) + 1e-30
        np.testing.assert_allclose(jac[:, i], fd, atol=2e-3 * scale, rtol=2e-3, err_msg=name)


def test_tank_jacobian_matches_common_random_number_differences():
    det = detectors.cylinder_tank()
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    _fd_vs_jac(det, src, ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"], 1 << 13)


def test_toy_tank_jacobian_matches_differences():
    det = detectors.toy_tank()
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    # the cathode's EFFICIENCY is a surface column of the detected share
    _fd_vs_jac(det, src, ["surfaces/CathodeSurface/eff"], 1 << 12)


def test_specular_sphere_exact_derivatives():
    A_, L, R = 1.0, 5.0, 0.5
    det = sensor_sphere(A_, L, R, "polished")
    src = sources.Point(position=(0.0, 0.0, 0.0), n_photons=1.0, lam=400.0)
    n = 1 << 12
    names = ["surfaces/Wall/R", "media/Liquid/absorption"]
    c = A.controls(grad_tabs=[det.params_index[k] for k in names])
    T, _ = oracle.trace(det, KEY, n, source=src, samples=n, controls=c)
    e1, e2 = math.exp(-A_ / L), math.exp(-2 * A_ / L)
    den = 1 - R * e2
    dq_dr = (-e1 * den + (1 - R) * e1 * e2) / den**2
    dq_dl = (1 - R) * (e1 * A_ / L**2 * den + e1 * R * e2 * 2 * A_ / L**2) / den**2
    assert T.jac[0, 0, 0] == pytest.approx(dq_dr, rel=1e-4)
    assert T.jac[0, 0, 1] == pytest.approx(dq_dl, rel=1e-4)
