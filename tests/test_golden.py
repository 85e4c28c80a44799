"""The checker's functions against golden vectors computed by the reference's own Python
(tests/golden/make_golden.py: Fresnel amplitudes, the dipole inverse CDF, the orthonormal basis, Geant4's water
Rayleigh table and GROUPVEL group index, evaluated by the reference's source on fixed inputs)."""

import os

import numpy as np
import pytest

import oracle
from lumen_b200 import optics as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "reference_vectors.npz")


@pytest.fixture(scope="module")
def g():
    return np.load(GOLD)


def test_fresnel_amplitudes(g):
    x = g["fresnel_in"]
    got = oracle.fresnel(x[:, 0], x[:, 1], x[:, 2], x[:, 3]).astype(np.float64)
    np.testing.assert_allclose(got, g["fresnel_out"], atol=3e-6, rtol=3e-6)


def test_basis(g):
    t1, t2 = oracle.basis(g["basis_in"])
    np.testing.assert_allclose(t1, g["basis_t1"], atol=2e-6)
    np.testing.assert_allclose(t2, g["basis_t2"], atol=2e-6)


def test_dipole_cos(g):
    # the reference's float64 evaluation against the float32 restatement: the inverse CDF amplifies the rounding of
    # its arccos / cos near c = +-1 (dc/du ~ 1 / sqrt(1 - c^2))
    got = oracle.math("dipole_cos", g["phase_u"].astype(np.float32))
    np.testing.assert_allclose(got, g["dipole_cos"], atol=1e-5)


def test_water_rayleigh_table(g):
    e, L = O.water_rayleigh((g["water_e"], g["water_n"]))
    np.testing.assert_allclose(L, g["water_rayleigh"], rtol=1e-6)


def test_geant4_group_index(g):
    got = oracle.group_index(g["water_e"], g["water_n"], g["groupvel_lam"])
    np.testing.assert_allclose(got, g["groupvel_ng"], rtol=2e-6)
