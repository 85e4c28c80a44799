"""The CPU checker (the oracle) against the reference's golden values and closed forms.

- threefry2x32-20 against the Random123 known-answer vectors (the reference's RNG, src/lumen/_core/rng.py);
- the uniforms' contract (open interval, determinism, block stability: src/lumen/_core/rng.py:81-95,
  tests/unit/test_core.py:58-76 of the reference);
- the float32 elementary functions against float64 (ulp bounds);
- the tutorial tank's published run (docs/tutorial/first-hour.md:101-111 of the reference, lumen.simulate with
  samples=2**18, seed=0): per-PMT arrivals, their errors, mean times and expected PE, to the printed digits;
- the weight balance of every photon's fates (src/lumen/api.py:492 Health.balance);
- closed-form sensor spheres (tests/physics/test_toys.py:126-159 of the reference).
"""

import math

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import api, detectors, geometry as G, optics as O, sources
from lumen_b200.detector import build

KEY0 = A.key_of_seed(0)


def test_threefry_known_answers():
    # Random123's known-answer vectors for threefry2x32 with 20 rounds (the ones JAX's tests pin too)
    assert oracle.threefry(0, 0, 0, 0) == (0x6B200159, 0x99BA4EFE)
    assert oracle.threefry(0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF, 0xFFFFFFFF) == (0x1CB996FC, 0xBB002BE7)
    assert oracle.threefry(0x13198A2E, 0x03707344, 0x243F6A88, 0x85A308D3) == (0xC4923A9C, 0x483DF7A0)


def test_uniforms_open_deterministic_block_stable():
    u = oracle.uniforms(KEY0, np.arange(20000), 3, 64).astype(np.float64)
    assert u.min() > 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 5 * math.sqrt(1 / 12 / u.size) and abs(u.var() - 1 / 12) < 1e-3
    assert np.array_equal(u, oracle.uniforms(KEY0, np.arange(20000), 3, 64))
    assert np.array_equal(u[:, :8], oracle.uniforms(KEY0, np.arange(20000), 3, 8))  # a longer draw keeps the first
    assert not np.array_equal(oracle.uniforms(KEY0, [0], 0, 8), oracle.uniforms(KEY0, [0], 1, 8))
    k = (u * 2**23 - 0.5)
    assert np.allclose(k, np.round(k))  # (k + 1/2) 2^-23 exactly


@pytest.mark.parametrize("fn,lo,hi,ulps", [("exp", -80.0, 80.0, 1.0), ("log", 1e-30, 1e30, 2.0),
                                           ("acos", -1.0, 1.0, 1.5), ("cbrt", -8.0, 8.0, 1.0)])  # fmt: skip
def test_math_accuracy(fn, lo, hi, ulps):
    rng = np.random.default_rng(1)
    x = np.float32(rng.uniform(lo, hi, 200000)) if fn != "log" else np.float32(np.exp(rng.uniform(-69, 69, 200000)))
    got = oracle.math(fn, x).astype(np.float64)
    ref = {"exp": np.exp, "log": np.log, "acos": np.arccos, "cbrt": np.cbrt}[fn](x.astype(np.float64))
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    assert np.max(np.abs(got - ref) / ulp) <= ulps


def test_sincos_and_erfinv():
    u = np.float32(np.random.default_rng(2).uniform(0, 1, 100000))
    s, c = oracle.math("sin2pi", u), oracle.math("cos2pi", u)
    a = 2 * np.pi * u.astype(np.float64)
    assert np.max(np.abs(s - np.sin(a))) < 2.5e-7 and np.max(np.abs(c - np.cos(a))) < 2.5e-7
    x = np.float32(np.random.default_rng(3).uniform(-0.999, 0.999, 100000))
    from scipy.special import erfinv

    assert np.max(np.abs(oracle.math("erfinv", x) - erfinv(x.astype(np.float64))) / np.maximum(
        np.abs(erfinv(x.astype(np.float64))), 1e-3)) < 2e-6  # fmt: skip


# the reference's published run of the tutorial tank (docs/tutorial/first-hour.md:101-111)
PUB_ARRIVALS = [394.54, 913.75, 547.76, 501.74, 515.31, 528.14, 320.36, 340.68]
PUB_ERRORS = [17.22, 26.23, 20.30, 19.43, 19.69, 19.94, 15.51, 16.03]
PUB_TIMES = [2.613, 1.699, 2.204, 2.202, 2.208, 2.204, 2.851, 2.844]
PUB_PE = [96.7, 223.9, 134.2, 122.9, 126.3, 129.4, 78.5, 83.5]
TOY_QE = ([300.0, 340.0, 380.0, 420.0, 460.0, 500.0, 540.0, 580.0, 600.0],
          [0.05, 0.20, 0.25, 0.24, 0.20, 0.14, 0.08, 0.04, 0.02])  # examples/data/toy_pmt.json  # fmt: skip


@pytest.fixture(scope="module")
def toy_run():
    det = detectors.toy_tank()
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    n = 1 << 18
    T, _ = oracle.trace(det, KEY0, n, source=src, samples=n)
    return det, T, n


def test_toy_tank_matches_the_published_run(toy_run):
    det, T, n = toy_run
    arr = T.arrival[0]
    err = api.moment_error(T.arrival2[0], arr, n)
    np.testing.assert_allclose(arr, PUB_ARRIVALS, atol=0.0051)
    np.testing.assert_allclose(err, PUB_ERRORS, atol=0.0051)
    np.testing.assert_allclose(T.arrival_t[0] / arr, PUB_TIMES, atol=0.0006)
    q = np.interp(400.0, *TOY_QE)
    np.testing.assert_allclose(arr * q, PUB_PE, atol=0.051)
    # the current rule's deposit records: every cathode crossing draws its covered specular outcome (an edge row,
    # estimator.py:146), and that photon goes on with weight 0 and its reference weight times e / (1 - e), so some
    # reach a second cathode (a record of q = 0) before the roulette ends them
    assert T.counts[A.C_DEPOSITS] == 5735


def test_toy_tank_published_record_count_under_the_rule_of_its_version():
    """The published run reports 'records': 5921 (docs/tutorial/first-hour.md:111). It was made by lumen 0.2.0, whose
    covered draw at a surface absorbing every photon at the reference kept the photon's reference weight
    (CHANGELOG.md, 0.2.1 "A photon in a closed cavity of absorbing walls now ends"): its zero-weight photons bounce on
    between facing cathodes until the water or the tank's wall ends them. Run under that rule the checker makes
    exactly the published count, and the arrivals do not move (those photons carry weight 0)."""
    det = detectors.toy_tank()
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    n = 1 << 18
    with oracle.rule_020():
        T, _ = oracle.trace(det, KEY0, n, source=src, samples=n)
    assert T.counts[A.C_DEPOSITS] == 5921
    np.testing.assert_allclose(T.arrival[0], PUB_ARRIVALS, atol=0.0051)


def test_weight_balance(toy_run):
    det, T, n = toy_run
    h = T.health
    fates = h[[0, 1, 2, 3, 4, 5, 6, 7, 8]].sum()
    assert abs(h[10] - fates) < 1e-6 * h[10]
    tank = detectors.cylinder_tank()
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    T2, _ = oracle.trace(tank, KEY0, 1 << 13, source=src, samples=1 << 13)
    h = T2.health
    assert abs(h[10] - h[[0, 1, 2, 3, 4, 5, 6, 7, 8]].sum()) < 1e-5 * h[10]


def sensor_sphere(A_, L, R, finish):
    """A liquid sphere of radius A_ (absorption length L) in an opaque sensor whose surface reflects R."""
    liquid = O.Material("Liquid", rindex=1.0, abslength=L)
    box = G.Volume("Cathode", G.Box(A_ + 0.5, A_ + 0.5, A_ + 0.5), "Opaque")
    inner = G.Volume("Inner", G.Sphere(A_), "Liquid")
    box.place(inner, (0.0, 0.0, 0.0), name="Inner")
    surf = O.OpticalSurface("Wall", "dielectric_metal", finish, reflectivity=R, efficiency=1.0)
    return build(box, {"Liquid": liquid, "Opaque": O.Material("Opaque")}, borders=[("Inner", "Cathode", surf)],
                 sensors={"s": "Cathode"})  # fmt: skip


def test_specular_sensor_sphere_closed_form():
    # Q = (1 - R) e^{-A/L} / (1 - R e^{-2A/L}) (tests/physics/test_toys.py:126 of the reference)
    A_, L, R = 1.0, 5.0, 0.5
    det = sensor_sphere(A_, L, R, "polished")
    src = sources.Point(position=(0.0, 0.0, 0.0), n_photons=1.0, lam=400.0)
    n = 1 << 14
    T, _ = oracle.trace(det, KEY0, n, source=src, samples=n)
    q = (1 - R) * math.exp(-A_ / L) / (1 - R * math.exp(-2 * A_ / L))
    err = api.moment_error(T.arrival2[0, 0], T.arrival[0, 0], n)
    assert abs(T.arrival[0, 0] - q) < max(4 * err, 3e-5 * q)


def test_lambertian_sensor_sphere_closed_form():
    # Q = (1 - R) e^{-b/2} / (1 - 2 R (1 - (1 + b) e^{-b}) / b^2), b = 2 A / L (test_toys.py:130-159)
    A_, L, R = 1.0, 3.0, 0.6
    det = sensor_sphere(A_, L, R, "ground")
    src = sources.Point(position=(0.0, 0.0, 0.0), n_photons=1.0, lam=400.0)
    n = 1 << 16
    T, _ = oracle.trace(det, KEY0, n, source=src, samples=n)
    b = 2 * A_ / L
    q = (1 - R) * math.exp(-A_ / L) / (1 - 2 * R * (1 - (1 + b) * math.exp(-b)) / b**2)
    err = api.moment_error(T.arrival2[0, 0], T.arrival[0, 0], n)
    assert abs(T.arrival[0, 0] - q) < 4 * err, (T.arrival[0, 0], q, err)


def test_enclosing_sensor_counts_everything_whatever_the_scattering():
    liquid = O.Material("Liquid", rindex=1.33, rayleigh=0.3)
    box = G.Volume("Cathode", G.Box(1.5, 1.5, 1.5), "Opaque")
    box.place(G.Volume("Inner", G.Sphere(1.0), "Liquid"), name="Inner")
    surf = O.OpticalSurface("Wall", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    det = build(box, {"Liquid": liquid, "Opaque": O.Material("Opaque")}, borders=[("Inner", "Cathode", surf)],
                sensors={"s": "Cathode"})  # fmt: skip
    n = 1 << 14
    T, _ = oracle.trace(det, KEY0, n, source=sources.Point((0.1, 0.2, -0.3), 1.0, lam=400.0), samples=n)
    # expected detection over the free path: unbiased, not one per photon (test_toys.py:162-172)
    err = api.moment_error(T.arrival2[0, 0], T.arrival[0, 0], n)
    assert abs(T.arrival[0, 0] - 1.0) < 4 * err, (T.arrival[0, 0], err)
    assert abs(T.health[5] - 1.0) < 1e-6  # every photon's weight ends absorbed at the cathode
    assert T.counts[1] / T.counts[0] > 3  # it scattered


def test_second_moment_is_exact_past_four_sensors():
    """arrival2 is the sum over photons of each photon's own per-sensor sum squared (run.py:483 _moment_adds), for
    any number of sensors a photon deposits on: the LAr box's photons scatter often and deposit their expected
    detection on many of its 120 sensors. Restated here in float64 from the checker's deposit records (photon order,
    each photon's chain ending at its head), and the count of sums past each photon's first four."""
    from lumen_b200.readout import Grid

    det = detectors.lar_box()
    src = sources.Scintillation(position=[(0.3, 0.2, -0.4)], lam=128.0, tau=(6.0, 1500.0), fraction=0.25)
    n = 1 << 12
    T, _ = oracle.trace(det, KEY0, n, source=src, samples=n,
                        groups={"sensor": Grid.bands((100.0, 200.0), nt=2, t0=0.0, dt=1.0)}, deposits=1 << 18)
    nrec = int(T.counts[A.C_RECORDS])
    assert 0 < nrec <= len(T.deposits)
    d = T.deposits[:nrec]
    head = d[:, 17] == 1
    photon = np.concatenate([[0], np.cumsum(head)[:-1]])  # records are in photon order, a head closes a photon
    w0 = d[head, 18].view(np.float32).astype(np.float64)[photon]
    sensor = d[:, 1].view(np.int32).astype(np.int64)
    v = d[:, 2].view(np.float32).astype(np.float64) * w0
    keys, inv = np.unique(photon * det.n_sensor + sensor, return_inverse=True)
    sums = np.zeros(len(keys))
    np.add.at(sums, inv, v)
    want = np.zeros(det.n_sensor)
    np.add.at(want, keys % det.n_sensor, sums**2)
    np.testing.assert_allclose(T.arrival2[0], want, rtol=1e-10, atol=1e-300)
    live = np.unique(keys[sums != 0.0] // det.n_sensor, return_counts=True)[1]
    assert live.max() > 4  # photons with more than four sensors: the register sums alone would not hold them
    assert int(T.counts[A.C_MULTI]) == int(np.maximum(live - 4, 0).sum())


def test_cathode_reflectivity_derivative_at_zero():
    """At a cathode of reflectivity 0 the reference draws its specular outcome from the defensive cover (an edge row,
    estimator.py:146): the photon goes on with weight 0 and the derivative of its weight in R, so the arrivals'
    derivative in R at R = 0 counts the light a reflection would send to the other PMTs. It matches the one-sided
    difference at the reference held at R = 0 (the same paths, weights moving with R)."""
    det = detectors.toy_tank()
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    n = 1 << 16
    key = "surfaces/CathodeSurface/R"
    c = A.controls(grad_tabs=[det.params_index[key]])
    T, _ = oracle.trace(det, KEY0, n, source=src, samples=n, controls=c)
    h = 1e-3
    hi, _ = oracle.trace(det, KEY0, n, source=src, samples=n, pool_live=det.pool_with({key: h}), pool_ref=det.pool)
    lo, _ = oracle.trace(det, KEY0, n, source=src, samples=n)
    jac = T.jac[0, :, 0]
    fd = (hi.arrival[0] - lo.arrival[0]) / h
    # d/dR of (1 - R) eff at the cathode is -1 per arrival; the reflections a cathode sends to the others add to it
    refl = jac + lo.arrival[0]
    assert (refl > -1e-9 * lo.arrival[0]).all() and refl[0] > 0 and refl[1] > 0  # PMTs 0 and 1 face each other
    np.testing.assert_allclose(fd, jac, rtol=2e-3)


def sensitive_cube(R=0.2, eff=0.7, born=True):
    """A 2 m water box holding a 0.4 m water cube that is a sensor (entered through a polished metal border of
    reflectivity R and efficiency eff) whose group counts the photons born inside it (``born``)."""
    water = O.Material("Water", rindex=1.33, abslength=20.0, rayleigh=5.0)
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    cube = G.Volume("Cube", G.Box(0.2, 0.2, 0.2), "Water")
    box.place(cube, (0.3, 0.0, 0.0), name="Cube")
    surf = O.OpticalSurface("Skin", "dielectric_metal", "polished", reflectivity=R, efficiency=eff)
    return build(box, {"Water": water}, borders=[("Box", "Cube", surf)], sensors={"s": "Cube"},
                 born=("s",) if born else ())  # fmt: skip


def test_photons_born_in_a_counting_sensor_deposit_its_entry_detection():
    """src/lumen/transport/step.py:574 _born: a photon emitted inside a sensor that counts by volume deposits, at its
    first step, what the sensor's entry detects at normal incidence ((1 - R) eff here), at its emission time, and ends
    (its whole weight absorbed at a surface); emitted outside, it is counted at the entry as before."""
    R, eff = 0.2, 0.7
    det = sensitive_cube(R, eff)
    assert det.arrays["cls_born"].max() >= 0
    n = 1 << 14
    inside = sources.Point(position=(0.35, 0.05, -0.1), n_photons=1.0, lam=400.0, time=3.0)
    T, _ = oracle.trace(det, KEY0, n, source=inside, samples=n)
    want = np.float32(1.0 - R) * np.float32(eff)
    np.testing.assert_allclose(T.arrival[0, 0], want, rtol=1e-6)
    np.testing.assert_allclose(T.arrival_t[0, 0] / T.arrival[0, 0], 3.0, rtol=1e-6)  # at the emission time
    assert T.counts[A.C_STEPS] == n and T.counts[A.C_DEPOSITS] == n  # one step, one deposit a photon
    h = T.health
    np.testing.assert_allclose(h[5], 1.0, rtol=1e-6)  # every weight absorbed at a surface
    outside = sources.Point(position=(-0.5, 0.0, 0.0), n_photons=1.0, lam=400.0)
    a, _ = oracle.trace(det, KEY0, n, source=outside, samples=n)
    b, _ = oracle.trace(sensitive_cube(R, eff, born=False), KEY0, n, source=outside, samples=n)
    np.testing.assert_allclose(a.arrival, b.arrival, rtol=1e-12)  # entered from outside: unchanged


def test_born_deposit_derivative_in_the_entry_efficiency():
    """The born deposit's tangent: d/d eff of (1 - R) eff is 1 - R per photon."""
    det = sensitive_cube()
    key = "surfaces/Skin/eff"
    c = A.controls(grad_tabs=[det.params_index[key]])
    n = 1 << 12
    inside = sources.Point(position=(0.35, 0.05, -0.1), n_photons=1.0, lam=400.0)
    T, _ = oracle.trace(det, KEY0, n, source=inside, samples=n, controls=c)
    np.testing.assert_allclose(T.jac[0, 0, 0], np.float32(1.0 - 0.2), rtol=1e-6)


def exit_sensor_cube(R=0.0, eff=0.6):
    """A 2 m water box holding a 0.4 m glass cube that is a sensor counted where photons LEAVE it: a border from the
    cube into the water (polished metal, reflectivity R, efficiency eff) whose detection is credited to the cube."""
    water = O.Material("Water", rindex=1.33, abslength=20.0)
    glass = O.Material("Glass", rindex=1.5, abslength=1e6)
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    cube = G.Volume("Cube", G.Box(0.2, 0.2, 0.2), "Glass")
    box.place(cube, (0.3, 0.0, 0.0), name="Cube")
    surf = O.OpticalSurface("Window", "dielectric_metal", "polished", reflectivity=R, efficiency=eff)
    return build(box, {"Water": water, "Glass": glass}, borders=[("Cube", "Box", surf)], sensors={"s": "Cube"})


def test_exit_sensor_credits_the_volume_left():
    """src/lumen/transport/step.py:615 _sensor_dep: at a border out of a sensor's volume whose surface has an
    EFFICIENCY (an exit sensor) the detected share goes to the sensor left. Photons emitted inside the glass cube
    meet its window (reflectivity 0) once: each deposits its efficiency on the cube's sensor, times its survival in
    the glass (absorption length 1e6 m)."""
    eff = 0.6
    det = exit_sensor_cube(0.0, eff)
    assert det.arrays["pair_pre"].sum() == 1
    n = 1 << 14
    src = sources.Point(position=(0.32, 0.05, -0.1), n_photons=1.0, lam=400.0)
    T, _ = oracle.trace(det, KEY0, n, source=src, samples=n)
    assert abs(T.arrival[0, 0] - eff) < 1e-6 * eff  # e^{-0.3 m / 1e6 m} of eff
    # a record at every window crossing: the photons' own, and those of the zero-weight ones the edge row's cover
    # sends back (the window's reflectivity is a keyed parameter at 0: its specular outcome is covered)
    assert T.counts[A.C_DEPOSITS] >= n
