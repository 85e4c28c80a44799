"""Parity of the CUDA engine with the CPU checker (the oracle), through the C ABI, on the same seeded inputs.

The engine evaluates each photon's path with the checker's arithmetic, operation for operation, so per-photon
records (vertices, deposits, end, first sensor hit, last volume, and the float sums) must agree bit for bit; the FP64
tallies agree to their summation order (atomics on the GPU, per-thread partial sums on the CPU): rel 1e-9.
Navigator queries on fixed ray sets: hit, volumes, classes, surface codes and sensors bit-exact, t and the normal
bit-exact (a stated tolerance of 0 ulp).
"""

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200.engine import DeviceRows, DeviceSource, DeviceTallies, Engine

pytestmark = pytest.mark.gpu

KEY = A.key_of_seed(0)
RTOL = 1e-9  # FP64 tallies: summation order only


@pytest.fixture(scope="module")
def toy():
    return detectors.toy_tank()


@pytest.fixture(scope="module")
def tank():
    return detectors.cylinder_tank()


@pytest.fixture(scope="module")
def lar():
    return detectors.lar_box()


@pytest.fixture(scope="module")
def facet_tank():
    return detectors.cylinder_tank(wall_finish="ground", sigma_alpha=0.1)


@pytest.fixture(scope="module")
def facet_lar():
    return detectors.lar_box(sigma_alpha=0.1)


def _engine(det):
    from lumen_b200 import make as build

    build.build()
    return Engine(det)


def _records_match(det, src, n, samples=None, controls=None):
    eng = _engine(det)
    c = controls or A.controls()
    ds = DeviceSource(src, samples or n)
    gi, gf = eng.trace_photons(KEY, n, source=ds, controls=c)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    _, (oi, of) = oracle.trace(det, KEY, n, source=src, samples=samples or n, records=True, controls=c)
    bad = np.flatnonzero((gi != oi).any(1) | (gf.view(np.uint32) != of.view(np.uint32)).any(1))
    return bad, gi, oi, gf, of


def test_toy_tank_photons_bit_exact(toy, built):
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    bad, gi, oi, gf, of = _records_match(toy, src, 1 << 16, samples=1 << 18)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def test_cylinder_tank_photons_bit_exact(tank, built):
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    bad, gi, oi, gf, of = _records_match(tank, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def test_lar_box_photons_bit_exact(lar, built):
    src = sources.Scintillation(position=[(0.3, 0.2, -0.4)], lam=128.0, tau=(6.0, 1500.0), fraction=0.25)
    bad, gi, oi, gf, of = _records_match(lar, src, 1 << 11)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def _tallies(det, src, n, controls=None, n_bins=0, pools=None):
    eng = _engine(det)
    if pools is not None:
        eng.set_pools(*pools)
    c = controls or A.controls()
    ds = DeviceSource(src, n)
    T = DeviceTallies(det.n_sensor, ds.n_events, n_bins, 0.0, 1.0, c.n_grad)
    eng.trace(KEY, n, source=ds, controls=c, tallies=T)
    O, _ = oracle.trace(det, KEY, n, source=src, samples=n, controls=c, n_events=ds.n_events, n_bins=n_bins,
                        bin_w=1.0, pool_live=None if pools is None else pools[0],
                        pool_ref=None if pools is None else pools[1])
    return T, O


def test_toy_tank_tallies_match(toy, built):
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    T, O = _tallies(toy, src, 1 << 18, n_bins=20)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL)
    np.testing.assert_allclose(T.arrival_t.cpu().numpy(), O.arrival_t, rtol=RTOL)
    np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL)
    np.testing.assert_allclose(T.hist.cpu().numpy(), O.hist, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-7, atol=1e-6)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


def test_tank_tallies_and_gradients_match(tank, built):
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"]
    c = A.controls(grad_tabs=[tank.params_index[k] for k in names])
    T, O = _tallies(tank, src, 1 << 15, controls=c, n_bins=200)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


def test_reference_run_matches(tank, built):
    """A run at live values other than the reference (draws at the reference, weights live / reference)."""
    src = sources.Point(position=(0.0, 2.0, -1.0), n_photons=1.0, lam_range=(300.0, 600.0))
    live = tank.pool_with({"media/Water/absorption": 45.0, "surfaces/BlackSheet/R": 0.12})
    T, O = _tallies(tank, src, 1 << 14, pools=(live, tank.pool))
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-6)


def test_batched_tracks_match(tank, built):
    rng = np.random.default_rng(3)
    e = 16
    u = rng.normal(size=(e, 3))
    src = sources.Tracks(start=rng.uniform(-3, 3, (e, 3)), direction=u, length=rng.uniform(0.5, 3.0, e),
                         lam_range=(300.0, 600.0), counts_=rng.integers(100, 2000, e))
    n = int(src.counts(0).sum())
    T, O = _tallies(tank, src, n)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)


@pytest.fixture(scope="module")
def solids():
    return detectors.solids_box()


@pytest.mark.parametrize("which", ["toy", "tank", "lar", "solids"])
def test_query_and_locate_bit_exact(which, toy, tank, lar, solids, built):
    det = {"toy": toy, "tank": tank, "lar": lar, "solids": solids}[which]
    rng = np.random.default_rng(7)
    n = 20000
    lo, hi = det.arrays["vol_f"][0, 12:15], det.arrays["vol_f"][0, 15:18]
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    eng = _engine(det)
    gi, gf = eng.query(o, d)
    oi, of = oracle.query(det, o, d)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    assert (gi == oi).all(), np.flatnonzero((gi != oi).any(1))[:10]
    assert (gf.view(np.uint32) == of.view(np.uint32)).all()
    gv = eng.locate(o).cpu().numpy()
    assert (gv == oracle.locate(det, o)).all()


def test_adjoint_replay_contracts_the_jacobian(tank, built):
    """lumen_b200_adjoint replays the photons from their keys: sum_s cot[s] d arrival[s] / d theta equals the
    contraction of the trace's Jacobian, and the checker's."""
    src = sources.Point(position=(-2.0, 1.0, 0.5), n_photons=1.0, lam_range=(300.0, 600.0))
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"]
    c = A.controls(grad_tabs=[tank.params_index[k] for k in names])
    n = 1 << 15
    eng = _engine(tank)
    ds = DeviceSource(src, n)
    T = DeviceTallies(tank.n_sensor, 1, 0, 0.0, 1.0, c.n_grad)
    eng.trace(KEY, n, source=ds, controls=c, tallies=T)
    cot = np.random.default_rng(5).normal(size=(1, tank.n_sensor))
    g = eng.adjoint(KEY, n, cot, source=ds, controls=c).cpu().numpy()
    jac = T.jac.cpu().numpy()[0]
    want = cot[0] @ jac
    np.testing.assert_allclose(g, want, rtol=1e-9, atol=1e-12)
    O, _ = oracle.trace(tank, KEY, n, source=src, samples=n, controls=c)
    np.testing.assert_allclose(g, cot[0] @ O.jac[0], rtol=1e-7, atol=1e-12)


def test_facet_tank_photons_bit_exact(facet_tank, built):
    """A ground unified wall (sigma_alpha 0.1): the facet path and its density per photon, as the checker's."""
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    bad, gi, oi, gf, of = _records_match(facet_tank, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def test_facet_lar_photons_bit_exact(facet_lar, built):
    src = sources.Scintillation(position=[(0.3, 0.2, -0.4)], lam=128.0, tau=(6.0, 1500.0), fraction=0.25)
    bad, gi, oi, gf, of = _records_match(facet_lar, src, 1 << 11)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def test_facet_tank_sigma_gradients_match(facet_tank, built):
    """The Jacobian in the wall's sigma_alpha (the facet path's score) and the other optical parameters."""
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R",
             "surfaces/BlackSheet/sigma_alpha"]  # fmt: skip
    c = A.controls(grad_tabs=[facet_tank.params_index[k] for k in names])
    T, O = _tallies(facet_tank, src, 1 << 15, controls=c, n_bins=200)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


def test_facet_reference_run_matches(facet_tank, built):
    """Live sigma_alpha 0.12 against the reference 0.1: the path drawn at 0.1, weighted by its density ratio."""
    src = sources.Point(position=(0.0, 2.0, -1.0), n_photons=1.0, lam_range=(300.0, 600.0))
    live = facet_tank.pool_with({"surfaces/BlackSheet/sigma_alpha": 0.12, "surfaces/BlackSheet/R": 0.12})
    T, O = _tallies(facet_tank, src, 1 << 14, pools=(live, facet_tank.pool))
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("which", ["tank", "facet_lar"])
def test_wavefront_tallies_match(which, tank, facet_lar, built):
    """The wavefront launch (rounds of a query kernel and a step kernel over slots in HBM): the same tallies."""
    if which == "tank":
        det = tank
        src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
        names, n = ["media/Water/absorption", "surfaces/BlackSheet/R"], 1 << 15
    else:
        det = facet_lar
        src = sources.Scintillation(position=[(0.3, 0.2, -0.4), (-1.0, 1.0, 0.5)], lam=128.0, tau=(6.0, 1500.0),
                                    fraction=0.25)  # fmt: skip
        names, n = ["surfaces/CageSurface/R", "media/LAr/rayleigh"], 1 << 12
    for grads in ((), names):
        c = A.controls(grad_tabs=[det.params_index[k] for k in grads], variant=A.VARIANT_WAVEFRONT)
        T, O = _tallies(det, src, n, controls=c, n_bins=50)
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.hist.cpu().numpy(), O.hist, rtol=RTOL, atol=1e-12)
        np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-7, atol=1e-6)
        if grads:
            np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
        assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


@pytest.mark.parametrize("variant", [0, A.VARIANT_WAVEFRONT])
def test_second_moment_past_four_sensors_matches(variant, lar, built):
    """The LAr box's photons deposit on many sensors: the sums past a photon's first four go to the moment table, and
    arrival2 (each photon's per-sensor sum squared) is the checker's exact one; the table never fills."""
    src = sources.Scintillation(position=[(0.3, 0.2, -0.4), (-1.0, 1.0, 0.5)], lam=128.0, tau=(6.0, 1500.0),
                                fraction=0.25)  # fmt: skip
    T, O = _tallies(lar, src, 1 << 14, controls=A.controls(variant=variant))
    np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL, atol=1e-15)
    cnt = T.counts.cpu().numpy()
    assert cnt[A.C_MULTI] == int(O.counts[A.C_MULTI]) > 0
    assert cnt[A.C_MOMENT_LOST] == 0


def test_cathode_reflectivity_derivative_at_zero_matches(toy, built):
    """The toy tank's cathodes (R = 0, an edge row): the covered specular draw carries d/dR; the checker's Jacobian."""
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
    c = A.controls(grad_tabs=[toy.params_index["surfaces/CathodeSurface/R"]])
    for variant in (0, A.VARIANT_WAVEFRONT):
        c.variant = variant
        T, O = _tallies(toy, src, 1 << 16, controls=c)
        np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
        assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


@pytest.mark.parametrize("rounds", [1, 0, 40])
@pytest.mark.parametrize("grad", [False, True])
def test_wavefront_asynchronous_rounds_then_drain_match(rounds, grad, tank, built):
    """LUMEN_F_ASYNC on the wavefront: a fixed number of rounds with no readback (1: the persistent drain does nearly
    everything; 0: the scene's estimate from the synchronous call before; 40: more rounds than the photons need, the
    last ones empty), then the persistent loop resumes the live slots and takes the photons left: the tallies are the
    checker's, as are those of the synchronous call (whose tail the drain takes)."""
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    names = ["media/Water/absorption", "surfaces/BlackSheet/R"] if grad else []
    gt = [tank.params_index[k] for k in names]
    n = 1 << 17
    eng = _engine(tank)
    ds = DeviceSource(src, n)
    O, _ = oracle.trace(tank, KEY, n, source=src, samples=n, controls=A.controls(grad_tabs=gt))
    for flags in (0, A.F_ASYNC):  # the synchronous call first: it sets the scene's estimate
        c = A.controls(grad_tabs=gt, variant=A.VARIANT_WAVEFRONT, flags=flags, wave_slots_log2=16,
                       wave_rounds=rounds)  # fmt: skip
        T = DeviceTallies(tank.n_sensor, 1, 0, 0.0, 1.0, len(gt))
        eng.trace(KEY, n, source=ds, controls=c, tallies=T)
        import torch

        torch.cuda.synchronize()
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-7, atol=1e-6)
        if grad:
            np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
        assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


@pytest.mark.parametrize("which", ["tank", "lar", "facet_lar"])
def test_sensor_reach_bound_changes_no_photon(which, tank, lar, facet_lar, built):
    """LUMEN_F_REACH (src/lumen/geometry/reach.py): bulk steps' queries stop just past the free path where no sensor
    can be met; every photon's record is still the unbounded checker's, bit for bit."""
    c = A.controls(flags=A.F_REACH)
    if which == "tank":
        src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
        bad, gi, oi, gf, of = _records_match(tank, src, 1 << 14, controls=c)
    else:
        det = lar if which == "lar" else facet_lar
        src = sources.Scintillation(position=[(0.3, 0.2, -0.4)], lam=128.0, tau=(6.0, 1500.0), fraction=0.25)
        bad, gi, oi, gf, of = _records_match(det, src, 1 << 11, controls=c)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.fixture(scope="module")
def scint():
    return detectors.scintillator_cube()


def test_scintillator_cube_photons_bit_exact(scint, built):
    """Rayleigh, Mie (G4OpMieHG) and WLS (G4OpWLS) channels in one medium: every photon's record is the checker's."""
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam_range=(330.0, 480.0))
    bad, gi, oi, gf, of = _records_match(scint, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.mark.parametrize("variant", [0, 3])
def test_scintillator_cube_tallies_gradients_and_reference(variant, scint, built):
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam_range=(330.0, 480.0))
    names = ["media/LAB/mie", "media/LAB/wls", "media/LAB/mie_g_forward", "media/LAB/wls_yield", "media/LAB/rayleigh"]
    c = A.controls(grad_tabs=[scint.params_index[k] for k in names], variant=variant)
    T, O = _tallies(scint, src, 1 << 14, controls=c, n_bins=50)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.hist.cpu().numpy(), O.hist, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()
    live = scint.pool_with({"media/LAB/mie_g_forward": 0.85, "media/LAB/wls_yield": 0.8,
                            "media/LAB/mie_forward_ratio": 0.75})  # fmt: skip
    T, O = _tallies(scint, src, 1 << 13, controls=A.controls(variant=variant), pools=(live, scint.pool))
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-6)


@pytest.fixture(scope="module")
def glisur():
    return detectors.glisur_tank()


def test_glisur_tank_photons_bit_exact(glisur, built):
    """GLISUR ground surfaces: a metal wall (cover-drawn facet paths) and a dielectric block (facets that reflect or
    refract, paths that end beyond the surface): every photon's record is the checker's."""
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam=400.0)
    bad, gi, oi, gf, of = _records_match(glisur, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.mark.parametrize("variant", [0, 3])
def test_glisur_tank_tallies_gradients_and_reference(variant, glisur, built):
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam=400.0)
    names = ["surfaces/Wall/polish", "surfaces/BlockIn/polish", "surfaces/BlockOut/polish", "surfaces/Wall/R"]
    c = A.controls(grad_tabs=[glisur.params_index[k] for k in names], variant=variant)
    T, O = _tallies(glisur, src, 1 << 14, controls=c, n_bins=50)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()
    live = glisur.pool_with({"surfaces/Wall/polish": 0.82, "surfaces/BlockIn/polish": 0.72})
    T, O = _tallies(glisur, src, 1 << 13, controls=A.controls(variant=variant), pools=(live, glisur.pool))
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-6)


@pytest.fixture(scope="module")
def fog():
    return detectors.fog_box()


FOG_SRC = sources.Point(position=(-1.0, 0.5, -0.5), n_photons=1.0, lam=400.0)


def test_fog_box_jump_photons_bit_exact(fog, built):
    """The diffusion jump (a Rayleigh walk inside the clearance grid's proven ball): every photon's record is the
    checker's, with the jump on and off."""
    for flags in (A.F_JUMP, 0):
        bad, gi, oi, gf, of = _records_match(fog, FOG_SRC, 1 << 13, controls=A.controls(flags=flags))
        assert len(bad) == 0, f"{flags}: {len(bad)} differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.mark.parametrize("variant", [0, 3])
def test_fog_box_jump_tallies_gradients_and_reference(variant, fog, built):
    names = ["media/Fog/rayleigh", "media/Fog/absorption", "media/Fog/index"]
    c = A.controls(grad_tabs=[fog.params_index[k] for k in names], variant=variant, flags=A.F_JUMP)
    T, O = _tallies(fog, FOG_SRC, 1 << 14, controls=c, n_bins=50)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.hist.cpu().numpy(), O.hist, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
    assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()
    live = fog.pool_with({"media/Fog/rayleigh": 0.55, "media/Fog/absorption": 28.0})
    T, O = _tallies(fog, FOG_SRC, 1 << 13, controls=A.controls(variant=variant, flags=A.F_JUMP),
                    pools=(live, fog.pool))  # fmt: skip
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-6)


CHER = sources.CherenkovSegment("Water", start=[(0.0, 0.0, -0.2), (-0.36, 0.0, 0.0)], direction=[(0, 0, 1), (1, 0, 0)],
                                length=[0.3, 0.12], beta=[0.99, 0.999], charge=[1.0, 2.0])  # fmt: skip


def test_cherenkov_segments_bit_exact(toy, built):
    """Cherenkov segments (src/lumen/sources/cherenkov.py:65): every photon's record and the two events' tallies are
    the checker's; the gradient in the medium's index (which moves the cone) is refused."""
    n = 1 << 14
    eng = _engine(toy)
    ds = DeviceSource(CHER, n, det=toy)
    gi, gf = eng.trace_photons(KEY, n, source=ds, controls=A.controls())
    _, (oi, of) = oracle.trace(toy, KEY, n, source=CHER, samples=n, records=True, n_events=2)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    bad = np.flatnonzero((gi != oi).any(1) | (gf.view(np.uint32) != of.view(np.uint32)).any(1))
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}"
    T = DeviceTallies(toy.n_sensor, 2, 50, 0.0, 1.0, 0)
    eng.trace(KEY, n, source=ds, controls=A.controls(), tallies=T)
    O, _ = oracle.trace(toy, KEY, n, source=CHER, samples=n, n_events=2, n_bins=50)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.hist.cpu().numpy(), O.hist, rtol=RTOL, atol=1e-12)
    np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-9)
    T = DeviceTallies(toy.n_sensor, 2, 0, 0.0, 1.0, 1)
    with pytest.raises(A.EngineError):
        eng.trace(KEY, n, source=ds, controls=A.controls(grad_tabs=[toy.params_index["media/Water/index"]]), tallies=T)


def test_material_scintillation_bit_exact(built):
    """A material's scintillation (src/lumen/sources/scintillation.py: ScintillationPoint, ScintillationSegment with
    Birks' law), drawn at reference shares (1, 0) under the defensive mixture and weighted to live (0.25, 0.75): every
    photon's record and the tallies are the checker's; the source's own tables are refused as gradient parameters."""
    det = detectors.scintillating_tank()
    live = det.pool_with({"media/Scint/scint_share1": 0.25, "media/Scint/scint_share2": 0.75})
    ref = det.pool_with({"media/Scint/scint_share1": 1.0, "media/Scint/scint_share2": 0.0})
    n = 1 << 14
    eng = _engine(det)
    eng.set_pools(live, ref)
    for src in (sources.ScintillationPoint("Scint", position=[(0.0, 0.0, 0.0), (0.2, 0.1, -0.3)], energy=[1.0, 0.5]),
                sources.ScintillationSegment("Scint", start=(-0.2, 0.0, 0.1), end=(0.2, 0.1, -0.1), t_start=1.0,
                                             t_end=3.0, energy=4.0, birks=0.1)):  # fmt: skip
        ds = DeviceSource(src, n, det=det)
        gi, gf = eng.trace_photons(KEY, n, source=ds, controls=A.controls())
        _, (oi, of) = oracle.trace(det, KEY, n, source=src, samples=n, records=True, pool_live=live, pool_ref=ref,
                                   n_events=ds.n_events)  # fmt: skip
        gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
        bad = np.flatnonzero((gi != oi).any(1) | (gf.view(np.uint32) != of.view(np.uint32)).any(1))
        assert len(bad) == 0, f"{type(src).__name__}: {len(bad)} photons differ, first {bad[:5]}"
        T = DeviceTallies(det.n_sensor, ds.n_events, 50, 0.0, 20.0, 0)
        eng.trace(KEY, n, source=ds, controls=A.controls(), tallies=T)
        O, _ = oracle.trace(det, KEY, n, source=src, samples=n, n_events=ds.n_events, n_bins=50, bin_w=20.0,
                            pool_live=live, pool_ref=ref)  # fmt: skip
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.hist.cpu().numpy(), O.hist, rtol=RTOL, atol=1e-12)
    T = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0, 1)
    with pytest.raises(A.EngineError):
        eng.trace(KEY, n, source=ds, controls=A.controls(grad_tabs=[det.params_index["media/Scint/scint_yield"]]),
                  tallies=T)  # fmt: skip


def test_solids_box_photons_bit_exact(solids, built):
    """Photons refracting through every solid of the catalogue (tori by bisection, cones, shells cut in phi and theta,
    quadrics, polycones, polyhedra, polytopes): every photon's record is the checker's."""
    src = sources.Point(position=(0.05, 0.02, -0.6), n_photons=1.0, lam=400.0)
    bad, gi, oi, gf, of = _records_match(solids, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.mark.parametrize(("which", "variant"), [("readout", 0), ("toy", 3)])
def test_truth_records_bit_exact(which, variant, toy, built):
    """Truth rows (LUMEN_F_TRUTH): each photon's analog record (sensor, time, wavelength, 1 / A_n, the crossing point,
    the volume) is the checker's bit for bit, and so are the arrivals of the run whose roulette keeps open analog
    fates; a wavefront request runs the persistent loop."""
    det = detectors.readout_tank() if which == "readout" else toy
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=float(1 << 14), lam_range=(330.0, 480.0))
    n = 1 << 14
    eng = _engine(det)
    ds = DeviceSource(src, n)
    c = A.controls(roulette=0.05, flags=A.F_TRUTH, variant=variant)
    T = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, 0).attach_truth(n)
    eng.trace(KEY, n, source=ds, controls=c, tallies=T)
    O, _ = oracle.trace(det, KEY, n, source=src, samples=n, controls=c, truth=True)
    g = T.truth.cpu().numpy()
    bad = np.flatnonzero((g.view(np.uint32) != O.truth.view(np.uint32)).any(1))
    assert len(bad) == 0, f"{len(bad)} records differ, first {bad[:5]}: gpu {g[bad[:2]]} cpu {O.truth[bad[:2]]}"
    assert (g[:, 0].view(np.int32) >= 0).sum() > 50
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)


def test_simulate_truth_rows(toy, built):
    from lumen_b200 import api
    from lumen_b200 import truth as TR

    n = 1 << 14
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=float(n), lam=400.0)
    light = api.simulate(toy, src, samples=n, seed=0, truth=TR.Truth(keep="absorbed", angle=True, position=True),
                         controls={"jump": False})  # fmt: skip
    O, _ = oracle.trace(toy, KEY, n, source=src, samples=n, controls=A.controls(flags=A.F_TRUTH), truth=True)
    want = TR.rows(TR.Truth(keep="absorbed", angle=True, position=True), toy, O.truth, KEY, 0, None)
    h = light.truth
    np.testing.assert_array_equal(h.photon, want.photon)
    np.testing.assert_array_equal(h.sensor, want.sensor)
    np.testing.assert_array_equal(h.time, want.time)
    np.testing.assert_array_equal(h.detected, want.detected)
    assert h.detected.all() and len(h.photon) > 50  # counting sensors: every absorbed photon is detected
    pos = h.position.astype(np.float64)  # on the PMT discs (r 0.05, half height 0.01): a face or the side
    assert ((np.abs(np.abs(pos[:, 2]) - 0.01) < 1e-5) | (np.abs(np.hypot(pos[:, 0], pos[:, 1]) - 0.05) < 1e-5)).all()
    with pytest.raises(ValueError):
        api.simulate(toy, sources.Point(position=(0.0, 0.0, 0.1), n_photons=2.0 * n, lam=400.0), samples=n,
                     truth=TR.Truth())  # fmt: skip


def _float64_det(which, toy, solids):
    if which == "coated":
        return detectors.coated_panel(precision="float64")
    return {"toy": toy, "solids": solids}[which].with_precision("float64")


@pytest.mark.parametrize("which", ["toy", "solids", "coated"])
def test_float64_query_and_locate_bit_exact(which, toy, solids, built):
    """The float64 navigator (lumen_b200_query64 / locate64): every query's integers and float64 t (and the float32
    normal, widened) are the checker's bit for bit."""
    det = _float64_det(which, toy, solids)
    rng = np.random.default_rng(7)
    n = 20000
    lo, hi = det.arrays["vol_f64"][0, 12:15], det.arrays["vol_f64"][0, 15:18]
    o = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d = d / np.linalg.norm(d, axis=1, keepdims=True)
    eng = _engine(det)
    gi, gf = eng.query(o, d)
    oi, of = oracle.query(det, o, d)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    assert gf.dtype == np.float64 and of.dtype == np.float64
    assert (gi == oi).all(), np.flatnonzero((gi != oi).any(1))[:10]
    assert (gf.view(np.uint64) == of.view(np.uint64)).all()
    gv = eng.locate(o).cpu().numpy()
    assert (gv == oracle.locate(det, o)).all()


@pytest.mark.parametrize("which", ["toy", "solids", "coated"])
def test_float64_photons_bit_exact(which, toy, solids, built):
    """Photons traced with the float64 navigator and position (the NAV64 instantiation): every record is the
    checker's, through the coating float32 steps over too."""
    det = _float64_det(which, toy, solids)
    pos = {"toy": (0.0, 0.0, 0.1), "solids": (0.05, 0.02, -0.6), "coated": (0.0, 0.0, 0.0)}[which]
    src = sources.Point(position=pos, n_photons=1.0, lam=420.0)
    bad, gi, oi, gf, of = _records_match(det, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def test_float64_tallies_gradients_and_truth(tank, toy, built):
    """The float64 instantiations with tangents (G = 8) and with truth rows (ANALOG): tallies, Jacobian and analog
    records are the checker's."""
    det = tank.with_precision("float64")
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    grads = [det.params_index[k] for k in ("media/Water/absorption", "media/Water/rayleigh")]
    c = A.controls(grad_tabs=grads, variant=3)  # a wavefront request runs the persistent loop in float64
    T, O = _tallies(det, src, 1 << 15, controls=c)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
    det = toy.with_precision("float64")
    n = 1 << 14
    src = sources.Point(position=(0.1, 0.0, 0.05), n_photons=float(n), lam_range=(330.0, 480.0))
    eng = _engine(det)
    ds = DeviceSource(src, n)
    c = A.controls(roulette=0.05, flags=A.F_TRUTH)
    Tt = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, 0).attach_truth(n)
    eng.trace(KEY, n, source=ds, controls=c, tallies=Tt)
    Ot, _ = oracle.trace(det, KEY, n, source=src, samples=n, controls=c, truth=True)
    g = Tt.truth.cpu().numpy()
    assert (g.view(np.uint32) == Ot.truth.view(np.uint32)).all()
    np.testing.assert_allclose(Tt.arrival.cpu().numpy(), Ot.arrival, rtol=RTOL, atol=1e-15)


@pytest.mark.parametrize("prec", ["float32", "float64"])
def test_mesh_tank_bit_exact(prec, built):
    """Tessellated meshes (the extended instantiation: chunk items, the watertight test, the facet rule, mesh surface
    codes): queries, locates and photons reflecting off the steel icosphere are the checker's bit for bit."""
    det = detectors.mesh_tank().with_precision(prec)
    dt, ut = (np.float64, np.uint64) if prec == "float64" else (np.float32, np.uint32)
    rng = np.random.default_rng(11)
    n = 20000
    o = rng.uniform(-1.45, 1.45, (n, 3)).astype(dt)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(dt)
    eng = _engine(det)
    gi, gf = eng.query(o, d)
    oi, of = oracle.query(det, o, d)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    assert ((oi[:, 2] > det.arrays["n_vol"])).sum() > 500  # rays that enter a mesh
    assert (gi == oi).all(), np.flatnonzero((gi != oi).any(1))[:10]
    assert (gf.view(ut) == of.view(ut)).all()
    assert (eng.locate(o).cpu().numpy() == oracle.locate(det, o)).all()
    src = sources.Point(position=(0.0, 0.5, -0.6), n_photons=1.0, lam=400.0)
    bad, gi, oi, gf, of = _records_match(det, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.mark.parametrize("which", ["overlap", "protrusion"])
def test_overlapping_siblings_bit_exact(which, built):
    """Overlapping siblings resolved by the ownership rule (an owner a candidate entered as a daughter, the rule's
    order in every locate) and a daughter sticking out of its mother (the mother a candidate whose face is an exit,
    in the extended instantiation): queries, locates and photons are the checker's bit for bit."""
    det = detectors.overlap_box() if which == "overlap" else detectors.protrusion_box()
    rng = np.random.default_rng(13)
    n = 20000
    o = rng.uniform(-0.99, 0.99, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    eng = _engine(det)
    gi, gf = eng.query(o, d)
    oi, of = oracle.query(det, o, d)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    assert (gi == oi).all(), np.flatnonzero((gi != oi).any(1))[:10]
    assert (gf.view(np.uint32) == of.view(np.uint32)).all()
    assert (eng.locate(o).cpu().numpy() == oracle.locate(det, o)).all()
    src = sources.Point(position=(0.0, 0.0, 0.0), n_photons=1.0, lam=400.0)
    bad, gi, oi, gf, of = _records_match(det, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


def test_wire_planes_with_frame_groups_bit_exact(built):
    """Frame groups (the +-60 degree wire planes walked in their own frame by the extended instantiation): queries,
    locates and photons are the checker's bit for bit (the checker scans every candidate: the winner does not depend
    on the traversal)."""
    det = detectors.wire_planes()
    assert det.arrays["n_group"] == 2
    rng = np.random.default_rng(17)
    n = 20000
    o = rng.uniform(-0.99, 0.99, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    eng = _engine(det)
    gi, gf = eng.query(o, d)
    oi, of = oracle.query(det, o, d)
    gi, gf = gi.cpu().numpy(), gf.cpu().numpy()
    assert ((oi[:, 2] > 0) & (oi[:, 2] <= 144)).sum() > 200  # rays that meet a wire
    assert (gi == oi).all(), np.flatnonzero((gi != oi).any(1))[:10]
    assert (gf.view(np.uint32) == of.view(np.uint32)).all()
    assert (eng.locate(o).cpu().numpy() == oracle.locate(det, o)).all()
    src = sources.Point(position=(-0.5, 0.0, 0.0), n_photons=1.0, lam=128.0)
    bad, gi, oi, gf, of = _records_match(det, src, 1 << 14)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"


@pytest.mark.parametrize("variant", [0, A.VARIANT_WAVEFRONT])
def test_batched_events_in_a_captured_graph_match(variant, tank, built):
    """256 uneven track events (the batched workload's shape, its counts log-uniform over 3 .. 300 photons instead of
    1e3 .. 1e6) in one LUMEN_F_ASYNC launch captured in a CUDA graph with its tallies' zeroing, replayed twice: the
    arrivals and the Jacobian per event are the checker's, on both replays; in the persistent loop and in the
    wavefront (its fixed rounds and the drain, no readback)."""
    import torch

    rng = np.random.default_rng(11)
    e = 256
    u = rng.normal(size=(e, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    start = np.column_stack([rng.uniform(-3.3, 3.3, (e, 2)), rng.uniform(-4.0, 4.0, e)])
    counts = np.exp(rng.uniform(np.log(3.0), np.log(300.0), e)).astype(np.int64)
    src = sources.Tracks(start=start, direction=u, length=rng.uniform(0.5, 3.0, e), cone_angle=np.radians(42.0),
                         n_photons=counts.astype(float), lam_range=(300.0, 600.0), counts_=counts)  # fmt: skip
    n = int(counts.sum())
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"]
    gt = [tank.params_index[k] for k in names]
    eng = _engine(tank)
    ds = DeviceSource(src, n)
    c = A.controls(grad_tabs=gt, flags=A.F_ASYNC, variant=variant, wave_slots_log2=16)
    T = DeviceTallies(tank.n_sensor, ds.n_events, 0, 0.0, 1.0, len(gt))
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):  # the first call on the side stream, before the capture
        eng.trace(KEY, n, source=ds, controls=c, tallies=T, stream=stream)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=stream):
        T.zero_()
        eng.trace(KEY, n, source=ds, controls=c, tallies=T, stream=stream)
    O, _ = oracle.trace(tank, KEY, n, source=src, samples=n, controls=A.controls(grad_tabs=gt), n_events=ds.n_events)
    assert O.arrival.shape[0] == e
    for _ in range(2):
        g.replay()
        torch.cuda.synchronize()
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
        assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()
    del g


def test_step_budget_ends_the_launch_with_an_error(tank, built):
    """A device step budget that runs out (LumenControls.step_budget): the kernel stops handing out photons and
    returns, the call raises StepBudgetExhausted, counts[LUMEN_C_ABORTED] is 1, and the engine serves the next call."""
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    eng = _engine(tank)
    n = 1 << 16
    ds = DeviceSource(src, n)
    for variant in (0, A.VARIANT_WAVEFRONT):
        T = DeviceTallies(tank.n_sensor, 1, 0, 0.0, 1.0)
        with pytest.raises(A.StepBudgetExhausted):
            eng.trace(KEY, n, source=ds, controls=A.controls(step_budget=1024, variant=variant), tallies=T)
        cnt = T.counts.cpu().numpy()
        assert cnt[A.C_ABORTED] == 1 and cnt[A.C_PHOTONS] < n
    T, O = _tallies(tank, src, n)
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)


@pytest.mark.parametrize("name", ["cylinder_tank", "lar_box", "solids_box"])
def test_engine_navigator_matches_the_reference_referee(name, built):
    """The engine's locate and query kernels on the reference referee's data (tests/test_reference_oracle.py: the
    reference's float64 Oracle on its own Scene of the detector), at the reference's thresholds."""
    import test_reference_oracle as R

    det = R.MAKERS[name]()
    eng = _engine(det)
    g = R.load(name)

    def query(o, d, v, tm):
        oi, of = eng.query(o, d, v, None, tm)
        return oi.cpu().numpy(), of.cpu().numpy()

    bad_pts, bad_rays, n = R.compare(det, g, lambda x: eng.locate(x).cpu().numpy(), query)
    assert bad_pts <= 2 and bad_rays <= 0.002 * n, (name, bad_pts, bad_rays)
    eng.close()


@pytest.fixture(scope="module")
def ref_dets():
    """The reference pipeline's own detectors (tests/golden/refdet_*.json, ``lumen_b200.reference``)."""
    import os

    from lumen_b200 import reference

    gold = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    return {n: reference.detector(reference.load(os.path.join(gold, f"refdet_{n}.json")))
            for n in ("example_tank", "yaml_toy", "yaml_scint", "yaml_mesh", "yaml_born", "yaml_comb")}  # fmt: skip


@pytest.mark.parametrize(("name", "pos", "n_photons", "lam"), [("example_tank", (0.0, 0.0, 0.1), 2e5, 400.0),
                                                               ("yaml_toy", (0.1, 0.0, 0.2), 1e5, 400.0),
                                                               ("yaml_scint", (0.0, 0.0, 0.1), 1e4, 380.0),
                                                               ("yaml_mesh", (0.0, 0.5, -0.6), 1.0, 400.0),
                                                               ("yaml_born", (0.35, 0.05, -0.1), 1.0, 400.0),
                                                               ("yaml_comb", (0.03, 0.4, 0.2), 1.0, 400.0)])  # fmt: skip
def test_reference_pipeline_detectors_match(name, pos, n_photons, lam, ref_dets, built):
    """The detectors the reference's own pipeline compiled: per-photon records bit-exact, then the tallies, the
    published runs' workloads (the toy tank's arrivals are the published table: tests/test_reference_detector.py)
    and the scintillator (Rayleigh, Mie, WLS)."""  # noqa: D205, D209
    det = ref_dets[name]
    src = sources.Point(position=pos, n_photons=n_photons, lam=lam)
    bad, gi, oi, gf, of = _records_match(det, src, 1 << 15, samples=1 << 18)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"
    for variant in (0, A.VARIANT_WAVEFRONT):
        T, O = _tallies(det, src, 1 << 18, controls=A.controls(variant=variant))
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL)
        np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL)
        np.testing.assert_allclose(T.arrival_t.cpu().numpy(), O.arrival_t, rtol=RTOL)
        assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()


def test_covered_mie_lobe_choice_matches(built):
    """A reference run at a Mie forward ratio of 1 for live values at 0.9: the lobe choice drawn at its defensive
    cover (LUMEN_MI_MIE_COVER), weighted live / covered; tallies and health are the checker's."""
    det = detectors.scintillator_cube(mie=0.5)
    key = "media/LAB/mie_forward_ratio"
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=1e4, lam=450.0)
    pools = (det.pool_with({key: 0.9}), det.pool_with({key: 1.0}))
    for variant in (0, A.VARIANT_WAVEFRONT):
        T, O = _tallies(det, src, 1 << 16, controls=A.controls(variant=variant), pools=pools)
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL)
        np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL)
        np.testing.assert_allclose(T.health.cpu().numpy(), O.health, rtol=1e-6, atol=1e-6)


def _born_cube():
    from lumen_b200 import geometry as G
    from lumen_b200 import optics as O
    from lumen_b200.detector import build

    water = O.Material("Water", rindex=1.33, abslength=20.0, rayleigh=5.0)
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    cube = G.Volume("Cube", G.Box(0.2, 0.2, 0.2), "Water")
    box.place(cube, (0.3, 0.0, 0.0), name="Cube")
    surf = O.OpticalSurface("Skin", "dielectric_metal", "polished", reflectivity=0.2, efficiency=0.7)
    return build(box, {"Water": water}, borders=[("Box", "Cube", surf)], sensors={"s": "Cube"}, born=("s",))


def test_photons_born_in_a_counting_sensor_match(built):
    """A sensor that counts the photons born inside it (LumenSceneDesc.cls_born): a source whose tracks start inside
    and outside the sensor cube; per-photon records bit-exact, tallies with a gradient in the entry efficiency in both
    schedules, and the truth rows' analog records."""
    det = _born_cube()
    rng = np.random.default_rng(3)
    e = 32
    start = np.column_stack([rng.uniform(0.0, 0.6, e), rng.uniform(-0.3, 0.3, e), rng.uniform(-0.3, 0.3, e)])
    u = rng.normal(size=(e, 3))
    u /= np.linalg.norm(u, axis=1)[:, None]
    counts = np.full(e, 512, np.int64)
    src = sources.Tracks(start=start, direction=u, length=rng.uniform(0.1, 0.5, e), cone_angle=np.radians(42.0),
                         n_photons=counts.astype(float), lam_range=(300.0, 600.0), counts_=counts)  # fmt: skip
    n = int(counts.sum())
    bad, gi, oi, gf, of = _records_match(det, src, n)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"
    gt = [det.params_index["surfaces/Skin/eff"]]
    for variant in (0, A.VARIANT_WAVEFRONT):
        T, O = _tallies(det, src, n, controls=A.controls(grad_tabs=gt, variant=variant))
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL)
        np.testing.assert_allclose(T.arrival2.cpu().numpy(), O.arrival2, rtol=RTOL)
        np.testing.assert_allclose(T.jac.cpu().numpy(), O.jac, rtol=1e-7, atol=1e-12)
        assert (T.counts.cpu().numpy()[:5] == O.counts.astype(np.int64)[:5]).all()
    eng = _engine(det)
    ds = DeviceSource(src, n)
    c = A.controls(flags=A.F_TRUTH)
    T = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0, 0).attach_truth(n)
    eng.trace(KEY, n, source=ds, controls=c, tallies=T)
    O, _ = oracle.trace(det, KEY, n, source=src, samples=n, controls=c, truth=True, n_events=ds.n_events)
    g = T.truth.cpu().numpy()
    assert (g.view(np.uint32) == O.truth.view(np.uint32)).all()


def test_exit_sensor_matches(built):
    """An exit sensor (LumenSceneDesc.pair_pre): photons emitted in a glass cube credited where they leave it through
    a window of reflectivity 0.3; records, tallies (persistent and wavefront) and readout-free truth rows."""
    from lumen_b200 import geometry as G
    from lumen_b200 import optics as O
    from lumen_b200.detector import build

    water = O.Material("Water", rindex=1.33, abslength=20.0)
    glass = O.Material("Glass", rindex=1.5, abslength=3.0)
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    cube = G.Volume("Cube", G.Box(0.2, 0.2, 0.2), "Glass")
    box.place(cube, (0.3, 0.0, 0.0), name="Cube")
    surf = O.OpticalSurface("Window", "dielectric_metal", "polished", reflectivity=0.3, efficiency=0.6)
    det = build(box, {"Water": water, "Glass": glass}, borders=[("Cube", "Box", surf)], sensors={"s": "Cube"})
    src = sources.Point(position=(0.32, 0.05, -0.1), n_photons=1.0, lam_range=(300.0, 600.0))
    n = 1 << 15
    bad, gi, oi, gf, of = _records_match(det, src, n)
    assert len(bad) == 0, f"{len(bad)} photons differ, first {bad[:5]}: gpu {gi[bad[:3]]} cpu {oi[bad[:3]]}"
    for variant in (0, A.VARIANT_WAVEFRONT):
        T, O_ = _tallies(det, src, n, controls=A.controls(variant=variant))
        np.testing.assert_allclose(T.arrival.cpu().numpy(), O_.arrival, rtol=RTOL)
        assert T.arrival.cpu().numpy()[0, 0] > 0.3
        assert (T.counts.cpu().numpy()[:5] == O_.counts.astype(np.int64)[:5]).all()
