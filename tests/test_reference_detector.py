"""Detectors from the reference's own host pipeline (``lumen_b200.reference``), against the reference's published runs.

``tests/golden/make_reference_detector.py`` had the reference convert and load its two shipped example detectors
(the tutorial's toy tank from examples/data/example_tank.gdml, the YAML toy from examples/data/yaml_toy) and wrote
what its photon loop runs on: the navigator scene's instances and flattened solids, the compiled optics (classes,
media, the surface table's rows with their Interactions, flags and supports), the packed parameters, the defensive
rows. Here ``reference.detector`` rebuilds them and the checker runs them:

- the toy tank reproduces the reference's published tutorial run (docs/tutorial/first-hour.md:101-111) to every
  printed digit, and is bit for bit the toy tank this package's own builder makes;
- the YAML toy (a tube tank with a ground unified liner, sigma_alpha 0.1, and six disc PMTs) agrees with its
  published run (docs/howto/yaml-detector.md:163, ``arrivals: [518.1 112.9 264.9 148.4 196.5 193.8]``) within the
  run's Monte Carlo error (chi^2 against the mean of 24 seeds), and is bit for bit the same detector built from
  its description by this package's builder. The published numbers are another sequence of draws of the same law
  (no seed of the checker reproduces them: they came from another version of the reference's random stream), so
  the pin is statistical.
"""

import os

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import api, detectors, reference, sources
from lumen_b200 import detector as D
from lumen_b200 import geometry as G
from lumen_b200 import optics as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
KEY0 = A.key_of_seed(0)
N = 1 << 18
RTOL = 1e-12  # FP64 sums of the same photons' deposits over the checker's threads, in another order
PUB_TOY = [394.54, 913.75, 547.76, 501.74, 515.31, 528.14, 320.36, 340.68]  # docs/tutorial/first-hour.md:101-111
PUB_TOY_ERR = [17.22, 26.23, 20.30, 19.43, 19.69, 19.94, 15.51, 16.03]
PUB_YAML = [518.1, 112.9, 264.9, 148.4, 196.5, 193.8]  # docs/howto/yaml-detector.md:163
TOY_SRC = sources.Point(position=(0.0, 0.0, 0.1), n_photons=2e5, lam=400.0)
YAML_SRC = sources.Point(position=(0.1, 0.0, 0.2), n_photons=1e5, lam=400.0)


def converted(name):
    return reference.detector(reference.load(os.path.join(GOLD, f"refdet_{name}.json")))


@pytest.fixture(scope="module")
def toy():
    return converted("example_tank")


@pytest.fixture(scope="module")
def yaml_toy():
    return converted("yaml_toy")


def yaml_toy_own(data):
    """The YAML toy from its description (examples/data/yaml_toy) through this package's builder, the PMTs at the
    poses and the tables on the knots the reference's conversion gave (RINDEX was written on wavelengths)."""  # noqa: D205, D209
    med = {m["name"]: m for m in data["media"]}["Water"]["tables"]
    water = O.Material("Water", rindex=tuple(med["index"]), abslength=tuple(med["absorption"]))
    tank = G.Volume("Tank", G.Tube(rmax=0.5, dz=0.5), "Water")
    pmt = G.Volume("PMT", G.Tube(rmax=0.04, dz=0.01), "Glass")
    for v in data["volumes"]:
        if v["definition"] == "PMT":
            tank.place(pmt, v["t"], v["R"], name=v["path"].split("/")[-1])
    liner = O.OpticalSurface("Liner", "dielectric_metal", "ground", "unified", sigma_alpha=0.1,
                             reflectivity=([1.5, 5.0], [0.1, 0.1]))  # fmt: skip
    cathode = O.OpticalSurface("Cathode", "dielectric_metal", "polished", reflectivity=([1.5, 5.0], [0.0, 0.0]),
                               efficiency=([1.5, 5.0], [1.0, 1.0]))  # fmt: skip
    borders = [("Tank", p.name, cathode) for p in tank.daughters]
    return D.build(tank, {"Water": water, "Glass": O.Material("Glass")}, borders=borders, skins={"Tank": liner},
                   sensors={"pmt": "PMT"}, after_tracking=("pmt",))  # fmt: skip


def test_fixtures_hold_the_reference_products():
    for name, n_vol, n_sensor in (("example_tank", 9, 8), ("yaml_toy", 7, 6)):
        x = reference.load(os.path.join(GOLD, f"refdet_{name}.json"))
        assert len(x["volumes"]) == n_vol and len(x["sensors"]["name"]) == n_sensor
        assert x["class_of"][reference.OUTSIDE_PV] >= 0 and all(r["model"] in reference.MODELS for r in x["rows"])
        assert any(r["edge"] for r in x["rows"])  # the defensive rows came with them


def test_toy_tank_from_the_reference_pipeline_is_the_published_run(toy):
    T, _ = oracle.trace(toy, KEY0, N, source=TOY_SRC, samples=N)
    arr = T.arrival[0]
    np.testing.assert_allclose(arr, PUB_TOY, atol=0.0051)
    np.testing.assert_allclose(api.moment_error(T.arrival2[0], arr, N), PUB_TOY_ERR, atol=0.0051)
    assert T.counts[A.C_DEPOSITS] == 5735  # the current rule's records (tests/test_oracle.py)
    own, _ = oracle.trace(detectors.toy_tank(), KEY0, N, source=TOY_SRC, samples=N)
    for a, b in ((own.arrival, T.arrival), (own.arrival2, T.arrival2), (own.arrival_t, T.arrival_t)):
        np.testing.assert_allclose(a, b, rtol=RTOL)  # the same photons: the threads' summation order only
    assert np.array_equal(own.counts, T.counts)


def test_parameters_carry_the_reference_keys(toy, yaml_toy):
    for key in ("materials/Water/RINDEX", "materials/Water/ABSLENGTH", "surfaces/CathodeSurface/REFLECTIVITY"):
        assert key in toy.params_index
    for key in ("surfaces/Liner/REFLECTIVITY", "surfaces/Liner/sigma_alpha", "surfaces/Cathode/REFLECTIVITY"):
        assert key in yaml_toy.params_index
    # a value given by its key moves the run as the same table of this package's own builder does
    n = 1 << 14
    a, _ = oracle.trace(toy, KEY0, n, source=TOY_SRC, samples=n,
                        pool_live=toy.pool_with({"materials/Water/ABSLENGTH": 10.0}), pool_ref=toy.pool)  # fmt: skip
    own = detectors.toy_tank()
    b, _ = oracle.trace(own, KEY0, n, source=TOY_SRC, samples=n,
                        pool_live=own.pool_with({"media/Water/absorption": 10.0}), pool_ref=own.pool)  # fmt: skip
    np.testing.assert_allclose(a.arrival, b.arrival, rtol=RTOL)


def test_yaml_toy_from_the_reference_pipeline_matches_its_published_run(yaml_toy):
    runs, err = [], []
    for seed in range(24):
        T, _ = oracle.trace(yaml_toy, A.key_of_seed(seed), N, source=YAML_SRC, samples=N)
        runs.append(T.arrival[0])
        err.append(api.moment_error(T.arrival2[0], T.arrival[0], N))
    mean, sd = np.mean(runs, 0), np.mean(err, 0)
    chi2 = float(np.sum(((np.asarray(PUB_YAML) - mean) / sd) ** 2))  # the published run's own error dominates
    assert chi2 / len(PUB_YAML) < 3.0, (mean, sd, chi2)
    assert np.all(np.abs(np.asarray(PUB_YAML) - mean) < 3.5 * sd)


def test_yaml_toy_is_the_detector_its_description_builds(yaml_toy):
    data = reference.load(os.path.join(GOLD, "refdet_yaml_toy.json"))
    own = yaml_toy_own(data)
    rows_ref = yaml_toy.arrays["row_i"].reshape(-1, 16)[:, :6]
    rows_own = own.arrays["row_i"].reshape(-1, 16)[:, :6]
    assert set(map(tuple, rows_ref)) == set(map(tuple, rows_own[rows_own[:, 5] > 0]))  # model, flags and cover
    n = 1 << 16
    a, _ = oracle.trace(yaml_toy, KEY0, n, source=YAML_SRC, samples=n)
    b, _ = oracle.trace(own, KEY0, n, source=YAML_SRC, samples=n)
    np.testing.assert_allclose(a.arrival, b.arrival, rtol=RTOL)
    np.testing.assert_allclose(a.arrival2, b.arrival2, rtol=RTOL)
    assert np.array_equal(a.counts, b.counts)


def test_refused_parts_name_themselves():
    data = reference.load(os.path.join(GOLD, "refdet_yaml_toy.json"))
    with pytest.raises(ValueError, match="not exported"):
        reference.detector(dict(data, format="other"))


def test_scintillator_from_the_reference_pipeline_is_this_builders_cube():
    """The reference's YAML reading of a scintillator cube (tests/golden/yaml_scint: Rayleigh, Mie, a WLS with an
    exponential profile, a ground unified wall) through ``reference.detector``: its media record carries every
    channel with the reference's keys and the Mie lobe's cover, and it traces bit for bit as
    ``detectors.scintillator_cube``, this builder's reading of the same values."""
    d = converted("yaml_scint")
    own = detectors.scintillator_cube()
    for key in ("materials/LAB/MIEHG_FORWARD_RATIO", "materials/LAB/WLSCOMPONENT", "materials/LAB/WLSTIMECONSTANT"):
        assert key in d.params_index
    mi = d.arrays["med_i"].reshape(-1, 16)
    assert mi[0, 11] == 1 and mi[0, 12] == 1  # the exponential profile; the covered lobe choice
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=1e4, lam=380.0)
    n = 1 << 16
    a, _ = oracle.trace(d, KEY0, n, source=src, samples=n)
    b, _ = oracle.trace(own, KEY0, n, source=src, samples=n)
    np.testing.assert_allclose(a.arrival, b.arrival, rtol=RTOL)
    np.testing.assert_allclose(a.arrival2, b.arrival2, rtol=RTOL)
    assert np.array_equal(a.counts, b.counts)


def test_covered_mie_lobe_choice():
    """The Mie lobe choice's defensive cover (src/lumen/media/phase.py:173 ``_mie_cover``, applied where the forward
    ratio is a keyed parameter, src/lumen/transport/medium.py:96): at a reference forward ratio of 1 the backward lobe
    is drawn at e / (1 - e) (the draws differ from the uncovered ones) and weighted live / covered, and the estimate
    for live values at 0.9 agrees with a direct run at 0.9 within its Monte Carlo error; between 0 and 1 the cover is
    the ratio itself (the same draws, bit for bit)."""
    key = "media/LAB/mie_forward_ratio"
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=1e4, lam=450.0)
    n = 1 << 17

    def run(ref_ratio, cover, seed=0):
        det = detectors.scintillator_cube(mie=0.5)
        det.arrays["med_i"].reshape(-1, 16)[0, 12] = cover
        T, _ = oracle.trace(det, A.key_of_seed(seed), n, source=src, samples=n, pool_live=det.pool_with({key: 0.9}),
                            pool_ref=det.pool_with({key: ref_ratio}))  # fmt: skip
        return T

    def total(T):
        return T.arrival[0].sum(), np.sqrt(np.sum(api.moment_error(T.arrival2[0], T.arrival[0], n) ** 2))

    np.testing.assert_allclose(run(0.8, 1).arrival, run(0.8, 0).arrival, rtol=RTOL)
    covered, plain, direct = run(1.0, 1), run(1.0, 0), run(0.9, 1, seed=1)
    assert np.max(np.abs(covered.arrival / plain.arrival - 1.0)) > 1e-6  # other draws, not another summation order
    (a, ea), (b, eb) = total(covered), total(direct)
    assert abs(a - b) < 4.0 * np.hypot(ea, eb), (a, b, ea, eb)


def test_tessellated_parts_from_the_reference_pipeline():
    """``detectors.mesh_tank`` written in the reference's YAML format (tests/golden/make_reference_detector.py
    ``mesh_tank_yaml``: a tessellated steel icosphere with a polished skin, a tessellated black box, a glass orb, eight
    sensor discs, a ground wall) and read by the reference: its meshes are the navigator's opaque pseudo-volumes with
    the reference's classes (the ball's own skin where the water enters it: Geant4's enteredDaughter order), and it
    traces bit for bit as this builder's reading of the same description at the reference's poses (its YAML rotations
    pass through Geant4's angles, which moves a matrix's last bits)."""
    x = reference.load(os.path.join(GOLD, "refdet_yaml_mesh.json"))
    assert [m["pv"].split("/")[-1] for m in x["meshes"]] == ["Ball", "Block"]
    d = reference.detector(x)
    pose = {v["pv"].split("/")[-2]: (v["R"], v["t"]) for v in x["volumes"] if "/" in v["pv"]}
    pose.update({m["pv"].split("/")[-2]: (m["R"], m["t"]) for m in x["meshes"]})
    box = G.Volume("Box", G.Box(1.5, 1.5, 1.5), "Water")
    for name, lv in (("Ball", G.Volume("Ball", G.Mesh(G.icosphere(0.4, 2)), "Steel")),
                     ("Block", G.Volume("Block", G.Mesh(G.box_mesh(0.3, 0.2, 0.25)), "Black")),
                     ("Orb", G.Volume("Orb", G.Orb(0.25), "Glass"))):  # fmt: skip
        box.place(lv, pose[name][1], pose[name][0], name=name)
    pmt = G.Volume("PMT", G.Tube(rmax=0.15, dz=0.01), "Photocathode")
    for i in range(8):
        box.place(pmt, pose[f"PMT_{i}"][1], pose[f"PMT_{i}"][0], name=f"PMT_{i}", copy=i)
    cathode = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    shiny = O.OpticalSurface("Shiny", "dielectric_metal", "polished", reflectivity=0.8)
    wall = O.OpticalSurface("Wall", "dielectric_metal", "ground", reflectivity=0.6, sigma_alpha=0.2, specularlobe=0.5)
    mats = {"Water": O.Material("Water", rindex=1.33, abslength=30.0, rayleigh=10.0),
            "Glass": O.Material("Glass", rindex=1.5, abslength=5.0), "Steel": O.Material("Steel"),
            "Black": O.Material("Black"), "Photocathode": O.Material("Photocathode")}  # fmt: skip
    own = D.build(box, mats, borders=[("Box", f"PMT_{i}", cathode) for i in range(8)],
                  skins={"Box": wall, "Ball": shiny}, sensors={"pmt": "PMT"}, after_tracking=("pmt",))  # fmt: skip
    src = sources.Point(position=(0.0, 0.5, -0.6), n_photons=1.0, lam=400.0)
    n = 1 << 16
    a, _ = oracle.trace(d, KEY0, n, source=src, samples=n)
    b, _ = oracle.trace(own, KEY0, n, source=src, samples=n)
    order = [own.sensors.name.index(s.split("/")[-2]) for s in d.sensors.name]  # the reference's sensor order
    np.testing.assert_allclose(a.arrival[0], b.arrival[0][order], rtol=RTOL)
    np.testing.assert_allclose(a.arrival2[0], b.arrival2[0][order], rtol=RTOL)
    assert np.array_equal(a.counts, b.counts)


def test_any_entry_sensor_counting_photons_born_inside():
    """An ``any_entry`` sensor group (the reference's default count="volume": src/lumen/rules/sensors.py:39
    counts_born) through the reference's pipeline: ``Optics.born_pair`` names the water the cube is entered from, and
    a photon emitted inside the cube deposits at its first step what that entry's counting row detects (1: the group's
    sensor model applies its efficiency after tracking) and ends; emitted outside, it is counted where it enters."""
    x = reference.load(os.path.join(GOLD, "refdet_yaml_born.json"))
    d = reference.detector(x)
    sensor_cls = x["class_of"]["BoxPV/CubePV/Cube"]
    assert x["born_pair"][sensor_cls] == x["class_of"]["BoxPV/Box"]
    assert d.arrays["cls_born"][sensor_cls] == x["class_of"]["BoxPV/Box"]
    n = 1 << 14
    inside = sources.Point(position=(0.35, 0.05, -0.1), n_photons=1.0, lam=400.0, time=2.0)
    T, _ = oracle.trace(d, KEY0, n, source=inside, samples=n)
    assert T.arrival[0, 0] == 1.0 and T.counts[A.C_STEPS] == n
    np.testing.assert_allclose(T.arrival_t[0, 0], 2.0, rtol=1e-7)
    outside = sources.Point(position=(-0.5, 0.0, 0.0), n_photons=1.0, lam=400.0)
    U, _ = oracle.trace(d, KEY0, n, source=outside, samples=n)
    assert 0.0 < U.arrival[0, 0] < 1.0 and U.counts[A.C_STEPS] > n


def test_split_union_pieces_are_volumes_of_their_union():
    """A union of 17 bars (one solid, past the reference's SPLIT_LEAVES = 16: src/lumen/build/lowering.py:699
    split_unions) is placed by the reference as its pieces, each a definition of its own (``Definition.piece_of``)
    whose class is its union's placement's. Converted, the pieces are 17 volumes of that class, and the detector
    traces bit for bit as this builder's 17 separate bars at the same places."""
    x = reference.load(os.path.join(GOLD, "refdet_yaml_comb.json"))
    pieces = [v for v in x["volumes"] if v["piece"]]
    assert len(pieces) == 17 and len({x["class_of"][v["pv"]] for v in pieces}) == 1
    d = reference.detector(x)
    box = G.Volume("Box", G.Box(1.0, 1.0, 1.0), "Water")
    bar = G.Volume("Bar", G.Box(0.02, 0.02, 0.6), "Steel")
    for k, xk in enumerate([0.0] + [-0.85 + 0.1 * k for k in range(1, 17)]):
        box.place(bar, (xk, 0.0, 0.0), name=f"Bar_{k}")
    pmt = G.Volume("PMT", G.Tube(rmax=0.15, dz=0.01), "Photocathode")
    for i, z in enumerate((0.95, -0.95)):
        box.place(pmt, (0.0, 0.0, z), name=f"PMT_{i}", copy=i)
    cathode = O.OpticalSurface("CathodeSurface", "dielectric_metal", "polished", reflectivity=0.0, efficiency=1.0)
    mats = {"Water": O.Material("Water", rindex=1.33, abslength=20.0, rayleigh=5.0), "Steel": O.Material("Steel"),
            "Photocathode": O.Material("Photocathode")}  # fmt: skip
    own = D.build(box, mats, borders=[("Box", f"PMT_{i}", cathode) for i in range(2)], sensors={"pmt": "PMT"},
                  after_tracking=("pmt",))  # fmt: skip
    src = sources.Point(position=(0.03, 0.4, 0.2), n_photons=1.0, lam=400.0)
    n = 1 << 16
    a, _ = oracle.trace(d, KEY0, n, source=src, samples=n)
    b, _ = oracle.trace(own, KEY0, n, source=src, samples=n)
    np.testing.assert_allclose(a.arrival, b.arrival, rtol=RTOL)
    np.testing.assert_allclose(a.arrival2, b.arrival2, rtol=RTOL)
    assert np.array_equal(a.counts, b.counts)
