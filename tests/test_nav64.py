"""The float64 navigator (src/lumen/rules/navigation.py:96 Precision, the load option precision="float64",
docs/dev/decisions.md:332) in the checker: the navigator's frames, boxes, leaves, roots, intervals and band and the
photon's position in float64, the physics in float32.

- every solid of the catalogue is located as its own float64 membership says, 1e-9 m from its surface (float32:
  1e-4 m);
- the torus's first crossings are the roots of its quartic to 1e-12 (float32: 2e-5);
- a 3 um coating at 5 m (float32's band there is 4.8 um) is entered by every ray that meets it, and left into the
  backing after exactly its thickness, where float32 steps over it into the backing (the reference's measurement
  behind the option);
- a float64 run's expected values agree in law with a float32 run's;
- a float64 scene without its float64 arrays is refused.
"""

import ctypes

import numpy as np
import pytest
from scipy import stats

import oracle
import test_solids as TS
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200 import geometry as G

KEY = A.key_of_seed(5)
P_MIN = 0.0027 / 400


@pytest.mark.parametrize("name", sorted(TS.CASES))
def test_solids_locate_in_float64(name):
    solid, member = TS.CASES[name]
    det = TS._placed(solid).with_precision("float64")
    rng = np.random.default_rng(3)
    low = solid.lower()
    pl = rng.uniform(low.lo - 0.1, low.hi + 0.1, (40000, 3))
    pw = pl @ TS.ROT.T + TS.POS
    pl = (pw - TS.POS) @ TS.ROT
    m = member(pl)
    sure = np.ones(len(m), bool)
    for a in range(3):
        for s in (-1e-9, 1e-9):
            q = pl.copy()
            q[:, a] += s
            sure &= member(q) == m
    assert sure.sum() > 39900
    v = oracle.locate(det, pw)
    bad = np.flatnonzero(((v == 1) != m) & sure)
    assert len(bad) == 0, f"{name}: {len(bad)} points differ, first {pl[bad[:3]]}"


def test_torus_crossings_in_float64():
    R, r = 0.8, 0.25
    det = TS._placed(G.Torus(rmax=r, rtor=R)).with_precision("float64")
    rng = np.random.default_rng(1)
    o = rng.uniform(-1.5, 1.5, (1500, 3))
    d = rng.normal(size=(1500, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    oi, of = oracle.query(det, o, d)
    assert of.dtype == np.float64
    ol, dl = (o - TS.POS) @ TS.ROT, d @ TS.ROT
    pp = np.polynomial.polynomial
    hits = 0
    for i in range(len(o)):
        a, b = ol[i], dl[i]
        sq = lambda k: pp.polymul([a[k], b[k]], [a[k], b[k]])  # noqa: E731
        xy = pp.polyadd(sq(0), sq(1))
        q = pp.polyadd(pp.polyadd(xy, sq(2)), [R * R - r * r])
        rts = np.roots(pp.polysub(pp.polymul(q, q), 4 * R * R * xy)[::-1])
        rts = rts[(np.abs(rts.imag) < 1e-7) & (rts.real > 1e-6)].real
        t_world = float(np.min((np.sign(d[i]) * 3 - o[i]) / d[i]))
        want = min(rts.min() if len(rts) else t_world, t_world)
        hits += bool(len(rts)) and rts.min() < t_world
        assert abs(of[i, 0] - want) < 1e-12 * (1 + want), (i, of[i, 0], want)
    assert hits > 150


def _coating_rays(n=400):
    rng = np.random.default_rng(0)
    ang, phi = np.deg2rad(rng.uniform(0, 20, n)), rng.uniform(0, 2 * np.pi, n)
    o = np.stack([rng.uniform(0, 1, n), rng.uniform(-0.3, 0.3, n), rng.uniform(-0.3, 0.3, n)], 1)
    d = np.stack([np.cos(ang), np.sin(ang) * np.cos(phi), np.sin(ang) * np.sin(phi)], 1)
    return o, d


def test_a_thin_coating_is_entered_in_float64_only():
    th = 3e-6
    det64 = detectors.coated_panel(thickness=th, precision="float64")
    det32 = det64.with_precision("float32")
    ic, ib = det64.names.index("Coating"), det64.names.index("Backing")
    o, d = _coating_rays()
    t1 = (5.0 - th - o[:, 0]) / d[:, 0]
    p1 = o + t1[:, None] * d
    meets = (np.abs(p1[:, 1]) < 0.999) & (np.abs(p1[:, 2]) < 0.999)
    assert meets.sum() > 200
    oi, of = oracle.query(det64, o, d)
    assert (oi[meets, 2] == ic).all()
    np.testing.assert_allclose(of[meets, 0], t1[meets], rtol=0, atol=1e-12)
    x1 = o + of[:, :1] * d
    oi2, of2 = oracle.query(det64, x1[meets], d[meets], vol=oi[meets, 2], srf=oi[meets, 5])
    assert (oi2[:, 2] == ib).all()  # out of the coating into the backing: after its thickness along the ray
    np.testing.assert_allclose(of2[:, 0], th / d[meets, 0], rtol=1e-6, atol=0)
    oi32, _ = oracle.query(det32, o, d)
    assert (oi32[meets, 2] == ib).all()  # float32 steps over the coating (its band at 5 m: 4.8 um)


@pytest.mark.parametrize("which", ["toy", "coated"])
def test_float64_runs_agree_in_law(which):
    if which == "toy":
        det = detectors.toy_tank()
        src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=float(1 << 16), lam=400.0)
    else:
        det = detectors.coated_panel(thickness=2e-4)  # thick enough for float32 too: the same physics in law
        src = sources.Point(position=(0.0, 0.0, 0.0), n_photons=float(1 << 16), lam=420.0)
    n = 1 << 16
    out = []
    for prec in ("float32", "float64"):
        T = oracle.trace(det.with_precision(prec), KEY, n, source=src, samples=n, controls=A.controls())[0]
        var = np.maximum(T.arrival2[0] - T.arrival[0] ** 2 / n, 0.0) * n / (n - 1)
        out.append((T.arrival[0], var))
        assert abs(T.health[:10].sum() - T.health[10]) < 1e-6 * T.health[10]
    (a0, v0), (a1, v1) = out
    keep = (v0 + v1) > 0
    c2 = float(np.sum((a1 - a0)[keep] ** 2 / (v0 + v1)[keep]))
    assert stats.chi2.sf(c2, keep.sum()) > P_MIN, c2


def test_a_float64_scene_needs_its_arrays():
    det = detectors.toy_tank().with_precision("float64")
    d, keep = det.desc()
    assert d.precision == 1 and bool(d.vol_f64) and bool(d.node_f64)
    d.leaf_f64 = ctypes.cast(None, A.c_f64p)
    vol = np.zeros(1, np.int32)
    st = oracle.lib().lumen_oracle_locate64(ctypes.byref(d), A.dptr(np.zeros(3)), 1, A.iptr(vol))
    assert st == 1  # LUMEN_ERR_ARG
    with pytest.raises(ValueError):
        det.with_precision("float16")
