"""The readout groups on the GPU against the checker, through the C ABI, on the same seeded photons.

The deposit records are the checker's bit for bit (compared as sorted multisets: the engine appends them with
atomics, in no fixed order; their chains differ only in index). The cells are FP64 sums of the same float32 adds in
another order (rel 1e-9), the per-photon moments sum each photon's adds before the square on both sides.
"""

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import api, detectors, sources
from lumen_b200.engine import DeviceSource, DeviceTallies, Engine
from lumen_b200.readout import Axis, Grid, Group, GroupCells

pytestmark = pytest.mark.gpu

KEY = A.key_of_seed(0)
RTOL = 1e-9
SRC = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam_range=(330.0, 480.0))
GRID = Grid(axes=(Axis("wavelength", "wavelength", knots=(300.0, 350.0, 400.0, 450.0, 500.0, 550.0)),
                  Axis("theta", "theta", knots=(0.0, 0.5, 1.0, 1.6))),
            delay_axes=(Axis("inc", "cos_incidence", edges=(0.0, 0.5, 1.0)),), t0=-2.0, dt=0.5, nt=60, weighted=True,
            normalise=True)  # fmt: skip
BANDS = Grid(axes=(Axis("gen", "generation", edges=(-0.5, 0.5, 1.5, 9.5)), Axis("rho", "rho", knots=(0.0, 0.05))),
             nt=40, t0=0.0, dt=1.0)  # fmt: skip


@pytest.fixture(scope="module")
def det():
    return detectors.readout_tank()


def _groups(det):
    w = np.random.default_rng(0).uniform(0.1, 0.3, GRID.shape)
    return {"pmt": Group(GRID, tuple(det.groups["pmt"]), w), "ref": BANDS}


def _pair(det, n, variant=0, capacity=1 << 16, static=False):
    from lumen_b200 import make as build

    build.build()
    eng = Engine(det)
    ds = DeviceSource(SRC, n)
    T = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0, 0)
    G = GroupCells(det, _groups(det), ds.n_events, eng.device)
    T.attach_groups(G, capacity)
    c = A.controls(variant=variant)
    if static:
        import ctypes

        A.check(eng.lib.lumen_b200_trace_static(eng.h, None, ctypes.byref(ds.c), KEY[0], KEY[1], 0, n, ctypes.byref(c),
                                                ctypes.byref(T.c), None))  # fmt: skip
    else:
        eng.trace(KEY, n, source=ds, controls=c, tallies=T)
    O, _ = oracle.trace(det, KEY, n, source=SRC, samples=n, controls=c, groups=_groups(det), deposits=capacity)
    return T, G, O


def _check(T, G, O):
    np.testing.assert_allclose(T.arrival.cpu().numpy(), O.arrival, rtol=RTOL, atol=1e-15)
    nrec = int(O.counts[A.C_RECORDS])
    assert int(T.counts[A.C_RECORDS].item()) == nrec > 0
    for k, name in enumerate(G.names):
        for kind, a in G.cells[k].items():
            np.testing.assert_allclose(a.cpu().numpy(), O.groups.cells[k][kind], rtol=RTOL, atol=1e-15,
                                       err_msg=f"{name} {kind}")  # fmt: skip
    np.testing.assert_allclose(G.pe2.cpu().numpy(), O.groups.pe2, rtol=RTOL, atol=1e-18)
    # the records' facts: the same multiset, bit for bit (words 1-16: sensor, q, time, lam, 1 / A_n, gen, volume,
    # the crossing point, direction and normal)
    g = T.records[:nrec].cpu().numpy().view(np.uint32)[:, 1:17]
    o = O.deposits[:nrec, 1:17]
    key = lambda a: a[np.lexsort(a.T[::-1])]  # noqa: E731
    np.testing.assert_array_equal(key(g), key(o))


@pytest.mark.parametrize("variant", [0, 3])
def test_groups_match_the_checker(variant, det):
    T, G, O = _pair(det, 1 << 13, variant)
    _check(T, G, O)


def test_static_entry_point_fills_the_groups(det):
    T, G, O = _pair(det, 1 << 12, static=True)
    _check(T, G, O)


def test_records_overflow_is_reported_and_fills_nothing(det):
    n = 1 << 12
    from lumen_b200 import make as build

    build.build()
    eng = Engine(det)
    ds = DeviceSource(SRC, n)
    T = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, 0)
    G = GroupCells(det, _groups(det), 1, eng.device)
    T.attach_groups(G, 16)
    with pytest.raises(A.RecordsOverflow):
        eng.trace(KEY, n, source=ds, controls=A.controls(), tallies=T)
    assert int(T.counts[A.C_RECORDS].item()) > 16
    assert all(float(a.abs().sum()) == 0.0 for cells in G.cells for a in cells.values())


def test_simulate_fills_groups_and_retries(det):
    n = 1 << 13
    light = api.simulate(det, SRC, samples=n, seed=0, groups=_groups(det), records=64)  # forces the retry
    O, _ = oracle.trace(det, KEY, n, source=SRC, samples=n, groups=_groups(det), deposits=1 << 16,
                        controls=A.controls(flags=A.F_JUMP))  # fmt: skip
    H = O.groups.histograms(n)
    for name, h in light.groups.items():
        np.testing.assert_allclose(h.charge, H[name].charge, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(h.time, H[name].time, rtol=RTOL, atol=1e-15)
        np.testing.assert_allclose(h.late, H[name].late, rtol=RTOL, atol=1e-15)
    qe = np.linspace(0.1, 0.3, GRID.shape[0])
    p = api.pe(light, {"pmt": {"tables": [(("wavelength",), qe)], "efficiency": 0.9}})
    want = 0.9 * np.einsum("slt,l->s", light.groups["pmt"].charge, qe)
    np.testing.assert_allclose(p[list(det.groups["pmt"])], want, rtol=1e-12)
    assert (p[list(det.groups["ref"])] == 0).all()
    assert (api.pe_error(light)[list(det.groups["pmt"])] > 0).all()
