"""The readout groups (src/lumen/readout/grid.py, fill.py:88): the checker's binning against a numpy restatement of the
reference's formulas applied to the checker's own deposit records, and the identities the histograms keep.

- charge: each deposit's q (times 1 / A_n on a normalising grid) on its cells with hat weights (knots) or one cell
  (edges), row-major over the axes; charge2 per cell and pe2 per sensor square each photon's summed adds;
- time: the cubic Lagrange split over the four nearest nodes, the signed shares beyond the ends into late / early
  (q and q t), weighted by the acceptance read at the deposit's charge cells;
- identities: hat weights sum to 1 (a knots-only grid's charge sums to the arrivals), the cubic weights sum to 1 (a
  sensor's time nodes plus its overflow hold its detection-weighted charge);
- 1 / A_n of a photocathode (complex index) at normal incidence: the closed form 1 / (1 - |r|^2),
  r = (n1 - n2) / (n1 + n2) with n2 = nr + i nk.
"""

import math

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200.readout import Axis, Grid, Group, expected_pe, tables_acceptance

SRC = sources.Point(position=(0.1, 0.0, 0.05), n_photons=1.0, lam_range=(330.0, 480.0))
GRID = Grid(axes=(Axis("wavelength", "wavelength", knots=(300.0, 350.0, 400.0, 450.0, 500.0, 550.0)),
                  Axis("theta", "theta", knots=(0.0, 0.5, 1.0, 1.6))),
            delay_axes=(Axis("inc", "cos_incidence", edges=(0.0, 0.5, 1.0)),), t0=-2.0, dt=0.5, nt=60, weighted=True,
            normalise=True)  # fmt: skip
BANDS = Grid.bands((300.0, 400.0, 500.0, 600.0), nt=40, t0=0.0, dt=1.0)


@pytest.fixture(scope="module")
def run():
    det = detectors.readout_tank()
    w = np.random.default_rng(0).uniform(0.1, 0.3, GRID.shape)
    groups = {"pmt": Group(GRID, tuple(det.groups["pmt"]), w), "ref": BANDS}
    n = 1 << 13
    T, _ = oracle.trace(det, A.key_of_seed(0), n, source=SRC, samples=n, groups=groups, deposits=1 << 16)
    return det, groups, n, T


def _features(det, d):
    """The records' features (float64 here; the checker computes them in float32)."""
    f = d.view(np.float32).astype(np.float64)
    vol = d[:, 7].astype(np.int64)
    vf = np.asarray(det.arrays["vol_f"], np.float64)[vol]
    R, t = vf[:, 0:9].reshape(-1, 3, 3), vf[:, 9:12]
    loc = lambda v: np.einsum("nij,ni->nj", R, v)  # noqa: E731 -- R^T v
    p = loc(f[:, 8:11] - t)
    cos_inc = np.abs(np.sum(loc(f[:, 11:14]) * loc(f[:, 14:17]), 1))
    return {"wavelength": f[:, 4], "theta": np.arctan2(np.sqrt(p[:, 0] ** 2 + p[:, 1] ** 2 + 1e-30), p[:, 2]),
            "cos_incidence": cos_inc, "generation": d[:, 6].astype(np.float64), "x": p[:, 0], "y": p[:, 1],
            "z": p[:, 2], "rho": np.hypot(p[:, 0], p[:, 1])}  # fmt: skip


def _axis_cells(ax, x):
    v = np.asarray(ax.values)
    c = np.searchsorted(v, x, side="right")
    if ax.knots is not None:  # grid.py:165 hats
        i = np.clip(c - 1, 0, len(v) - 2)
        f = np.clip((x - v[i]) / (v[i + 1] - v[i]), 0.0, 1.0)
        return [(i, 1.0 - f), (i + 1, f)]
    b = c - 1
    return [(np.where((b >= 0) & (b < len(v) - 1), b, -1), np.ones_like(x))]


def _cells(axes, feats):
    out = None
    for ax in axes:  # grid.py:173 cells: row-major
        cs = _axis_cells(ax, feats[ax.feature])
        if out is None:
            out = cs
            continue
        out = [(np.where((i >= 0) & (j >= 0), i * ax.size + j, -1), w * v) for i, w in out for j, v in cs]
    n = len(next(iter(feats.values())))
    return out if out is not None else [(np.zeros(n, np.int64), np.ones(n))]


def _restate(det, groups, d, n_sensor):
    """Bin records d (photon-ordered, the engine's layout) as grid.py / fill.py do: {group: (charge, charge2, time,
    over_q, over_qt)}, pe2."""  # noqa: D205, D209
    f = d.view(np.float32).astype(np.float64)
    sensor, q, time, inv_an = d[:, 1].astype(np.int64), f[:, 2], f[:, 3], f[:, 5]
    photon = np.cumsum(np.concatenate([[0], d[:-1, 17]])).astype(np.int64)  # a head ends its photon's run
    w0 = np.zeros(len(d))
    for p in np.unique(photon):
        sel = np.flatnonzero(photon == p)
        w0[sel] = f[sel[-1], 18]
    feats = _features(det, d)
    out, pe2 = {}, np.zeros(n_sensor)
    for name, g in groups.items():
        gr, sens, wts = (g.grid, g.sensors, g.weights) if isinstance(g, Group) else (g, None, None)
        sens = det.groups[name] if sens is None else sens
        pos = np.full(n_sensor, -1)
        pos[list(sens)] = np.arange(len(sens))
        ns = len(sens)
        mine = pos[sensor] >= 0
        qd = q * inv_an if gr.normalise else q
        charge = np.zeros(ns * gr.n_cells)
        m2 = {}
        acc = np.zeros(len(d))
        for idx, w in _cells(gr.axes, feats):
            ok = mine & (idx >= 0)
            flat = pos[sensor] * gr.n_cells + idx
            np.add.at(charge, flat[ok], (qd * w * w0)[ok])
            for k in np.flatnonzero(ok):
                m2[(photon[k], flat[k])] = m2.get((photon[k], flat[k]), 0.0) + qd[k] * w[k] * w0[k]
            if wts is not None:
                acc[ok] += (w * np.asarray(wts).ravel()[np.maximum(idx, 0)])[ok]
        charge2 = np.zeros_like(charge)
        for (_, c), v in m2.items():
            charge2[c] += v * v
        if wts is not None:
            mp = {}
            for k in np.flatnonzero(mine):
                mp[(photon[k], sensor[k])] = mp.get((photon[k], sensor[k]), 0.0) + qd[k] * acc[k] * w0[k]
            for (_, s), v in mp.items():
                pe2[s] += v * v
        tm = oq = oqt = None
        if gr.nt:
            qq = qd * (acc if gr.weighted else 1.0)
            x = np.clip((time - gr.t0) / gr.dt, -4.0, gr.nt + 4.0)
            j = np.floor(x)
            gg = x - j
            j = j.astype(np.int64)
            tc = [(j - 1, -gg * (gg - 1) * (gg - 2) / 6), (j, (gg + 1) * (gg - 1) * (gg - 2) / 2),
                  (j + 1, -(gg + 1) * gg * (gg - 2) / 2), (j + 2, (gg + 1) * gg * (gg - 1) / 6)]  # fmt: skip
            late = sum(np.where(nn >= gr.nt, fw, 0.0) for nn, fw in tc)
            early = sum(np.where(nn < 0, fw, 0.0) for nn, fw in tc)
            tm, oq, oqt = np.zeros(ns * gr.n_delay * gr.nt), np.zeros(ns * gr.n_delay * 2), np.zeros(ns * gr.n_delay * 2)
            for bi, bw in _cells(gr.delay_axes, feats):
                ok = mine & (bi >= 0)
                row = pos[sensor] * gr.n_delay + bi
                for nn, fw in tc:
                    o2 = ok & (nn >= 0) & (nn < gr.nt)
                    np.add.at(tm, (row * gr.nt + nn)[o2], (qq * bw * fw * w0)[o2])
                for side, sh in ((0, late), (1, early)):
                    np.add.at(oq, (row * 2 + side)[ok], (qq * bw * sh * w0)[ok])
                    np.add.at(oqt, (row * 2 + side)[ok], (qq * bw * sh * time * w0)[ok])
        out[name] = (charge, charge2, tm, oq, oqt)
    return out, pe2


def test_checker_binning_matches_the_restatement(run):
    det, groups, n, T = run
    nrec = int(T.counts[A.C_RECORDS])
    assert 0 < nrec <= len(T.deposits)
    d = T.deposits[:nrec]
    assert d[-1, 17] == 1 and (d[:, 0].view(np.int32)[1:][d[:-1, 17] == 1] == -1).all()  # chains per photon
    ref, pe2 = _restate(det, groups, d, det.n_sensor)
    for k, cells in enumerate(T.groups.cells):
        name = T.groups.names[k]
        for kind, want in zip(("charge", "charge2", "time", "over_q", "over_qt"), ref[name]):
            if want is None:
                continue
            got = cells[kind]
            scale = float(np.abs(want).max()) or 1.0
            np.testing.assert_allclose(got, want, rtol=2e-5, atol=1e-6 * scale, err_msg=f"{name} {kind}")
    np.testing.assert_allclose(T.groups.pe2[: det.n_sensor], pe2, rtol=2e-5, atol=1e-12)


def test_histogram_identities(run):
    det, groups, n, T = run
    H = T.groups.histograms(n)
    ref = H["ref"]  # edges covering every wavelength the run has: a sensor's charge is its arrivals
    np.testing.assert_allclose(ref.charge.sum(1), T.arrival[0][list(det.groups["ref"])], rtol=1e-12)
    total = ref.time.sum(-1) + ref.late[..., 0] + ref.early[..., 0]  # the cubic weights sum to 1
    np.testing.assert_allclose(total, ref.charge.sum(1), rtol=1e-5, atol=1e-12)
    pmt = H["pmt"]  # knots: hat weights sum to 1; a normalised deposit is q / A_n > q
    assert (pmt.charge.sum((1, 2)) > T.arrival[0][list(det.groups["pmt"])]).all()
    acc = groups["pmt"].weights
    pe = expected_pe(pmt, acc)
    np.testing.assert_allclose(pmt.time.sum((-1, -2)) + pmt.late[..., 0].sum(-1) + pmt.early[..., 0].sum(-1), pe,
                               rtol=1e-5)  # fmt: skip
    assert (pmt.charge2 >= 0).all() and (pmt.pe_error > 0).all()
    assert (pmt.pe_error < pe).all()


def test_normal_absorptance_of_a_photocathode(run):
    det, groups, n, T = run
    d = T.deposits[: int(T.counts[A.C_RECORDS])]
    f = d.view(np.float32)
    pmt = np.isin(d[:, 1], det.groups["pmt"])
    lam = f[pmt, 4].astype(np.float64)
    e = 1239.84198433200208 / lam
    n1 = np.interp(e, [1.5, 2.5, 3.5, 5.0], [1.47, 1.48, 1.50, 1.53])
    r = (n1 - (2.7 + 1.5j)) / (n1 + (2.7 + 1.5j))
    np.testing.assert_allclose(f[pmt, 5], 1.0 / (1.0 - np.abs(r) ** 2), rtol=2e-5)
    np.testing.assert_array_equal(f[~pmt, 5], 1.0)  # a row not read per normal incidence: 1


def test_grid_and_group_checks():
    with pytest.raises(ValueError):
        Axis("w", "wavelength", knots=(400.0, 300.0))
    with pytest.raises(ValueError):
        Axis("w", "colour", knots=(300.0, 400.0))
    with pytest.raises(ValueError):
        Axis("w", "wavelength", knots=(300.0, 400.0), edges=(1.0, 2.0))
    with pytest.raises(ValueError):
        Grid(nt=5, dt=0.0)
    ax = [Axis(f"a{i}", "x", knots=(0.0, 1.0)) for i in range(5)]
    with pytest.raises(ValueError):
        Grid(axes=tuple(ax))
    det = detectors.readout_tank()
    from lumen_b200.readout import GroupCells

    with pytest.raises(ValueError):  # a weighted grid reads its acceptance
        GroupCells(det, {"pmt": GRID})
    with pytest.raises(ValueError):  # a sensor in two groups
        GroupCells(det, {"pmt": BANDS, "all": Group(BANDS, None)})


def test_tables_acceptance_broadcasts_in_axis_order():
    g = Grid(axes=(Axis("wavelength", "wavelength", knots=(300.0, 400.0, 500.0)), Axis("theta", "theta", knots=(0.0, 1.0))))
    qe, ce = np.array([0.1, 0.2, 0.3]), np.array([1.0, 0.5])
    acc = tables_acceptance(g, [(("wavelength",), qe), (("theta",), ce)])
    np.testing.assert_allclose(acc, np.outer(qe, ce))
    both = tables_acceptance(g, [(("theta", "wavelength"), np.outer(ce, qe))])
    np.testing.assert_allclose(both, np.outer(qe, ce))
    assert math.isclose(float(acc.sum()), float(qe.sum() * ce.sum()))
