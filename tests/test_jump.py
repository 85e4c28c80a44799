"""The diffusion jump (src/lumen/transport/fastpath.py): a bulk Rayleigh event's walk inside a proven clear ball.

- The clearance grid (lumen_b200.jump, after src/lumen/geometry/clearance.py) is a proven bound: at random points of
  the medium, c(x) = clear[nearest node] - |x - node| never exceeds the true distance to the nearest surface.
- The grid is built only where it can act (a volume at least R_0 = 4 scattering lengths across), so none of the
  benchmark detectors has one.
- The walk is the plain walk in law: the arrivals with and without it agree (chi2 at the reference's suite-wide level)
  and every photon's weight still ends in one fate; it takes fewer steps.
"""

import math

import numpy as np
from scipy import stats

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources

P_MIN = 0.0027 / 400


def _true_distance(x, half, block_c, block_h, discs):
    """The exact distance from points x to the nearest surface of the fog box, its block and its discs."""
    d = np.min(half - np.abs(x), 1)  # the box's own faces, from inside
    o = np.maximum(np.abs(x - block_c) - block_h, 0.0)
    d = np.minimum(d, np.where((np.abs(x - block_c) <= block_h).all(1), 0.0, np.linalg.norm(o, axis=1)))
    for c, ax in discs:  # finite cylinders r 0.3, half-height 0.01
        v = x - c
        z = v @ ax
        rho = np.linalg.norm(v - z[:, None] * ax, axis=1)
        dr, dz = np.maximum(rho - 0.3, 0.0), np.maximum(np.abs(z) - 0.01, 0.0)
        d = np.minimum(d, np.hypot(dr, dz))
    return d


def test_clearance_is_a_proven_bound():
    det = detectors.fog_box()
    a = det.arrays
    assert len(a["jump_i"]) == 1 and a["jump_report"][0]["built"]
    lo, h = a["jump_f"][0, :3].astype(np.float64), float(a["jump_f"][0, 3])
    n = a["jump_i"][0, 1:4]
    clear = a["clear"].reshape(tuple(n)).astype(np.float64)
    rng = np.random.default_rng(0)
    x = rng.uniform(-4.0, 4.0, (200000, 3))
    i = np.clip(np.floor((x - lo) / h + 0.5).astype(int), 0, n - 1)
    node = lo + h * i
    c = clear[i[:, 0], i[:, 1], i[:, 2]] - np.linalg.norm(x - node, axis=1)
    discs = [(np.array(p), np.array(ax, float)) for p, ax in [((-3.98, 0.0, 0.0), (1, 0, 0)), ((3.98, 1.0, 0.0), (-1, 0, 0)),
                                                              ((0.0, -3.98, 1.0), (0, 1, 0)), ((0.5, 0.0, 3.98), (0, 0, -1))]]
    d = _true_distance(x, 4.0, np.array([1.5, -1.0, 0.5]), 0.5, discs)
    assert (c <= d + 1e-6).all(), float((c - d).max())
    assert (c > 0).mean() > 0.1  # the grid does act somewhere


def test_benchmark_detectors_have_no_grid():
    for det in (detectors.toy_tank(), detectors.cylinder_tank(n_pmt=200), detectors.lar_box()):
        assert len(det.arrays["jump_i"]) == 0


def test_jump_is_the_plain_walk_in_law():
    det = detectors.fog_box()
    src = sources.Point(position=(-1.0, 0.5, -0.5), n_photons=1.0, lam=400.0)
    n = 1 << 18
    out = {}
    for flags in (0, A.F_JUMP):
        T, _ = oracle.trace(det, A.key_of_seed(5), n, source=src, samples=n, controls=A.controls(flags=flags))
        h = T.health
        assert abs(h[:10].sum() - h[10]) < 1e-6 * h[10]
        var = np.maximum(T.arrival2[0] - T.arrival[0] ** 2 / n, 0.0) * n / (n - 1)
        out[flags] = (T.arrival[0], var, int(T.counts[1]))
    (a0, v0, s0), (a1, v1, s1) = out[0], out[A.F_JUMP]
    c2 = float(np.sum((a1 - a0) ** 2 / (v0 + v1)))
    assert stats.chi2.sf(c2, len(a0)) > P_MIN, c2
    assert s1 < 0.8 * s0  # the walks skip their queries


def test_jump_jacobian_matches_differences():
    """The walk is drawn at the reference Rayleigh rate and weighted to the live one, so common-random-number
    differences in the fog's lengths reproduce the Jacobian the jump carries (d / d value, every table value moving
    together)."""
    det = detectors.fog_box()
    src = sources.Point(position=(-1.0, 0.5, -0.5), n_photons=1.0, lam=400.0)
    n = 1 << 12
    names = ["media/Fog/rayleigh", "media/Fog/absorption"]
    c = A.controls(grad_tabs=[det.params_index[k] for k in names], flags=A.F_JUMP)
    T, _ = oracle.trace(det, A.key_of_seed(3), n, source=src, samples=n, controls=c)
    assert T.arrival.sum() > 0
    for i, name in enumerate(names):
        off, k = det.arrays["tab"][det.params_index[name]]
        vals = det.pool[off + k:off + 2 * k].astype(np.float64)
        dv = 0.0025 * float(np.abs(vals).min())
        arr = [oracle.trace(det, A.key_of_seed(3), n, source=src, samples=n, pool_live=det.pool_with({name: v}),
                            pool_ref=det.pool, controls=A.controls(flags=A.F_JUMP))[0].arrival[0]
               for v in (vals + dv, vals - dv)]  # fmt: skip
        fd = (arr[0] - arr[1]) / (2 * dv)
        scale = np.max(np.abs(fd))
        np.testing.assert_allclose(T.jac[0][:, i], fd, atol=3e-3 * scale + 1e-12, rtol=3e-3, err_msg=name)
