"""The benchmark workloads at full size on the GPU, checked through properties that do not depend on the size.

The checker finishes a few hundred thousand photons in seconds; the benchmark runs 2^24 (the 2000-PMT tank) and
2^26 (the LAr box). At those sizes the engine is checked against itself, through what the photon loop guarantees
whatever the count:
- the weight balance: every photon's starting weight ends in exactly one fate (health[START] = the sum of the
  fates, src/lumen/api.py:445 Health);
- additivity over photon ids (a checksum of checksums): the tallies of ids [0, n) are the sum of those of [0, n/2)
  and [n/2, n) traced as two calls (first_id), which is also what the multi-GPU sharding relies on;
- schedule independence: the wavefront and the persistent loop give every photon the same path, so the counts
  (photons, steps, deposits) are equal and the FP64 tallies agree to their summation order;
- the moment table holds every sum (counts[MOMENT_LOST] = 0).
"""

import numpy as np
import pytest
import torch

from lumen_b200 import _abi as A
from lumen_b200 import detectors, sources
from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

pytestmark = pytest.mark.gpu

KEY = A.key_of_seed(0)
RTOL = 1e-9  # FP64 tallies of the same photons: the atomics' order only


def _run(eng, ds, n, first=0, variant=A.VARIANT_WAVEFRONT, gt=(), T=None):
    c = A.controls(grad_tabs=list(gt), variant=variant)
    T = T or DeviceTallies(eng.n_sensor, ds.n_events, 0, 0.0, 1.0, len(gt))
    eng.trace(KEY, n, source=ds, first_id=first, controls=c, tallies=T)
    torch.cuda.synchronize()
    return T


def _balance(T):
    h = T.health.cpu().numpy()
    assert abs(h[A.N_HEALTH - 1] - h[:9].sum()) <= 1e-6 * h[A.N_HEALTH - 1], h


def test_headline_tank_at_full_size(built):
    """The headline workload (the 2000-PMT tank, one isotropic point, 300-600 nm) at 2^24 photons."""
    det = detectors.cylinder_tank()
    src = sources.Point(position=(-2.6176, -1.7591, 2.8547), n_photons=1.0, lam_range=(300.0, 600.0))
    n = 1 << 24
    eng = Engine(det)
    ds = DeviceSource(src, n)
    full = _run(eng, ds, n)
    cnt = full.counts.cpu().numpy()
    assert cnt[A.C_PHOTONS] == n and cnt[A.C_MOMENT_LOST] == 0 and cnt[A.C_ABORTED] == 0
    _balance(full)
    halves = DeviceTallies(eng.n_sensor, 1, 0, 0.0, 1.0, 0)
    _run(eng, ds, n // 2, 0, T=halves)
    _run(eng, ds, n // 2, n // 2, T=halves)
    np.testing.assert_allclose(halves.arrival.cpu().numpy(), full.arrival.cpu().numpy(), rtol=RTOL)
    np.testing.assert_allclose(halves.arrival2.cpu().numpy(), full.arrival2.cpu().numpy(), rtol=RTOL)
    assert (halves.counts.cpu().numpy()[:5] == cnt[:5]).all()
    pers = _run(eng, ds, n, variant=0)
    np.testing.assert_allclose(pers.arrival.cpu().numpy(), full.arrival.cpu().numpy(), rtol=RTOL)
    np.testing.assert_allclose(pers.arrival_t.cpu().numpy(), full.arrival_t.cpu().numpy(), rtol=RTOL)
    assert (pers.counts.cpu().numpy()[:5] == cnt[:5]).all()


def test_lar_box_at_full_size_with_gradients(built):
    """The LAr box (10^4 scintillation points, the cage ground unified at sigma_alpha 0.1) at 2^26 photons with the
    Jacobian in two parameters: the balance, the moment table (its photons cross many sensors), and the two halves."""
    det = detectors.lar_box(sigma_alpha=0.1)
    pts = np.random.default_rng(77).uniform([-2.4, -1.9, -1.9], [2.4, 1.9, 1.9], (10000, 3))
    src = sources.Scintillation(position=pts, lam=128.0, tau=(6.0, 1500.0), fraction=0.25, n_photons=1.0)
    gt = [det.params_index[k] for k in ("surfaces/CageSurface/R", "media/LAr/rayleigh")]
    n = 1 << 26
    eng = Engine(det)
    ds = DeviceSource(src, n)
    full = _run(eng, ds, n, gt=gt)
    cnt = full.counts.cpu().numpy()
    assert cnt[A.C_PHOTONS] == n and cnt[A.C_MOMENT_LOST] == 0 and cnt[A.C_MULTI] > 0
    _balance(full)
    halves = DeviceTallies(eng.n_sensor, ds.n_events, 0, 0.0, 1.0, len(gt))
    _run(eng, ds, n // 2, 0, gt=gt, T=halves)
    _run(eng, ds, n // 2, n // 2, gt=gt, T=halves)
    np.testing.assert_allclose(halves.arrival.cpu().numpy(), full.arrival.cpu().numpy(), rtol=RTOL)
    np.testing.assert_allclose(halves.arrival2.cpu().numpy(), full.arrival2.cpu().numpy(), rtol=RTOL)
    np.testing.assert_allclose(halves.jac.cpu().numpy(), full.jac.cpu().numpy(), rtol=1e-7, atol=1e-12)
    assert (halves.counts.cpu().numpy()[:5] == cnt[:5]).all()
