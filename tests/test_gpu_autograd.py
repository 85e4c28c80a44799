"""The run as a torch.autograd.Function (lumen_b200.autograd.Simulate): forward lumen_b200_trace, backward
lumen_b200_adjoint, the drop-in for the reference's derivative rule (src/lumen/api.py:748-787).

- torch.autograd.grad of cotangent . arrivals equals cotangent @ Jacobian, the Jacobian of the forward tangents the
  trace carries in the same photons (the engine's) and the checker's: rel 1e-7 (FP64 sums in another order);
- it agrees with central differences of +-1 % at the reference held (common random numbers: the same photons, their
  weights moving with the values), over independent seeds within 3 combined standard errors, and to rel 2e-3.
"""

import numpy as np
import pytest

import oracle
from lumen_b200 import _abi as A
from lumen_b200 import autograd, detectors, sources

pytestmark = pytest.mark.gpu

NAMES = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"]
BASE = [50.0, 80.0, 0.1]
SRC = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))


@pytest.fixture(scope="module")
def tank(built):
    return detectors.cylinder_tank()


def _grad(det, values, cot, n, seed, reference=None):
    import torch

    v = torch.tensor(values, dtype=torch.float64, requires_grad=True)
    arr = autograd.simulate(det, SRC, v, NAMES, samples=n, seed=seed, reference=reference)
    loss = (arr * torch.as_tensor(cot, device=arr.device)).sum()
    (g,) = torch.autograd.grad(loss, v)
    return float(loss), g.numpy()


def test_backward_is_the_jacobian_contraction(tank):
    import torch

    from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

    n = 1 << 14
    cot = np.random.default_rng(5).normal(size=tank.n_sensor)
    loss, g = _grad(tank, BASE, cot, n, 0)
    # the forward tangents of the same photons, on the engine and on the checker
    gt = [tank.params_index[k] for k in NAMES]
    c = A.controls(grad_tabs=gt, flags=A.F_JUMP)
    eng = Engine(tank)
    ds = DeviceSource(SRC, n)
    T = DeviceTallies(tank.n_sensor, 1, 0, 0.0, 1.0, len(gt))
    eng.trace(A.key_of_seed(0), n, source=ds, controls=c, tallies=T)
    torch.cuda.synchronize()
    jac = T.jac.cpu().numpy()[0]
    np.testing.assert_allclose(g, cot @ jac, rtol=1e-7)
    assert loss == pytest.approx(float(cot @ T.arrival.cpu().numpy()[0]), rel=1e-9)
    O, _ = oracle.trace(tank, A.key_of_seed(0), n, source=SRC, samples=n, controls=c)
    np.testing.assert_allclose(g, cot @ O.jac[0], rtol=1e-7)
    eng.close()


def test_backward_matches_common_random_number_differences(tank):
    n, seeds, h = 1 << 16, range(4), 0.01
    cot = np.random.default_rng(6).normal(size=tank.n_sensor)
    gs, fds = [], []
    for seed in seeds:
        _, g = _grad(tank, BASE, cot, n, seed)
        fd = np.zeros(len(NAMES))
        held = dict(zip(NAMES, BASE, strict=True))  # the draws at the base values: the same photons on both sides
        for p in range(len(NAMES)):
            up, dn = list(BASE), list(BASE)
            up[p] *= 1.0 + h
            dn[p] *= 1.0 - h
            lu, _ = _grad(tank, up, cot, n, seed, reference=held)
            ld, _ = _grad(tank, dn, cot, n, seed, reference=held)
            fd[p] = (lu - ld) / (2.0 * h * BASE[p])
        gs.append(g)
        fds.append(fd)
    gs, fds = np.array(gs), np.array(fds)
    d = (gs - fds).mean(0)
    se = np.sqrt(gs.var(0, ddof=1) / len(gs) + fds.var(0, ddof=1) / len(fds))
    assert (np.abs(d) <= 3.0 * se + 1e-12).all(), (d, se)
    np.testing.assert_allclose(gs.mean(0), fds.mean(0), rtol=2e-3)
