"""lumen_b200_trace_static, the trace entry point that allocates nothing, against lumen_b200_trace.

Some callers cannot allocate device memory during a call, such as a framework whose pool owns the device's memory
while it runs a step. For them the trace's scratch and its moment table come from fixed arrays in the library. These
tests call that entry point through the C ABI and check its results against the allocating entry point's, within the
tolerance of the parity tests (the FP64 tallies' summation order: rel 1e-9):
- twice in a row on the same inputs: the second call must not see the first call's contents left in the arrays;
- with no allocation from the device's default memory pool (which lumen_b200_trace's scratch comes from) and none by
  torch, while an allocating call on the same inputs does allocate from that pool;
- with gradient parameters (the Jacobian), with truth rows, and on the photons of the LAr box, some of which deposit
  on more than four sensors (their sums held in the fixed moment table);
- after a call whose step budget ran out, whose abort flag the next call must clear.
The file sorts last, so a run that stops at its first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

from lumen_b200 import _abi as A
from lumen_b200 import detectors, make, sources
from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

pytestmark = pytest.mark.gpu

KEY = A.key_of_seed(0)
TANK_SRC = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))


def _stream():
    import torch

    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def _static(eng, ds, n, c, T):
    """One call of lumen_b200_trace_static through the C ABI; returns its status."""
    return A.engine().lumen_b200_trace_static(eng.h, None, ctypes.byref(ds.c), KEY[0], KEY[1], 0, n, ctypes.byref(c),
                                              ctypes.byref(T.c), _stream())  # fmt: skip


def _same(T, ref, n_count=5):
    for name in ("arrival", "arrival_t", "arrival2", "hist"):
        a = getattr(T, name)
        if a is None:
            continue
        np.testing.assert_allclose(a.cpu().numpy(), getattr(ref, name).cpu().numpy(), rtol=1e-9, atol=1e-15,
                                   err_msg=name)  # fmt: skip
    np.testing.assert_allclose(T.health.cpu().numpy(), ref.health.cpu().numpy(), rtol=1e-7, atol=1e-9)
    assert (T.counts.cpu().numpy()[:n_count] == ref.counts.cpu().numpy()[:n_count]).all()


@pytest.fixture(scope="module")
def tank():
    make.build()
    det = detectors.cylinder_tank()
    eng = Engine(det)
    yield det, eng
    eng.close()


def test_static_trace_matches_trace_on_two_calls(tank):
    det, eng = tank
    n = 1 << 16
    ds = DeviceSource(TANK_SRC, n)
    c = A.controls()
    ref = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    eng.trace(KEY, n, source=ds, controls=c, tallies=ref)
    for _ in range(2):
        T = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
        A.check(_static(eng, ds, n, c, T))
        _same(T, ref)
        assert T.counts.cpu().numpy()[0] == n


def _pool_high():
    """The default memory pool's high-water mark of memory in use since it was last reset to 0."""
    import torch
    from cuda.bindings import runtime as rt

    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    err, v = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh)
    assert err == rt.cudaError_t.cudaSuccess
    return int(v), pool


def _pool_reset(pool):
    from cuda.bindings import driver
    from cuda.bindings import runtime as rt

    err, = rt.cudaMemPoolSetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemHigh, driver.cuuint64_t(0))
    assert err == rt.cudaError_t.cudaSuccess


def test_static_trace_allocates_nothing(tank):
    import torch

    det, eng = tank
    n = 1 << 16
    ds = DeviceSource(TANK_SRC, n)
    c = A.controls()
    T = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    A.check(_static(eng, ds, n, c, T))  # its first call on the device looks up the arrays' addresses
    torch.cuda.synchronize()
    _, pool = _pool_high()
    # the control: the allocating entry point takes its scratch and moment table from this pool
    _pool_reset(pool)
    eng.trace(KEY, n, source=ds, controls=c, tallies=DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0))
    torch.cuda.synchronize()
    assert _pool_high()[0] > 0
    # the static entry point: nothing from the pool, nothing from torch's allocator
    T = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    torch.cuda.synchronize()
    before = torch.cuda.memory_stats()
    _pool_reset(pool)
    A.check(_static(eng, ds, n, c, T))
    torch.cuda.synchronize()
    assert _pool_high()[0] == 0
    after = torch.cuda.memory_stats()
    for k in ("allocation.all.allocated", "segment.all.allocated"):
        assert after.get(k, 0) == before.get(k, 0), k


def test_static_trace_gradients_and_variants(tank):
    det, eng = tank
    n = 1 << 15
    ds = DeviceSource(TANK_SRC, n)
    names = ["media/Water/absorption", "media/Water/rayleigh", "surfaces/BlackSheet/R"]
    gt = [det.params_index[k] for k in names]
    ref = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, len(gt))
    eng.trace(KEY, n, source=ds, controls=A.controls(grad_tabs=gt), tallies=ref)
    for variant, bps in ((0, 0), (1, 0), (2, 2), (A.VARIANT_WAVEFRONT, 0)):  # the wavefront runs as shape 0
        T = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0, len(gt))
        A.check(_static(eng, ds, n, A.controls(grad_tabs=gt, variant=variant, blocks_per_sm=bps), T))
        _same(T, ref)
        np.testing.assert_allclose(T.jac.cpu().numpy(), ref.jac.cpu().numpy(), rtol=1e-7, atol=1e-12)


def test_static_trace_truth_rows():
    import torch

    det = detectors.toy_tank()
    eng = Engine(det)
    src = sources.Point(position=(0.0, 0.0, 0.1), n_photons=1.0, lam=400.0)
    n = 1 << 14
    ds = DeviceSource(src, n)
    c = A.controls(flags=A.F_TRUTH)
    ref = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0)
    ref.attach_truth(n)
    eng.trace(KEY, n, source=ds, controls=c, tallies=ref)
    T = DeviceTallies(det.n_sensor, 1, 0, 0.0, 1.0)
    T.attach_truth(n)
    A.check(_static(eng, ds, n, c, T))
    torch.cuda.synchronize()
    _same(T, ref)
    assert (T.truth.cpu().numpy().view(np.uint32) == ref.truth.cpu().numpy().view(np.uint32)).all()
    eng.close()


def test_static_trace_moment_table_on_the_lar_box():
    det = detectors.lar_box()
    eng = Engine(det)
    src = sources.Scintillation(position=[(0.3, 0.2, -0.4), (-1.0, 1.0, 0.5)], lam=128.0, tau=(6.0, 1500.0),
                                fraction=0.25)  # fmt: skip
    n = 1 << 14
    ds = DeviceSource(src, n)
    c = A.controls()
    ref = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0)
    eng.trace(KEY, n, source=ds, controls=c, tallies=ref)
    for _ in range(2):
        T = DeviceTallies(det.n_sensor, ds.n_events, 0, 0.0, 1.0)
        A.check(_static(eng, ds, n, c, T))
        _same(T, ref)
        cnt = T.counts.cpu().numpy()
        assert cnt[A.C_MULTI] > 0 and cnt[A.C_MOMENT_LOST] == 0
    eng.close()


def test_static_trace_after_a_step_budget_abort(tank):
    det, eng = tank
    n = 1 << 16
    ds = DeviceSource(TANK_SRC, n)
    T = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    st = _static(eng, ds, n, A.controls(step_budget=1024), T)
    assert st == A.ERR_STEP_BUDGET
    assert T.counts.cpu().numpy()[A.C_ABORTED] == 1
    ref = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    eng.trace(KEY, n, source=ds, controls=A.controls(), tallies=ref)
    T = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    assert _static(eng, ds, n, A.controls(), T) == 0  # the abort flag left in the array is cleared
    _same(T, ref)
    assert T.counts.cpu().numpy()[A.C_ABORTED] == 0
