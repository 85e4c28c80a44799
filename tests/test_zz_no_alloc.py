"""lumen_b200_trace_static, the trace entry point that allocates nothing, against lumen_b200_trace.

Some callers cannot allocate device memory during a call, such as a framework whose pool owns the device's memory
while it runs a step. For them the trace's scratch comes from a fixed array in the library. This test calls that entry
point through the C ABI twice in a row, on the same inputs, and checks both results against the allocating entry
point's, within the tolerance of the parity tests (the FP64 tallies' summation order: rel 1e-9). The second call
must not see the first call's counts left in the shared array. The file sorts last, so a run that stops at its
first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

from lumen_b200 import _abi as A
from lumen_b200 import detectors, make, sources
from lumen_b200.engine import DeviceSource, DeviceTallies, Engine

pytestmark = pytest.mark.gpu


def test_static_trace_matches_trace_on_two_calls():
    import torch

    make.build()
    det = detectors.cylinder_tank()
    eng = Engine(det)
    key = A.key_of_seed(0)
    n = 1 << 16
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    ds = DeviceSource(src, n)
    c = A.controls()
    ref = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
    eng.trace(key, n, source=ds, controls=c, tallies=ref)
    lib = A.engine()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for _ in range(2):
        T = DeviceTallies(det.n_sensor, 1, 50, 0.0, 2.0)
        A.check(lib.lumen_b200_trace_static(eng.h, None, ctypes.byref(ds.c), key[0], key[1], 0, n, ctypes.byref(c),
                                            ctypes.byref(T.c), stream))  # fmt: skip
        for name in ("arrival", "arrival_t", "arrival2", "hist"):
            np.testing.assert_allclose(getattr(T, name).cpu().numpy(), getattr(ref, name).cpu().numpy(), rtol=1e-9,
                                       atol=1e-15, err_msg=name)  # fmt: skip
        np.testing.assert_allclose(T.health.cpu().numpy(), ref.health.cpu().numpy(), rtol=1e-7, atol=1e-9)
        assert (T.counts.cpu().numpy()[:5] == ref.counts.cpu().numpy()[:5]).all()
        assert T.counts.cpu().numpy()[0] == n
    eng.close()
