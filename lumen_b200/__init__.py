"""lumen_b200: the photon-transport hot path of lumen (the photon loop behind ``lumen.simulate``) on NVIDIA B200.

    import lumen_b200 as lumen
    det = lumen.detectors.toy_tank()
    light = lumen.simulate(det, lumen.sources.Point((0, 0, 0.1), lam=400.0, n_photons=2e5), samples=2**18, seed=0)
    light.arrivals, light.arrivals_error, light.mean_arrival_time, light.health

The transport runs in the CUDA library ``lumen_b200/liblumen_b200.so`` (sm_100a) behind the C ABI of
``include/lumen_b200.h``; this package builds detectors, holds device buffers and mirrors lumen's Python API.
"""

from lumen_b200 import autograd, detectors, geometry, optics, reference, sources  # noqa: F401
from lumen_b200.api import Health, Light, moment_error, pe, simulate  # noqa: F401
from lumen_b200.detector import Detector, build  # noqa: F401

__all__ = ["simulate", "Light", "Health", "moment_error", "pe", "Detector", "build", "detectors", "sources",
           "geometry", "optics", "autograd", "reference"]  # fmt: skip
