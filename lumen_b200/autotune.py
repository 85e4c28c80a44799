"""The autotuner: picks the trace's launch shape for a workload by timing it on a sample of the workload's photons.

Tunables (``LumenControls``): the kernel variant (the persistent loop at threads per block x blocks per SM it is
compiled for: 256 x 4 with 64 registers, 128 x 8 with 64, 256 x 3 with 85, the register budget against the warps an
SM switches between; or the wavefront's rounds of a query kernel and a step kernel over slots in HBM) and the
resident blocks per SM launched (fewer blocks can cut atomic contention on small detectors). Each candidate traces the
same photon ids (the same paths: results do not depend on the shape), timed with CUDA events after a warm-up; the
fastest is cached per (detector, source kind, gradient count).
"""

from __future__ import annotations

import torch

from lumen_b200 import _abi as A
from lumen_b200.engine import DeviceTallies

_cache: dict = {}


def candidates(asynchronous=False):
    """The (variant, blocks per SM) shapes to time; the wavefront (host-driven rounds) only for synchronous calls."""
    out = []
    for v in range(A.N_VARIANT):
        if v == A.VARIANT_WAVEFRONT:
            if not asynchronous:
                out.append((v, 0))
            continue
        for bps in (0, 2):
            out.append((v, bps))
    return out


def tune(eng, source, n_sample, grad_tabs=(), n_events=1, key=(0, 0), reps=2, asynchronous=False):
    """Return ((variant, blocks_per_sm), {shape: ms}) for this engine's detector and ``source``
    (``asynchronous``: the shape is for LUMEN_F_ASYNC calls, e.g. under CUDA graph capture)."""  # noqa: D205
    sig = (id(eng.det), getattr(source, "c", None) and source.c.kind, len(grad_tabs), n_events, asynchronous)
    if sig in _cache:
        return _cache[sig]
    T = DeviceTallies(eng.n_sensor, n_events, 0, 0.0, 1.0, len(grad_tabs), eng.device)
    times = {}
    for v, bps in candidates(asynchronous):
        c = A.controls(grad_tabs=grad_tabs, variant=v, blocks_per_sm=bps)
        eng.trace(key, min(n_sample, 1 << 16), source=source, controls=c, tallies=T)
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.trace(key, n_sample, source=source, controls=c, tallies=T)
            e1.record()
            torch.cuda.synchronize(eng.device)
            best = min(best, e0.elapsed_time(e1))
        times[(v, bps)] = best
    pick = min(times, key=times.get)
    _cache[sig] = (pick, times)
    return pick, times
