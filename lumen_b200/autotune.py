"""The autotuner: picks the trace's launch shape for a workload by timing it on a sample of the workload's photons.

Tunables (``LumenControls``):
- the kernel variant: the persistent loop at the threads per block x blocks per SM it is compiled for (256 x 4 with 64
  registers, 128 x 8 with 64, 256 x 3 with 85: the register budget against the warps an SM switches between), or the
  wavefront's rounds of a query kernel and a step kernel over slots in HBM;
- the persistent loop's resident blocks per SM (fewer blocks: more photons per thread, less atomic contention on
  small detectors);
- the wavefront's photons per slot (its slots 2^k = n / photons per slot: more slots keep more photons in flight,
  fewer leave less state in HBM and a shorter tail of half-empty rounds).
Each candidate traces the same photon ids (the same paths: results do not depend on the shape), timed with CUDA events
after a warm-up; the fastest is cached per (detector, source kind, gradient count, events, asynchronous). An
asynchronous call reads no round back: the wavefront runs the rounds the scene's last synchronous call of that shape
needed per photon a slot carries, and the persistent loop finishes what is left (``LumenControls.wave_rounds``). The BVH
stack depth is the scene's (checked at scene creation against LUMEN_MAX_BVH_DEPTH), not a launch choice.
"""

from __future__ import annotations

import math
from typing import NamedTuple

import torch

from lumen_b200 import _abi as A
from lumen_b200.engine import DeviceTallies

_cache: dict = {}
PHOTONS_PER_SLOT = (2, 4, 8, 16, 32)


class Shape(NamedTuple):
    """A launch shape: the variant, the persistent loop's blocks per SM (0: as many as fit) and the wavefront's
    photons per slot."""  # noqa: D205, D209

    variant: int
    blocks_per_sm: int = 0
    photons_per_slot: int = 0  # 0: the library's default slots (2^21)

    def slots_log2(self, n: int) -> int:
        """The wavefront's slots for a call of n photons: 2^k, n / photons per slot rounded up, k in 16 .. 23 (0:
        the library's default)."""  # noqa: D205
        if self.variant != A.VARIANT_WAVEFRONT or self.photons_per_slot <= 0:
            return 0
        want = max(1, math.ceil(n / self.photons_per_slot))
        return min(23, max(16, math.ceil(math.log2(want))))

    def controls(self, n: int, grad_tabs=(), flags=0, **kw):
        """The LumenControls of a call of n photons in this shape."""
        return A.controls(grad_tabs=grad_tabs, flags=flags, variant=self.variant, blocks_per_sm=self.blocks_per_sm,
                          wave_slots_log2=self.slots_log2(n), **kw)  # fmt: skip

    def label(self) -> str:
        return f"{self.variant}/{self.blocks_per_sm}" + (f"/{self.photons_per_slot}pps"
                                                          if self.variant == A.VARIANT_WAVEFRONT else "")


def candidates(asynchronous=False):
    """The shapes to time: the persistent loop's variants at two resident-block counts, the wavefront at each photons
    per slot (an asynchronous call runs the scene's estimated rounds, then the persistent loop drains the slots)."""  # noqa: D205, D209
    out = []
    for v in range(A.N_VARIANT):
        if v == A.VARIANT_WAVEFRONT:
            out += [Shape(v, 0, p) for p in PHOTONS_PER_SLOT]
            continue
        out += [Shape(v, bps) for bps in (0, 2)]
    return out


def tune(eng, source, n_sample, grad_tabs=(), n_events=1, key=(0, 0), reps=2, asynchronous=False, flags=0):
    """Return (Shape, {label: ms}) for this engine's detector and ``source`` (``asynchronous``: the shape is for
    LUMEN_F_ASYNC calls, e.g. under CUDA graph capture; ``flags``: the run's other LUMEN_F_* flags)."""  # noqa: D205
    sig = (id(eng.det), getattr(source, "c", None) and source.c.kind, len(grad_tabs), n_events, asynchronous, flags)
    if sig in _cache:
        return _cache[sig]
    T = DeviceTallies(eng.n_sensor, n_events, 0, 0.0, 1.0, len(grad_tabs), eng.device)
    times = {}
    shapes = {}
    fl = flags | (A.F_ASYNC if asynchronous else 0)
    for sh in candidates(asynchronous):
        warm = min(n_sample, 1 << 16)
        eng.trace(key, warm, source=source, controls=sh.controls(warm, grad_tabs, fl), tallies=T)
        if asynchronous and sh.variant == A.VARIANT_WAVEFRONT:  # the scene's rounds estimate at this shape
            eng.trace(key, n_sample, source=source, controls=sh.controls(n_sample, grad_tabs, flags), tallies=T)
        c = sh.controls(n_sample, grad_tabs, fl)
        best = float("inf")
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            eng.trace(key, n_sample, source=source, controls=c, tallies=T)
            e1.record()
            torch.cuda.synchronize(eng.device)
            best = min(best, e0.elapsed_time(e1))
        times[sh.label()] = best
        shapes[sh.label()] = sh
    pick = shapes[min(times, key=times.get)]
    if asynchronous and pick.variant == A.VARIANT_WAVEFRONT:  # leave the picked shape's rounds estimate in the scene
        eng.trace(key, n_sample, source=source, controls=pick.controls(n_sample, grad_tabs, flags), tallies=T)
        torch.cuda.synchronize(eng.device)
    _cache[sig] = (pick, times)
    return pick, times
