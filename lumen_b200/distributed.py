"""The run across ranks: contiguous photon-id ranges per rank, one all-reduce of the tallies.

The reference runs a simulation's photons in chunks of contiguous ids, each keyed by ``fold_in(key, first_id + i)``,
and adds the chunks' exact sums (src/lumen/api.py:1078-1111, src/lumen/run.py:18-29): the photon set does not depend
on how it is cut. Across GPUs the cut is one range per rank. Each rank traces its range of ids into its own FP64
tallies and one ``all_reduce(SUM)`` over the process group adds every tally (arrivals, arrival x time, the second
moment, the time histograms, the Jacobian, health, counts and the readout groups' cells): weak scaling, with no other
exchange. Every rank returns the run's Light.

    import torch.distributed as dist
    dist.init_process_group("nccl")                    # one process per GPU
    light = lumen_b200.distributed.simulate_sharded(det, src, samples=2**26, seed=0)

``trace_shard`` and ``all_reduce_tallies`` are the two halves, for a caller timing them (bench.py).
"""

from __future__ import annotations

import numpy as np
import torch

from lumen_b200 import _abi as A
from lumen_b200.engine import DeviceRows, DeviceSource, DeviceTallies


def shard_range(total: int, rank: int, world: int) -> tuple[int, int]:
    """Return (first id, photons) of ``rank``'s contiguous share of photon ids 0 .. total - 1: the first
    ``total % world`` ranks take one photon more."""  # noqa: D205, D209
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside a world of {world}")
    base, extra = divmod(int(total), int(world))
    first = rank * base + min(rank, extra)
    return first, base + (1 if rank < extra else 0)


def _group_info(group):
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return 0, 1
    return dist.get_rank(group), dist.get_world_size(group)


def trace_shard(eng, key, first, n, *, source=None, rows=None, controls=None, tallies=None, stream=None):
    """Trace photon ids first .. first + n - 1 on this rank's engine into ``tallies`` (added to)."""
    if n > 0:
        eng.trace(key, n, source=source, rows=rows, first_id=first, controls=controls, tallies=tallies, stream=stream)
    return tallies


def tally_arrays(T) -> list:
    """The tallies' arrays every rank adds (torch tensors, in one fixed order; absent ones skipped)."""
    out = [T.arrival, T.arrival_t, T.arrival2, T.health, T.counts]
    out += [t for t in (T.hist, T.jac) if t is not None]
    G = getattr(T, "groups", None)
    if G is not None:  # the readout groups' FP64 cells (lumen_b200.readout.GroupCells) and pe2
        out += [t for t in G.outs if torch.is_tensor(t)]
    return out


def all_reduce_tallies(T, group=None) -> None:
    """Add every rank's tallies in place: one all_reduce(SUM) of one flat FP64 buffer (counts travel as float64,
    exact below 2^53) on the tallies' device (NCCL for CUDA tensors, gloo for CPU ones)."""  # noqa: D205, D209
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return
    arrs = tally_arrays(T)
    flat = torch.cat([a.reshape(-1).to(torch.float64) for a in arrs])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    off = 0
    for a in arrs:
        k = a.numel()
        a.copy_(flat[off:off + k].reshape(a.shape).to(a.dtype))
        off += k


def simulate_sharded(det, source, params=None, *, samples=None, seed=0, reference=None, controls=None,
                     gradients=(), time_bins=None, group=None, device=None, tracer=None):
    """Return the Light of ``samples`` photons of ``source`` with this rank's share of the photon ids traced here and
    the tallies added over ``group`` (``lumen_b200.simulate``'s arguments; the run's photons and results are those of
    one process tracing every id). ``tracer(first, n, key, controls, tallies)``: what traces a share (default: this
    rank's engine; a test passes the CPU checker)."""  # noqa: D205
    from lumen_b200 import api
    from lumen_b200.sources import FromArrays

    rank, world = _group_info(group)
    live = det.pool_with(params)
    ref = None if reference is None else det.pool_with({**(params or {}), **reference})
    det.check_values(live, "simulate_sharded")
    ctl = dict(roulette=0.01, max_distance=0.0, max_vertices=1 << 22, variant=None, jump=True) | (controls or {})
    gnames = list(gradients)
    gt = [det.params_index[k] for k in gnames]
    variant = ctl["variant"] if ctl["variant"] is not None else A.VARIANT_WAVEFRONT
    c = A.controls(ctl["max_distance"] or 0.0, ctl["roulette"], ctl["max_vertices"], gt, variant=variant,
                   flags=A.F_JUMP if ctl["jump"] else 0)  # fmt: skip
    nb, t0, tw = (0, 0.0, 1.0) if time_bins is None else time_bins
    n_ev = source.events()
    key = A.key_of_seed(seed)
    if isinstance(source, FromArrays):
        total = len(source.rows()["x"])
    else:
        if samples is None:
            raise ValueError("simulate_sharded: give samples")
        total = int(samples)
    first, n = shard_range(total, rank, world)
    if tracer is None:
        eng = api._engine(det, device)
        eng.set_pools(live, ref)
        T = DeviceTallies(det.n_sensor, n_ev, nb, t0, tw, len(gt), eng.device)
        if isinstance(source, FromArrays):  # the shard's own rows: row i of the call is photon first + i
            share = {k: (v[first:first + n] if v is not None and np.ndim(v) > 0 else v) for k, v in source.rows().items()}
            rows = DeviceRows(share, eng.device)
            trace_shard(eng, key, first, n, rows=rows, controls=c, tallies=T)
        else:
            ds = DeviceSource(source, total, eng.device, det)
            trace_shard(eng, key, first, n, source=ds, controls=c, tallies=T)
    else:
        T = tracer(first, n, key, c, DeviceTallies(det.n_sensor, n_ev, nb, t0, tw, len(gt), "cpu"))
    all_reduce_tallies(T, group)
    light = api._light(det, T, n_ev, total, seed, gnames, (nb, t0, tw), source)
    light.provenance.update(world=world, rank=rank, shard=(first, n))
    return light


__all__ = ["shard_range", "trace_shard", "all_reduce_tallies", "tally_arrays", "simulate_sharded"]
