"""The multi-GPU path's host logic on CPU (lumen_b200.distributed): photons sharded by contiguous id ranges across
ranks (weak scaling, no data-path exchange), then one all-reduce (sum) of every FP64 tally, as over NCCL on GPUs. Two
``gloo`` ranks run ``simulate_sharded`` with the checker as each rank's tracer (there is no GPU here); the Light they
return must be the one of one process tracing every id (photon i is keyed by its global id, src/lumen/run.py:309),
to the tallies' summation order: arrivals, their errors and mean times, the time histograms, the Jacobian, the
health and the counts."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from lumen_b200.distributed import shard_range

N = (1 << 12) + 3  # not a multiple of the world: the first ranks take one photon more
NAMES = ["media/Water/absorption", "surfaces/BlackSheet/R"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _checker_tracer(det, src, total):
    """A share traced by the checker into the (CPU) tallies simulate_sharded hands it."""
    import torch

    import oracle

    def trace(first, n, key, controls, T):
        O, _ = oracle.trace(det, key, n, source=src, samples=total, first_id=first, controls=controls,
                            n_events=T.arrival.shape[0], n_bins=T.hist.shape[-1] if T.hist is not None else 0,
                            bin_w=1.0)  # fmt: skip
        for name in ("arrival", "arrival_t", "arrival2", "hist", "jac", "health"):
            t = getattr(T, name)
            if t is not None:
                t.copy_(torch.from_numpy(np.ascontiguousarray(getattr(O, name))))
        T.counts.copy_(torch.from_numpy(O.counts.astype(np.int64)))
        return T

    return trace


def _run(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch.distributed as dist

    from lumen_b200 import detectors, distributed, sources

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    det = detectors.cylinder_tank()
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    light = distributed.simulate_sharded(det, src, samples=N, seed=0, gradients=NAMES, time_bins=(50, 0.0, 1.0),
                                         tracer=_checker_tracer(det, src, N))  # fmt: skip
    out.put((rank, light.arrivals, light.arrivals_error, light.mean_arrival_time, light.diagnostics["time"],
             np.stack([light.gradients[k] for k in NAMES], 1), light.health.photons, light.health.steps,
             light.health.absorbed_surface, light.provenance["shard"]))  # fmt: skip
    dist.barrier()
    dist.destroy_process_group()


def test_shard_ranges_partition_the_ids():
    for total in (0, 1, 7, 4099):
        for world in (1, 2, 3, 8):
            got = [shard_range(total, r, world) for r in range(world)]
            assert sum(n for _, n in got) == total
            assert all(got[r][0] + got[r][1] == got[r + 1][0] for r in range(world - 1))
            assert max(n for _, n in got) - min(n for _, n in got) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def test_two_rank_sharding_equals_one_process():
    import oracle
    from lumen_b200 import _abi as A
    from lumen_b200 import api, detectors, sources

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_run, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict((r[0], r[1:]) for r in (q.get(timeout=180), q.get(timeout=180)))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert got[0][-1] == (0, N // 2 + 1) and got[1][-1] == (N // 2 + 1, N // 2)
    det = detectors.cylinder_tank()
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    c = A.controls(grad_tabs=[det.params_index[k] for k in NAMES], flags=A.F_JUMP)
    T, _ = oracle.trace(det, A.key_of_seed(0), N, source=src, samples=N, controls=c, n_bins=50, bin_w=1.0)
    err = api.moment_error(T.arrival2[0], T.arrival[0], N)
    want = (T.arrival[0], err, T.arrival_t[0] / np.where(T.arrival[0] > 0, T.arrival[0], 1.0), T.hist[0], T.jac[0])
    for rank in (0, 1):  # every rank returns the run's Light
        arr, e, mt, hist, jac, photons, steps, a_surf, _ = got[rank]
        np.testing.assert_allclose(arr, want[0], rtol=1e-9, atol=1e-15)
        np.testing.assert_allclose(e, want[1], rtol=1e-7, atol=1e-12)
        ok = want[0] > 0
        np.testing.assert_allclose(mt[ok], want[2][ok], rtol=1e-9)
        np.testing.assert_allclose(hist, want[3], rtol=1e-9, atol=1e-15)
        np.testing.assert_allclose(jac, want[4], rtol=1e-9, atol=1e-15)
        assert photons == N and steps == int(T.counts[A.C_STEPS])
        assert a_surf == pytest.approx(T.health[5], rel=1e-9)
