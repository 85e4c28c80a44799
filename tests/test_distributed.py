"""The multi-GPU path's host logic on CPU: photons sharded by contiguous id ranges across ranks (weak scaling, no
data-path exchange), then one all-reduce (sum) of the FP64 tallies, as ``bench.py`` does over NCCL. Here two ``gloo``
ranks each trace their range with the checker and all-reduce; the result must equal one process tracing every id
(photon i is keyed by its global id, src/lumen/run.py:309), to the tallies' summation order."""

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

N = 1 << 12


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import datetime

    import torch
    import torch.distributed as dist

    import oracle
    from lumen_b200 import _abi as A
    from lumen_b200 import detectors, sources

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    det = detectors.cylinder_tank()
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    per = N // world
    T, _ = oracle.trace(det, A.key_of_seed(0), per, source=src, samples=N, first_id=rank * per, n_bins=50)
    tal = [torch.from_numpy(np.ascontiguousarray(x)) for x in (T.arrival, T.arrival_t, T.arrival2, T.hist, T.health)]
    for t in tal:
        dist.all_reduce(t)
    if rank == 0:
        out.put([t.numpy() for t in tal])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharding_equals_one_process():
    import oracle
    from lumen_b200 import _abi as A
    from lumen_b200 import detectors, sources

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    det = detectors.cylinder_tank()
    src = sources.Point(position=(1.0, -0.5, 2.0), n_photons=1.0, lam_range=(300.0, 600.0))
    T, _ = oracle.trace(det, A.key_of_seed(0), N, source=src, samples=N, n_bins=50)
    for a, b in zip(got, (T.arrival, T.arrival_t, T.arrival2, T.hist, T.health), strict=True):
        np.testing.assert_allclose(a, b, rtol=1e-9, atol=1e-15)
