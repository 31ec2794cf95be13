"""Host logic of the N > 1 paths on CPU: two gloo ranks (spawned processes)
run the ensemble sharding of bench.py and the max-over-ranks timing
reduction, with no GPU."""
import datetime
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys

    import torch
    import torch.distributed as dist

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    from resistivemhd_gpu_b200 import setups

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        rng_sizes = setups.ENSEMBLE_SIZES

        class Run:                       # what _shard reads of a Setup
            def __init__(self, n):
                self.interior_cells = n * n

        import numpy as np

        sizes = np.random.default_rng(4).choice(rng_sizes, size=40)
        runs = [Run(int(n)) for n in sizes]
        parts = bench._shard(runs, world)
        mine = parts[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        # the elapsed times reduce to the slowest rank's
        t = torch.tensor([10.0 * (rank + 1)], dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        loads = [sum(runs[r].interior_cells for r in p) for p in parts]
        out.put((rank, parts, gathered, float(t.item()), loads, max(r.interior_cells for r in runs)))
    finally:
        dist.destroy_process_group()


def test_ensemble_sharding_and_timing_reduction_on_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    parts0 = results[0][1]
    for rank, parts, gathered, tmax, loads, biggest in results:
        assert parts == parts0                       # every rank computes the same assignment
        assert gathered == parts0                    # and takes its own part of it
        assert tmax == 10.0 * world                  # the slowest rank's time
        assert max(loads) - min(loads) <= biggest    # largest-first greedy balance
    flat = sorted(r for p in parts0 for r in p)
    assert flat == list(range(40))                   # disjoint and complete
