"""Multi-rank host logic of the ensemble benchmark, world size 2 over gloo on CPU.

Realisations shard across ranks with no exchange on the data path: each rank builds its
own realisations (disjoint seeds), the only collectives are the barrier and the
max / sum reductions of the timing and voxel counts, and one gather of the
per-realisation summaries after the timed region.
"""
import os
import socket

import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import numpy as np
    import bench
    d = bench.Dist(world, rank)
    specs, opts = bench.shard_workload(rank, world, 4)
    nvox = sum(int(np.prod(s["voxels"].shape)) for s in specs)
    seeds = [o["seed"] for o in opts]
    d.barrier()
    total = d.reduce(nvox, "sum")
    slowest = d.reduce(1.0 + rank, "max")

    class FakeSim:                      # per-realisation progress, as csp_get_info reports it
        def info(self, r):
            return type("I", (), {"step": 10 * rank + r, "stopped": r % 2})()

    gathered = d.gather_summaries(FakeSim(), 4)
    q.put((rank, seeds, nvox, total, slowest, gathered))
    d.close()


def test_two_ranks_shard_realisations_without_exchange():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, n0, t0, m0, g0), (r1, s1, n1, t1, m1, g1) = res
    assert g0 == g1 == 8, "every rank's realisation summaries reach every rank"

    assert set(s0).isdisjoint(s1), "ranks must draw different realisations"
    assert t0 == t1 == n0 + n1
    assert m0 == m1 == 2.0
