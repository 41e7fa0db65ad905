"""Multi-rank host logic of the ensemble, world size 2 over gloo on CPU.

Realisations shard across ranks with no exchange on the data path: the benchmark's whole
job is one ensemble whose realisations the ranks split by estimated cost, each rank
building only its own share; the only collectives are the barrier, the max / sum
reductions of the timing and voxel counts, and one all_gather of the per-realisation
statistics after the timed region.
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


class _ConstSim:
    """Stands in for a GPU handle (no GPU in this process)."""

    def __init__(self, specs, opts):
        self.n = len(specs)
        self.opts = opts

    def info(self, j):
        return type("I", (), {"step": 10 + j, "stopped": j % 2})()

    def outputs(self, j):
        import numpy as np
        z = np.zeros((5, 5))
        return z, z, z, np.zeros(1, dtype=np.int32)

    def close(self):
        pass


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import importlib
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import numpy as np
    import bench
    ens_mod = importlib.import_module("hpc-ca-phospattern_b200.ensemble")
    d = ens_mod.Ranks(world, rank)
    ens = bench.ensemble_workload(d, 4, simulation=_ConstSim)
    nvox = sum(int(np.prod(s["voxels"].shape)) for s in ens.specs)
    seeds = [o["seed"] for o in ens.opts]
    d.barrier()
    total = d.reduce(nvox, "sum")
    slowest = d.reduce(1.0 + rank, "max")
    gathered = len(ens.statistics()["index"])
    q.put((rank, ens.mine, seeds, nvox, total, slowest, gathered))
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
    (r0, i0, s0, n0, t0, m0, g0), (r1, i1, s1, n1, t1, m1, g1) = res
    assert i0 == [0, 2, 4, 6] and i1 == [1, 3, 5, 7], "equal costs: round-robin over the whole job"
    assert g0 == g1 == 8, "every rank's realisation statistics reach every rank"
    assert set(s0).isdisjoint(s1), "ranks must draw different realisations"
    assert t0 == t1 == n0 + n1
    assert m0 == m1 == 2.0


def _ensemble_worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import importlib
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import numpy as np
    ens_mod = importlib.import_module("hpc-ca-phospattern_b200.ensemble")
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    draws = synth.config4_draws(64)
    costs = [ens_mod.realisation_cost(d["shape"], d["h"], d["opts"], 220000.0) for d in draws]

    class FakeSim:
        """Stands in for a GPU handle: outputs are a known function of the global index."""

        def __init__(self, specs, opts):
            self.globals = [s["index"] for s in specs]
            self.offsets = [o["stream_offset"] for o in opts]
            self.steps = 0

        def advance(self, k):
            self.steps += k
            return np.array([int(g % 3 == 0) for g in self.globals], dtype=np.int32)

        def info(self, j):
            g = self.globals[j]
            return type("I", (), {"step": self.steps + g, "stopped": int(g % 3 == 0)})()

        def outputs(self, j):
            g = self.globals[j]
            base = np.arange(25, dtype=np.float64).reshape(5, 5)
            return base + g, base * 2 + g, base * 3 + g, np.array([g % 2, 1], dtype=np.int32)

        def close(self):
            pass

    def build(idx):
        return [dict(index=i) for i in idx], [dict(draws[i]["opts"]) for i in idx]

    ranks = ens_mod.Ranks()
    ens = ens_mod.Ensemble(64, build, costs=costs, ranks=ranks, simulation=FakeSim)
    ens.advance(7)
    stats = ens.statistics()
    stopped = ens.all_stopped()
    q.put((rank, ens.mine, ens.local_cost(), ens.sim.offsets, stats, stopped, costs))
    ranks.close()


def test_ensemble_cost_balanced_shards_and_statistics_gather():
    """hpc-ca-phospattern_b200.ensemble on the 64 uneven grids of config 4 (costs =
    voxels x steps from the draws): the two shares are disjoint and cover every
    realisation, their costs are balanced to within the largest single realisation, every
    realisation draws from the Philox stream of its global index, and one all_gather
    gives every rank every realisation's statistics in index order."""
    import numpy as np
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_ensemble_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((q.get(timeout=180) for _ in procs), key=lambda x: x[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (_, m0, c0, off0, st0, stop0, costs), (_, m1, c1, off1, st1, stop1, _) = res
    assert sorted(m0 + m1) == list(range(64)) and not set(m0) & set(m1)
    assert abs(c0 - c1) <= max(costs), (c0, c1, max(costs))
    assert c0 + c1 == sum(costs)
    assert off0 == [g - j for j, g in enumerate(m0)] and off1 == [g - j for j, g in enumerate(m1)]
    for st in (st0, st1):
        assert list(st["index"]) == list(range(64))
        assert list(st["stopped"]) == [int(g % 3 == 0) for g in range(64)]
        assert list(st["step"]) == [7 + g for g in range(64)]
        assert list(st["open"]) == [g % 2 + 1 for g in range(64)]
        base = np.arange(25, dtype=np.float64).reshape(5, 5)
        for g in (0, 17, 63):
            np.testing.assert_array_equal(st["min"][g][:5, :5], base + g)
            np.testing.assert_array_equal(st["total"][g][:5, :5], base * 3 + g)
            assert np.isnan(st["max"][g][:, 5:]).all()
    assert stop0 is False and stop1 is False
