"""Ensembles across GPUs: realisations sharded over ranks by estimated cost, one gather of
their output statistics.

The realisations of a batched ensemble are independent, so a multi-GPU ensemble needs no
exchange on the data path.  With one process per GPU (torch.distributed: NCCL between
GPUs, gloo on CPU), every rank builds and advances only its own share, through one handle
of libcsparks_cuda.so on its own GPU; the only collectives are the barrier, scalar
reductions and one all_gather of the per-realisation statistics.  That gather takes the
place of the reference's gather of the per-rank output scalars to rank 0
(fvm_mpi/src/species.c:2866-2912, MPI_Gather of min / max / total per domain and
species); here each row is one whole realisation.

Assignment (assign): realisations in order of decreasing estimated cost (voxels x time
steps; ties by index) are dealt out one at a time, each to the rank with the least
assigned cost so far (ties to the lower rank): the round-robin by cost of the uneven
ensemble, which for equal costs is plain round-robin.

Every realisation draws its channel gating from the Philox stream of its index in the
whole ensemble (csp_options.stream_offset), so a realisation's trajectory does not
depend on how many GPUs share the ensemble.
"""
import math

import numpy as np

MAX_DOMAINS = 5
MAX_SPECIES = 8
# one statistics row: index, steps taken, stopped, open channels, then min / max / total
# [MAX_DOMAINS][MAX_SPECIES] (NaN where a realisation has fewer domains or species)
ROW = 4 + 3 * MAX_DOMAINS * MAX_SPECIES


def sigma_max(spec):
    return max(max(ds["sigma"]) for ds in spec["domain_species"].values() if ds["sigma"])


def step_count(h, opts, sig_max):
    """Time steps of `for (t = 0; t < tstop; t += dt)` (calcium_sparks.c:190) for the
    options' dt, or the automatic dt = 0.95 h^2 / (6 sigma_max) (species.c:265)."""
    dt = opts.get("dt", -1.0)
    if not dt or dt <= 0:
        dt = 0.95 * h * h / (6.0 * sig_max)
    return max(0, int(math.ceil(opts.get("tstop", 10.0) / dt - 1e-9)))


def realisation_cost(shape, h_geom, opts, sig_max):
    """Estimated work of one realisation: species voxels x time steps."""
    h = opts.get("h", 6.0)
    sub = max(1, int(math.floor(h_geom / h + 1e-9)))
    nvox = int(np.prod(shape)) * sub ** 3
    return nvox * step_count(h, opts, sig_max)


def spec_cost(spec, opts):
    return realisation_cost(spec["voxels"].shape, spec["h"], opts, sigma_max(spec))


def assign(costs, world):
    """Indices of the realisations of every rank (each list ascending)."""
    load = [0.0] * world
    share = [[] for _ in range(world)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        k = min(range(world), key=lambda w: (load[w], w))
        share[k].append(i)
        load[k] += costs[i]
    return [sorted(s) for s in share]


class Ranks:
    """torch.distributed plumbing for one process per GPU (NCCL on GPUs, gloo on CPU)."""

    def __init__(self, world=None, local=None, timeout_s=300):
        import os
        self.world = int(os.environ.get("WORLD_SIZE", "1")) if world is None else world
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", str(self.rank))) if local is None else local
        self.dist = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            if not dist.is_initialized():
                backend = "nccl" if torch.cuda.is_available() else "gloo"
                if backend == "nccl":
                    torch.cuda.set_device(self.local)
                dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist
            self.torch = torch
            self.rank = dist.get_rank()
            self.dev = (torch.device("cuda", self.local) if dist.get_backend() == "nccl" else torch.device("cpu"))

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def reduce(self, x, op):
        """x reduced over the ranks ("max" or "sum"), on every rank."""
        if not self.dist:
            return x
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return float(t.item())

    def all_gather_rows(self, rows):
        """Concatenation over the ranks of every rank's rows (float64 [m][ROW]), in rank order."""
        if not self.dist:
            return rows
        m = int(self.reduce(rows.shape[0], "max"))
        pad = np.full((m, rows.shape[1]), np.nan)
        pad[:rows.shape[0]] = rows
        pad[rows.shape[0]:, 0] = -1.0                  # padding rows carry index -1
        t = self.torch.tensor(pad, dtype=self.torch.float64, device=self.dev)
        out = [self.torch.empty_like(t) for _ in range(self.world)]
        self.dist.all_gather(out, t)
        allr = np.concatenate([o.cpu().numpy() for o in out])
        return allr[allr[:, 0] >= 0]

    def close(self):
        if self.dist and self.dist.is_initialized():
            self.dist.destroy_process_group()


class Ensemble:
    """n independent realisations over the ranks of the process group.

    build(indices) -> (specs, options) of the given global indices: every rank builds only
    its own share.  costs: estimated work per realisation (default: spec_cost of every
    built model, which builds every realisation on every rank).  simulation(specs,
    options): the handle of a rank's share (default: the package's Simulation on this
    rank's GPU).
    """

    def __init__(self, n, build, costs=None, ranks=None, simulation=None):
        self.ranks = ranks or Ranks()
        self.n = n
        if costs is None:
            specs, opts = build(list(range(n)))
            costs = [spec_cost(s, o) for s, o in zip(specs, opts)]
        self.costs = list(costs)
        self.shares = assign(self.costs, self.ranks.world)
        self.mine = self.shares[self.ranks.rank]
        self.sim = None
        self.specs, self.opts = [], []
        if self.mine:
            specs, opts = build(self.mine)
            # channel draws from the stream of the global index (batch index + offset)
            self.specs = specs
            self.opts = [dict(o, stream_offset=g - j) for j, (g, o) in enumerate(zip(self.mine, opts))]
            if simulation is None:
                import importlib
                pkg = importlib.import_module(__package__)
                pkg.set_device(self.ranks.local)
                simulation = pkg.Simulation
            self.sim = simulation(self.specs, self.opts)

    def local_cost(self):
        return sum(self.costs[i] for i in self.mine)

    def advance(self, nsteps):
        """Advance this rank's realisations; returns their stop flags (local order)."""
        return self.sim.advance(nsteps) if self.sim else np.zeros(0, dtype=np.int32)

    def all_stopped(self):
        """True on every rank once every realisation of every rank has stopped."""
        mine = 1.0
        if self.sim:
            mine = float(all(self.sim.info(j).stopped for j in range(len(self.mine))))
        return self.ranks.reduce(-mine, "max") == -1.0

    def local_rows(self):
        rows = np.full((len(self.mine), ROW), np.nan)
        for j, g in enumerate(self.mine):
            inf = self.sim.info(j)
            mn, mx, tot, op = self.sim.outputs(j)
            nd, ns = mn.shape
            rows[j, :4] = (g, inf.step, inf.stopped, int(np.sum(op)))
            for k, a in enumerate((mn, mx, tot)):
                blk = np.full((MAX_DOMAINS, MAX_SPECIES), np.nan)
                blk[:nd, :ns] = a
                rows[j, 4 + k * MAX_DOMAINS * MAX_SPECIES: 4 + (k + 1) * MAX_DOMAINS * MAX_SPECIES] = blk.ravel()
        return rows

    def statistics(self):
        """Every realisation's statistics on every rank (one all_gather), by global index:
        dict(index, step, stopped, open [n]; min, max, total [n][MAX_DOMAINS][MAX_SPECIES])."""
        rows = self.ranks.all_gather_rows(self.local_rows())
        rows = rows[np.argsort(rows[:, 0], kind="stable")]
        b = MAX_DOMAINS * MAX_SPECIES
        return {"index": rows[:, 0].astype(np.int64), "step": rows[:, 1].astype(np.int64),
                "stopped": rows[:, 2].astype(np.int32), "open": rows[:, 3].astype(np.int64),
                "min": rows[:, 4:4 + b].reshape(-1, MAX_DOMAINS, MAX_SPECIES),
                "max": rows[:, 4 + b:4 + 2 * b].reshape(-1, MAX_DOMAINS, MAX_SPECIES),
                "total": rows[:, 4 + 2 * b:4 + 3 * b].reshape(-1, MAX_DOMAINS, MAX_SPECIES)}

    def close(self):
        if self.sim:
            self.sim.close()
            self.sim = None
