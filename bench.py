"""Benchmark of the B200 calcium_sparks step: ensemble voxel-steps/s.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (per GPU): the batched ensemble of 256 independent spark realisations, each
100x100x50 voxels at 6 nm, with 16-100 RyRs, 0-50 % pRyR and compact / elongated /
fragmented clusters drawn from the seed, SERCA on the network-SR sheet, abort 1.5 ms
after all channels close (synth.config3).  Inputs are synthetic (the reference ships no
input for this configuration).  A step is one time step of every realisation.  With N
GPUs every rank advances its own 256 realisations (weak scaling, no collective on the
data path); rank 0 prints one JSON line.

value: voxel-steps/s over the K timed steps, device-timed with CUDA events on the
handle's stream (max over ranks).  e2e: the same metric through the C ABI with host
buffers: initial fields uploaded from host memory, K calls of csp_advance(1) each
returning the per-realisation stop flags, final fields downloaded.  The state (5.1 GB
per GPU) is larger than L2, so no flush is needed between steps.

--impl reference times the reference's CPU implementation of the step on the host cores
(the FP64 port of the reference in oracle/; one realisation per step sample).
"""
import argparse
import ctypes as C
import importlib
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_REAL = 256
SHAPE = (100, 100, 50)
BYTES_PER_VOXEL_STEP = 41     # 5 species x (4 B read + 4 B written) + 1 B domain id, FP32


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class Dist:
    """torch.distributed plumbing: barrier and max/sum over ranks (NCCL on GPUs)."""

    def __init__(self, world, local):
        self.world = world
        self.dist = None
        if world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
            self.dist = dist
            self.torch = torch
            self.dev = torch.device("cuda", local) if backend == "nccl" else torch.device("cpu")

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def reduce(self, x, op):
        if not self.dist:
            return x
        t = self.torch.tensor([float(x)], dtype=self.torch.float64, device=self.dev)
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX if op == "max" else self.dist.ReduceOp.SUM)
        return float(t.item())

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


class Clocks:
    """nvidia-smi samples of the SM clock and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        self.proc.wait()
        sm = [float(r[0]) for r in self.rows if len(r) >= 8 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 8 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) < 8:
                continue
            for n, v in zip(names, r[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def shard_workload(rank, world, nreal):
    """The realisations of one rank: its own seed range (weak scaling, nothing shared)."""
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    specs, opts = synth.config3(n=nreal, seed=3 + 1000 * rank)
    return specs, opts


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(nvox):
    """DRAM bytes per launch of the voxel kernel from the committed ncu summary, scaled
    from the captured case to this launch by voxel count (traffic grows in proportion)."""
    p = os.path.join(ROOT, "profiles", "k_voxels_staged_config3.md")
    if not os.path.exists(p):
        return None
    m = re.search(r"dram_bytes_per_voxel:\s*([0-9.]+)", open(p).read())
    return float(m.group(1)) * nvox if m else None


def cpu_port_rate(steps, spec, opts):
    """voxel-steps/s of the FP64 port of the reference (oracle/, one thread)."""
    from oracle.oracle import Oracle
    orc = Oracle(spec, opts)
    nvox = int(np.prod(spec["voxels"].shape))
    orc.step(2)
    t0 = time.perf_counter()
    orc.step(steps)
    dt = time.perf_counter() - t0
    return nvox * steps / dt, dt


def run_reference(args, rank, world):
    """--impl reference: the reference's step on the host cores, rank 0 only."""
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    if rank != 0:
        return 0
    specs, opts = synth.config3(n=1)
    steps = max(1, args.steps)
    rate, dt = cpu_port_rate(steps, specs[0], opts[0])
    unit = "voxel-steps/s"
    line = {"impl": "reference", "metric": "ensemble voxel-steps/s", "value": rate, "unit": unit,
            "n_gpus": world, "steps": steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "batched ensemble, realisation 100x100x50 voxels at 6 nm (config 3); "
                                   "CPU arm samples one realisation per step", "realisations": N_REAL,
                       "voxels_per_realisation": int(np.prod(SHAPE))},
            "cpu_baseline": {"value": rate, "unit": unit, "cores": 1, "kind": "port",
                             "sample": f"{steps} steps of one 100x100x50 realisation, FP64 port of the reference"},
            "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--realisations", type=int, default=N_REAL)
    ap.add_argument("--cpu-steps", type=int, default=200)
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    pkg = importlib.import_module("hpc-ca-phospattern_b200")
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    D = Dist(world, local)
    pkg.set_device(local)
    nreal = args.realisations
    specs, opts = shard_workload(rank, world, nreal)
    sim = pkg.Simulation(specs, opts)
    nvox = sum(int(np.prod(s["voxels"].shape)) for s in specs)
    W, K = max(3, args.warmup), args.steps

    # ---- device-timed steps (graph replay, CUDA events on the handle stream) ----
    sim.advance(W)
    D.barrier()
    clocks = Clocks(local)
    clocks.start()
    sim.advance(K)
    ms = sim.last_ms()
    clk = clocks.stop()
    D.barrier()
    ms_max = D.reduce(ms, "max")
    vox_total = D.reduce(nvox, "sum")
    value = vox_total * K / (ms_max / 1e3)

    # ---- roofline of the dominant kernel: per-launch CUDA events ----
    nprof = min(K, 100)
    vms, bms = sim.profile(nprof)
    t_launch = vms / nprof / 1e3
    achieved = BYTES_PER_VOXEL_STEP * nvox / t_launch / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic(nvox)

    # ---- e2e through the C ABI with host buffers ----
    sim2 = pkg.Simulation(specs, opts)
    host = [sim2.state(r) for r in range(nreal)]
    lib = sim2.lib
    flags = np.zeros(nreal, dtype=np.int32)
    fp = flags.ctypes.data_as(C.POINTER(C.c_int32))
    D.barrier()
    t0 = time.perf_counter()
    for r in range(nreal):
        sim2.set_state(host[r], r)
    for _ in range(K):
        rc = lib.csp_advance(sim2.h, 1, fp)
        if rc:
            raise RuntimeError(f"csp_advance failed: {rc}")
    out = [sim2.state(r) for r in range(nreal)]
    e2e_s = time.perf_counter() - t0
    e2e_s = D.reduce(e2e_s, "max")
    e2e = vox_total * K / e2e_s
    ns = len(specs[0]["species"])
    field_bytes = 4 * ns * nvox                     # FP32 fields copied per direction
    h2d = field_bytes / K
    d2h = (field_bytes + K * nreal * 48) / K        # final fields + per-step progress / stop flags
    assert all(np.isfinite(o).all() for o in out)

    # ---- CPU baseline (rank 0, N=1 only): FP64 port of the reference ----
    cpu = None
    if world == 1 and rank == 0 and args.cpu_steps > 0:
        rate, dt = cpu_port_rate(args.cpu_steps, specs[0], opts[0])
        cpu = {"value": rate, "unit": "voxel-steps/s", "cores": 1, "kind": "port",
               "sample": f"{args.cpu_steps} steps of one 100x100x50 realisation of the workload "
                         f"({dt:.1f} s), FP64 port of the reference"}

    # per step: voxel kernel, density-row flux kernel, channel-row gating/flux kernel, step
    # epilogue (the workload has both kinds of flux rows)
    kernels = 4 * K
    if rank == 0:
        line = {
            "metric": "ensemble voxel-steps/s", "value": value, "unit": "voxel-steps/s",
            "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": ms_max / K,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": f"batched ensemble (config 3): {nreal} realisations of 100x100x50 voxels at 6 nm "
                                   "per GPU, RyR/pRyR clusters + SERCA, FP32 fields",
                       "realisations_per_gpu": nreal, "voxels_per_gpu": nvox,
                       "l2": "state 5.1 GB per GPU > L2, no flush needed", "parallelism": f"ensemble x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_voxels_staged", "launch_ms": t_launch * 1e3,
                         "bytes_per_voxel": BYTES_PER_VOXEL_STEP, "peak_source": peak_kind,
                         "boundary_kernel_ms": bms / nprof},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "voxel-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
            "gpu_launches": kernels,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    sim.close()
    sim2.close()
    D.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
