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
buffers, one csp_run_states call: every realisation's FP32 state uploaded from
page-locked host memory, K steps with every realisation's stop flag after every step read
back, the final fields downloaded, pipelined by realisation groups (the copies of one
group overlap the steps of another).  The state (5.1 GB per GPU) is larger than L2, so no
flush is needed between steps.  parity: the FP32 error against the reference program's
FP64 run on config 2 (tests/golden/configs/config2_short.npz).

cpu_baseline and --impl reference time the reference program itself (oracle/_ref: the
reference's fvm_mpi sources built with a single-rank MPI stub and the project's HDF5
subset, FP64, OpenMP on every physical core) on one realisation of the workload, from its
own main-loop timer; the FP64 port in oracle/ stands in only when oracle/_ref is absent.
"""
import argparse
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


def ensemble_workload(ranks, nreal_per_gpu, simulation=None):
    """The whole job: nreal_per_gpu x world realisations of config 3 (seed 3), assigned to
    the ranks by estimated cost (voxels x steps: equal here, so round-robin) with
    hpc-ca-phospattern_b200.ensemble; every rank builds and advances only its own share
    (weak scaling, nothing exchanged on the data path)."""
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    ens = importlib.import_module("hpc-ca-phospattern_b200.ensemble")
    n = nreal_per_gpu * ranks.world
    draws = synth.config3_draws(n=n, seed=3)
    costs = [ens.realisation_cost(d["shape"], d["h"], d["opts"], 220000.0) for d in draws]
    return ens.Ensemble(n, lambda idx: synth.config3(n=n, seed=3, only=idx), costs=costs, ranks=ranks,
                        simulation=simulation)


def pinned_copy(a):
    """A copy of a numpy array in page-locked host memory (torch's pinned allocator), so
    that the state copies of the e2e leg run at full PCIe speed; a plain copy without torch."""
    try:
        import torch
        tdt = {np.dtype(np.float64): torch.float64, np.dtype(np.float32): torch.float32}[a.dtype]
        t = torch.empty(a.shape, dtype=tdt, pin_memory=torch.cuda.is_available())
        out = t.numpy()
        out[...] = a
        _PINNED.append(t)          # keeps the pinned block alive with the array
        return out
    except ImportError:
        return a.copy()


_PINNED = []


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


def host_cores():
    """Physical cores of this host (the reference's OpenMP threads)."""
    try:
        import psutil
        n = psutil.cpu_count(logical=False)
        if n:
            return int(n)
    except ImportError:
        pass
    return os.cpu_count() or 1


def reference_binary():
    from oracle import refrun
    return refrun.ref_binary()


def reference_run(spec, opts, nsteps, threads, workdir):
    """One run of the reference program (oracle/_ref) for nsteps time steps; returns
    (time steps taken, seconds of its MAINLOOP timer, calcium_sparks.c:188-229)."""
    from oracle import refrun
    h = float(opts.get("h", spec["h"]))
    dt = 0.95 * h * h / (6 * 220000.0)           # the workload's automatic dt (sigma_max = 220000 nm^2/ms)
    o = dict(opts)
    o["tstop"] = nsteps * dt
    o["dt_save"] = o["tstop"]
    res = refrun.run(spec, o, workdir, threads=threads, verbose=True)
    steps = max(out["time_index"] for out in res["outputs"])
    if not res["mainloop_s"]:
        raise RuntimeError("reference printed no MAINLOOP time")
    return steps, res["mainloop_s"]


def reference_rate(spec, opts, target_s, threads, workdir, steps_hint=None):
    """voxel-steps/s of the reference program on `threads` host cores, on a sample of
    about target_s seconds of its main loop (sized by a short calibration run)."""
    nvox = int(np.prod(spec["voxels"].shape))
    s0, t0 = reference_run(spec, opts, 300, threads, workdir)
    est = nvox * s0 / max(t0, 0.05)
    nsteps = steps_hint or max(300, int(target_s * est / nvox))
    steps, secs = reference_run(spec, opts, nsteps, threads, workdir)
    return nvox * steps / secs, steps, secs


def run_reference(args, rank, world):
    """--impl reference: the reference program's step on the host cores (rank 0 only).

    oracle/_ref is the reference's own FP64 OpenMP build (fvm_mpi sources, single-rank
    MPI stub, HDF5 subset), run on one realisation of the workload with every physical
    core; one "step" of this arm is m time steps of that realisation, m sized so the K
    timed steps take about 30 s of the reference's main loop."""
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    if rank != 0:
        return 0
    specs, opts = synth.config3(n=1)
    K = max(1, args.steps)
    unit = "voxel-steps/s"
    nvox = int(np.prod(SHAPE))
    config = {"workload": "batched ensemble (config 3): realisations of 100x100x50 voxels at 6 nm, RyR/pRyR "
                          "clusters + SERCA; the CPU arm runs one realisation at a time",
              "realisations_per_gpu": N_REAL, "voxels_per_realisation": nvox, "parallelism": "OpenMP"}
    if reference_binary():
        import tempfile
        cores = host_cores()
        wd = tempfile.mkdtemp(prefix="csp_ref_")
        s0, t0 = reference_run(specs[0], opts[0], 300, cores, wd)          # warm-up + calibration
        est = nvox * s0 / max(t0, 0.05)
        m = max(1, int(30.0 * est / (nvox * K)))
        steps, secs = reference_run(specs[0], opts[0], m * K, cores, wd)
        rate = nvox * steps / secs
        kind = "reference"
        sample = (f"{steps} time steps ({K} samples of {m}) of one 100x100x50 realisation of the workload, "
                  f"{secs:.1f} s of the reference's main loop (oracle/_ref: its own FP64 OpenMP build), "
                  f"{cores} threads")
        ms_per_step = 1e3 * secs / K
    else:
        cores = 1
        rate, dt = cpu_port_rate(K, specs[0], opts[0])
        kind = "port"
        sample = f"{K} steps of one 100x100x50 realisation, FP64 port of the reference (oracle/_ref not built)"
        ms_per_step = 1e3 * dt / K
    line = {"impl": "reference", "metric": "ensemble voxel-steps/s", "value": rate, "unit": unit,
            "n_gpus": world, "steps": K, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": config,
            "cpu_baseline": {"value": rate, "unit": unit, "cores": cores, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def surrogate_run(pkg, specs, opts, W, K, tc=1):
    """The workload with dt_update_react = 10 dt, with and without the learned reaction
    surrogate.  Training pairs are harvested from a run of the workload itself (32 of its
    realisations stepped 0.2 ms, about 1e6 pairs taken every 0.02 ms, log-uniform in Ca as
    far as the states allow), the network trained on them on device; then both ensembles
    are timed like the main run, and both are compared on 8 realisations over 400 steps
    with the run that reacts every step (max relative error per species).  tc: the network
    tiles on warp mma.sync (1) or tcgen05 (2)."""
    dt = 0.95 * 36 / (6 * 220000.0)
    o10 = [dict(o, dt_update_react=10 * dt) for o in opts]
    harv = pkg.Simulation(specs[:32], o10[:32])
    held = 0
    t0 = time.perf_counter()
    for k in range(10):
        harv.advance(772)
        _, held = harv.mlp_harvest(1_000_000, seed=100 + k, capacity=10_500_000)
    params, rep = harv.mlp_train(samples=0, val_samples=65536, epochs=8, batch=8192, lr=2e-3, seed=5, harvested=True)
    harvest_train_s = time.perf_counter() - t0
    harv.close()
    nvox = sum(int(np.prod(s["voxels"].shape)) for s in specs)
    out = {}
    for name, use in (("surrogate", True), ("plain_T10", False)):
        sim = pkg.Simulation(specs, o10)
        if use:
            sim.set_surrogate(params, 1e-4)
            sim.set_surrogate_tensor_cores(tc)
        sim.advance(W)
        sim.advance(K)
        out[name] = nvox * K / (sim.last_ms() / 1e3)
        if use:
            vx, ev, fb = sim.surrogate_counts()
        sim.close()
    # accuracy against reacting every step
    n8, steps = 8, 400
    fine = pkg.Simulation(specs[:n8], opts[:n8])
    fine.advance(steps)
    uf = [fine.state(r) for r in range(n8)]
    fine.close()
    errs = {}
    for name, use in (("surrogate", True), ("plain_T10", False)):
        sim = pkg.Simulation(specs[:n8], o10[:n8])
        if use:
            sim.set_surrogate(params, 1e-4)
            sim.set_surrogate_tensor_cores(tc)
        sim.advance(steps)
        e = np.zeros(len(specs[0]["species"]))
        for r in range(n8):
            u = sim.state(r)
            scale = np.max(np.abs(uf[r]), axis=(1, 2, 3))
            e = np.maximum(e, np.max(np.abs(u - uf[r]), axis=(1, 2, 3)) / scale)
        errs[name] = e
        sim.close()
    return {"value": out["surrogate"], "unit": "voxel-steps/s", "dt_update_react": "10 dt",
            "network_tiles": "tcgen05" if tc == 2 else "mma.sync",
            "without_network": {"value": out["plain_T10"], "unit": "voxel-steps/s",
                                "max_rel_err_vs_every_step": float(errs["plain_T10"].max()),
                                "per_species": [float(v) for v in errs["plain_T10"]]},
            "max_rel_err_vs_every_step": float(errs["surrogate"].max()),
            "per_species": [float(v) for v in errs["surrogate"]],
            "accuracy_check": f"{n8} realisations x {steps} steps against the same run reacting every step",
            "training": {"pairs": held, "source": "harvested from the workload (32 realisations, 0.2 ms)",
                         "harvest_and_train_s": harvest_train_s, "train_ms": rep["train_ms"],
                         "val_accept_rate": rep["val_accept_rate"]},
            "voxel_increments": vx, "network_fraction": ev / vx if vx else None,
            "fallback_fraction": fb / vx if vx else None}


def parity_leg(pkg):
    """FP32 accuracy on one 200x200x100 grid (config 2: 10x10 RyR lattice with vacancies,
    20 % pRyR), 0.5 ms = 19,296 steps with channels forced, against the reference
    program's FP64 run stored in tests/golden/configs/config2_short.npz: max over the stored
    voxels (a lattice of every 5th voxel and the cleft planes around the cluster) of
    |diff| / max |ref| per species."""
    golden = os.path.join(ROOT, "tests", "golden")
    path = os.path.join(golden, "configs", "config2_short.npz")
    if not os.path.exists(path):
        return None
    sys.path.insert(0, golden)
    mcp = importlib.import_module("make_config_parity")
    z = np.load(path)
    spec, opts = mcp.build("config2_short")
    sim = pkg.Simulation(spec, opts)
    steps = int(z["time_index"][-1])
    sim.advance(steps)
    lat, win = mcp.samples(sim.state(), spec)
    sim.close()
    err = []
    for s in range(lat.shape[0]):
        e = 0.0
        for got, ref in ((lat[s], z["lattice"][s].astype(np.float64)), (win[s], z["window"][s].astype(np.float64))):
            e = max(e, float(np.max(np.abs(got - ref)) / np.max(np.abs(ref))))
        err.append(e)
    return {"workload": "config 2: one 200x200x100 grid, 0.5 ms, channels forced (-O/-C)", "steps": steps,
            "against": "reference program FP64 (oracle/_ref), stored fixture", "max_rel_err": max(err),
            "per_species": dict(zip(spec["species"], err)), "bar": 1e-4}


def config_leg(pkg, specs, opts, W, K, workload):
    """One more configuration on the same kernels: autotuned tile, W untimed steps, K steps
    timed on the device (graph replay); voxel-steps summed over the realisations."""
    sim = pkg.Simulation(specs, opts)
    tune = sim.autotune(repeats=3)
    sim.advance(W)
    sim.advance(K)
    ms = sim.last_ms()
    nvox = sum(int(np.prod(s["voxels"].shape)) for s in specs)
    tv, tb = sim.profile(8)
    sim.close()
    ch = tune["chosen"]
    return {"value": nvox * K / (ms / 1e3), "unit": "voxel-steps/s", "ms_per_step": ms / K,
            "voxel_kernel_ms": tv / 8, "boundary_ms": tb / 8, "voxels": nvox, "realisations": len(specs),
            "tile": {"threads": ch["threads"], "x_planes_per_unit": ch["segment"]}, "workload": workload}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--realisations", type=int, default=N_REAL)
    ap.add_argument("--extras", type=int, default=1,
                    help="also time the plain single-realisation path and the surrogate run (0: skip)")
    ap.add_argument("--surrogate-tc", type=int, default=1, choices=[1, 2],
                    help="network tiles of the surrogate run: warp mma.sync (1) or tcgen05 (2)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="length of the CPU baseline sample (0: skip)")
    args = ap.parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        return run_reference(args, rank, world)

    pkg = importlib.import_module("hpc-ca-phospattern_b200")
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    ensemble = importlib.import_module("hpc-ca-phospattern_b200.ensemble")
    D = ensemble.Ranks(world, local)
    pkg.set_device(local)
    ens = ensemble_workload(D, args.realisations)
    sim, specs, opts = ens.sim, ens.specs, ens.opts
    nreal = len(specs)
    nvox = sum(int(np.prod(s["voxels"].shape)) for s in specs)
    W, K = max(3, args.warmup), args.steps

    # ---- tile shape of the staged voxel kernel: the autotuner's pick ----
    tune = sim.autotune(repeats=3)

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
    # per-realisation statistics (steps, stop flag, open channels, per-domain min / max /
    # total of every species) of every rank on every rank: one all_gather
    gathered = int(len(ens.statistics()["index"]))

    # ---- roofline of the dominant kernel: per-launch CUDA events ----
    nprof = min(K, 100)
    vms, bms = sim.profile(nprof)
    t_launch = vms / nprof / 1e3
    achieved = BYTES_PER_VOXEL_STEP * nvox / t_launch / 1e9
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic(nvox)

    # ---- e2e through the C ABI with host buffers: csp_run_states (upload every
    # realisation's FP32 state from page-locked host memory, K steps with every
    # realisation's stop flag read back after every step, download), pipelined by
    # realisation groups so the copies overlap the steps ----
    sim2 = pkg.Simulation(specs, opts)
    host = [pinned_copy(sim2.state(r).astype(np.float32)) for r in range(nreal)]
    outb = [pinned_copy(np.zeros_like(h)) for h in host]
    sim2.run_states(host, W, outb)                  # warm-up: the same call, untimed
    D.barrier()
    t0 = time.perf_counter()
    flags, step_flags = sim2.run_states(host, K, outb, step_flags=True)
    e2e_s = time.perf_counter() - t0
    e2e_s = D.reduce(e2e_s, "max")
    e2e = vox_total * K / e2e_s
    ns = len(specs[0]["species"])
    field_bytes = 4 * ns * nvox                     # FP32 host state copied per direction
    h2d = field_bytes / K
    d2h = (field_bytes + K * nreal * 4) / K         # final fields + every step's stop flags
    assert all(np.isfinite(o).all() for o in outb) and step_flags.shape == (K, nreal)

    # ---- plain path: one realisation of the same workload on the same kernels ----
    plain_single, sur, configs, parity = None, None, None, None
    if args.extras:
        single = pkg.Simulation(specs[:1], opts[:1])
        single.advance(W)
        single.advance(K)
        plain_single = int(np.prod(specs[0]["voxels"].shape)) * K / (single.last_ms() / 1e3)
        single.close()
        # ---- learned reaction surrogate (dt_update_react = 10 dt): train, deploy, time ----
        sur = surrogate_run(pkg, specs, opts, W, K, args.surrogate_tc)
        # ---- configs 2 and 4 on the same kernels ----
        s2, o2 = synth.config2()
        s4, o4 = synth.config4()
        parity = parity_leg(pkg)
        configs = {
            "config2": config_leg(pkg, [s2], [o2], W, K,
                                  "one 200x200x100 grid at 6 nm, 10x10 RyR lattice with vacancies, 20 % pRyR"),
            "config4": config_leg(pkg, s4, o4, W, K,
                                  "64 grids from 64^3 to 256x256x128 at h = 6-10 nm (dt per realisation), "
                                  "dt_update_react = 5 dt"),
        }

    # ---- CPU baseline (rank 0, N=1 only): FP64 port of the reference ----
    cpu = None
    if world == 1 and rank == 0 and args.cpu_seconds > 0:
        if reference_binary():
            import tempfile
            cores = host_cores()
            rate, steps, secs = reference_rate(specs[0], opts[0], args.cpu_seconds, cores,
                                               tempfile.mkdtemp(prefix="csp_ref_"))
            cpu = {"value": rate, "unit": "voxel-steps/s", "cores": cores, "kind": "reference",
                   "sample": f"{steps} time steps of one 100x100x50 realisation of the workload, {secs:.1f} s "
                             f"of the reference's main loop (its own FP64 OpenMP build, oracle/_ref)"}
        else:
            steps = 200
            rate, dt = cpu_port_rate(steps, specs[0], opts[0])
            cpu = {"value": rate, "unit": "voxel-steps/s", "cores": 1, "kind": "port",
                   "sample": f"{steps} steps of one 100x100x50 realisation of the workload "
                             f"({dt:.1f} s), FP64 port of the reference"}

    # per step: voxel kernel, density-row flux kernel, channel-row gating/flux kernel, step
    # epilogue (the workload has both kinds of flux rows), in the device-timed region
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
                       "l2": "state 5.1 GB per GPU > L2, no flush needed", "parallelism": f"ensemble x{world}",
                       "tile": {"threads": tune["chosen"]["threads"], "x_planes_per_unit": tune["chosen"]["segment"],
                                "autotuned_from": len(tune["candidates"])}},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "kernel": "k_voxels_direct" if tune["chosen"]["segment"] < 0 else "k_voxels_staged",
                         "launch_ms": t_launch * 1e3,
                         "bytes_per_voxel": BYTES_PER_VOXEL_STEP, "peak_source": peak_kind,
                         "boundary_kernel_ms": bms / nprof},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "voxel-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": K, "call": "csp_run_states (FP32 host state, pipelined by realisation groups)"},
            "parity": parity,
            "gpu_launches": kernels,
            "plain_single_realisation": None if plain_single is None else {
                "value": plain_single, "unit": "voxel-steps/s",
                "workload": "one 100x100x50 realisation of the workload, same kernels"},
            "surrogate": sur,
            "other_configs": configs,
            "gathered_realisations": gathered,
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ens.close()
    sim2.close()
    D.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
