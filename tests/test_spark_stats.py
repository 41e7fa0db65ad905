"""Stochastic gating: GPU Philox streams against the reference's MT19937, statistically.

The two generators cannot give the same draws, so the channel dynamics are compared as
distributions.  The reference program ran an ensemble of stochastic sparks (one RyR
forced open at t = 0, every other channel gated by evaluate_RyR_stochastically,
boundaryfluxes.c:295-359) with seeds 1..N; tests/golden/make_spark_stats.py stored its
per-realisation statistics.  Here one batched handle runs the same model with a Philox
stream per (seed, realisation), and the per-realisation distributions must not differ at
the 1 % level (two-sample Kolmogorov-Smirnov, p > 0.01):
  spark amplitude -- peak over the outputs of the cleft's average Ca;
  spark duration  -- time of the last output with a channel open;
  open-channel counts -- the time-averaged and the peak open count of each realisation.
"""
import math
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
GOLD = os.path.join(HERE, "golden", "spark_stats_ref.npz")
N_GPU = 320


def gpu_ensemble(pkg, n, seed=20261203):
    from make_spark_stats import DT_SAVE, TSTOP, spark_stats_model, stats_from_outputs
    spec = spark_stats_model()
    opts = dict(h=6.0, tstop=TSTOP, dt_save=DT_SAVE, seed=seed, open_states={"ryr": [0]})
    sim = pkg.Simulation([spec] * n, [opts] * n)
    info = sim.info(0)
    dt, total = info.dt, info.total_steps
    save_interval = max(1, math.floor(DT_SAVE / dt))
    ci, si = spec["domains"].index("cleft"), spec["species"].index("Ca")
    vol = np.count_nonzero(spec["voxels"] == ci) * spec["h"] ** 3
    series = [([], [], []) for _ in range(n)]
    k, t = 0, 0.0
    while k + save_interval <= total:
        sim.advance(save_interval)
        for _ in range(save_interval):
            t += dt
        k += save_interval
        for r in range(n):
            mn, mx, tot, op = sim.outputs(r)
            series[r][0].append(t)
            series[r][1].append(tot[ci, si] / vol)
            series[r][2].append(int(op.sum()))
    sim.close()
    return [stats_from_outputs(*s) for s in series]


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(GOLD), reason="reference spark statistics not generated")
def test_spark_statistics_match_reference(pkg):
    from scipy.stats import ks_2samp
    ref = np.load(GOLD)
    res = gpu_ensemble(pkg, N_GPU)
    amp = np.array([r[0] for r in res])
    dur = np.array([r[1] for r in res])
    opn = np.stack([r[2] for r in res])
    ropn = ref["open"]
    assert opn.shape[1] == ropn.shape[1], "different number of outputs"
    checks = {
        "amplitude": (ref["amplitude"], amp),
        "duration": (ref["duration"], dur),
        "mean open channels": (ropn.mean(axis=1), opn.mean(axis=1)),
        "peak open channels": (ropn.max(axis=1), opn.max(axis=1)),
    }
    report = []
    for name, (a, b) in checks.items():
        p = ks_2samp(a, b).pvalue
        report.append(f"{name}: ref median {np.median(a):.4g}, gpu median {np.median(b):.4g}, KS p = {p:.3f}")
        assert p > 0.01, "\n".join(report)
    print("\n".join(report))
