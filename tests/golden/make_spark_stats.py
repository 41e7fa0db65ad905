"""Spark statistics of the reference program (MT19937 channel gating), for test_spark_stats.

Runs oracle/_ref (the reference's own FP64 build) on the stochastic spark model of
spark_stats_model() with seeds 1..N, one channel of "ryr" forced open at t = 0 (-O ryr 0)
and every other channel gated stochastically, and stores per realisation:
  amplitude -- max over the outputs (t > 0) of the cleft's average Ca (uM);
  duration  -- time (ms) of the last output with a channel open;
  open      -- open channels at every output t > 0 (pooled by the test).
Writes tests/golden/spark_stats_ref.npz.  Needs oracle/_ref (built from the reference checkout);
takes a few minutes on 8 cores:  python tests/golden/make_spark_stats.py [N]
"""
import multiprocessing as mp
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

TSTOP, DT_SAVE = 2.0, 0.02


def spark_stats_model():
    import importlib
    synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
    g = np.array([-3, 0, 3])
    pts = np.array([(12 + a, 12 + b) for a in g for b in g])
    pmask = np.zeros(9, bool)
    pmask[[2, 6]] = True
    return synth.spark_model((24, 24, 20), channels=pts, pryr_mask=pmask, serca=True, patch_frac=0.6, margin=2,
                             jsr_voxels=3)


def stats_from_outputs(times, cleft_avg, open_counts):
    """Per-realisation statistics from the output series (t > 0 only)."""
    times, cleft_avg, open_counts = map(np.asarray, (times, cleft_avg, open_counts))
    sel = times > 0
    t, c, o = times[sel], cleft_avg[sel], open_counts[sel]
    amp = float(c.max())
    dur = float(t[o > 0].max()) if np.any(o > 0) else 0.0
    return amp, dur, o.astype(np.int32)


def one(seed):
    from oracle import refrun
    spec = spark_stats_model()
    wd = tempfile.mkdtemp(prefix=f"sparkstat{seed}_")
    res = refrun.run(spec, dict(h=6.0, tstop=TSTOP, dt_save=DT_SAVE, seed=seed, open_states={"ryr": [0]}), wd,
                     threads=1)
    outs = res["outputs"]
    times = [o["time"] for o in outs]
    cleft = [o["scalars"][("cleft", "Ca")][2] for o in outs]
    opn = [sum(int(v.sum()) for v in o["discrete"].values()) for o in outs]
    return stats_from_outputs(times, cleft, opn)


def main():
    n = int(sys.argv[1]) if len(sys.argv) > 1 else 160
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        res = pool.map(one, range(1, n + 1))
    amp = np.array([r[0] for r in res])
    dur = np.array([r[1] for r in res])
    opn = np.stack([r[2] for r in res])
    out = os.path.join(HERE, "spark_stats_ref.npz")
    np.savez_compressed(out, amplitude=amp, duration=dur, open=opn, tstop=TSTOP, dt_save=DT_SAVE)
    print(f"wrote {out}: {n} realisations, amplitude median {np.median(amp):.1f}, duration median "
          f"{np.median(dur):.3f} ms")


if __name__ == "__main__":
    main()
