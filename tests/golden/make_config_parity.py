"""Generate the fixtures of the benchmark-size parity tests by running the reference program.

    python tests/golden/make_config_parity.py [case ...]

The four benchmark configurations, each run by the reference program (oracle/_ref, its
own FP64 OpenMP build from its sources) with every channel forced (-O lists, -C times
for every discrete boundary: no random draw, deterministic):

  config1_full      100x100x50 at 6 nm, 5x5 RyR cluster, RyR 0 open, the full 2 ms
                    (77,194 steps) -- the plain FP64 configuration;
  config2_short     200x200x100 at 6 nm, 10x10 lattice with vacancies, 20 % pRyR,
                    dt_update_stoch = dt, shortened to 0.5 ms (19,298 steps);
  config3_r0        realisation 0 of the batched ensemble (100x100x50, its own cluster
                    shape and pRyR pattern), shortened to 1 ms, no -X;
  config4_largest   the largest grid of the uneven ensemble (h between 6 and 10 nm,
                    dt_update_react = 5 dt), shortened to about 2,000 steps.

What is stored per case (np.savez_compressed, a few hundred KB each):
  * the per-(domain, species) min / max / average of every output (species.c:2785-2880);
  * the channel states of every discrete boundary at the last output;
  * the last output's fields (--all_data) in float32 at two voxel sets: a lattice of
    every s-th voxel along each axis (s chosen so a species has at most 40,000 lattice
    voxels) and, at full resolution, the planes from one below the cleft to the first
    SR plane in a window around the channel cluster (the steepest gradients);
  * a SHA-1 of the model (voxels, boundary pairs) so a test can tell that the builder
    still makes the same inputs.

The tests rebuild each model from CASES and compare the CUDA path through the C ABI.
"""
import hashlib
import importlib
import json
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
synth = importlib.import_module("hpc-ca-phospattern_b200.synth")

LATTICE_MAX = 40000
WINDOW_MARGIN = 6
OUT = os.path.join(HERE, "configs")


def _dt(h):
    return 0.95 * h * h / (6 * 220000.0)


def _config1():
    spec, opts = synth.config1()
    opts = dict(opts, dt_save=0.25, t_close={"ryr": 2.0})
    return spec, opts


def _config2():
    spec, opts = synth.config2()
    names = [b["name"] for b in spec["boundaries"]]
    n_ryr = len(spec["boundaries"][names.index("ryr")]["pairs"])
    n_pryr = len(spec["boundaries"][names.index("p_ryr")]["pairs"])
    opts = dict(opts, tstop=0.5, dt_save=0.125, dt_update_stoch=_dt(6.0),
                open_states={"ryr": list(range(0, n_ryr, 9)), "p_ryr": list(range(0, n_pryr, 6))},
                t_close={"ryr": 0.3, "p_ryr": 0.2})
    return spec, opts


def _config3():
    specs, opts = synth.config3(n=1)
    spec, o = specs[0], dict(opts[0])
    o.pop("tabort", None)
    names = [b["name"] for b in spec["boundaries"]]
    o["open_states"] = {"ryr": [0]}
    o["t_close"] = {"ryr": 0.6}
    if "p_ryr" in names:
        o["open_states"]["p_ryr"] = [0]
        o["t_close"]["p_ryr"] = 0.4
    o.update(tstop=1.0, dt_save=0.25)
    return spec, o


def _config4():
    specs, opts = synth.config4()
    big = int(np.argmax([s["voxels"].size for s in specs]))
    spec, o = specs[big], dict(opts[big])
    dt = _dt(o["h"])
    tstop = 2000 * dt
    o.update(tstop=tstop, dt_save=tstop / 4, open_states={"ryr": [0, 12]}, t_close={"ryr": tstop / 2})
    return spec, o


CASES = {"config1_full": _config1, "config2_short": _config2, "config3_r0": _config3,
         "config4_largest": _config4}


def build(case):
    return CASES[case]()


def model_digest(spec):
    """SHA-1 of the geometry and boundary pairs of a model."""
    m = hashlib.sha1()
    m.update(np.ascontiguousarray(spec["voxels"]).tobytes())
    for b in spec["boundaries"]:
        m.update(b["name"].encode())
        m.update(np.ascontiguousarray(b["pairs"], dtype=np.uint16).tobytes())
    return m.hexdigest()


def lattice_stride(shape):
    s = 1
    while np.prod([(n + s - 1) // s for n in shape]) > LATTICE_MAX:
        s += 1
    return s


def window(spec):
    """(x0, x1, y0, y1, z0, z1): the channel cluster's bounding box widened by
    WINDOW_MARGIN in x and y, from one plane below the cleft to the first SR plane."""
    pts = np.concatenate([np.asarray(b["pairs"])[:, :2] for b in spec["boundaries"] if b["type"] == "discrete"])
    nx, ny, _ = spec["voxels"].shape
    lay = spec["layout"]
    x0 = max(0, int(pts[:, 0].min()) - WINDOW_MARGIN)
    x1 = min(nx, int(pts[:, 0].max()) + WINDOW_MARGIN + 1)
    y0 = max(0, int(pts[:, 1].min()) - WINDOW_MARGIN)
    y1 = min(ny, int(pts[:, 1].max()) + WINDOW_MARGIN + 1)
    z0 = max(0, lay["cleft_z"][0] - 1)
    z1 = lay["sr_z"][0] + 1
    return x0, x1, y0, y1, z0, z1


def samples(fields, spec):
    """The two stored voxel sets of fields [species][x][y][z]: (lattice, window)."""
    s = lattice_stride(fields.shape[1:])
    x0, x1, y0, y1, z0, z1 = window(spec)
    return fields[:, ::s, ::s, ::s], fields[:, x0:x1, y0:y1, z0:z1]


def main(names):
    from oracle import refrun
    for case in names:
        spec, opts = build(case)
        t = time.time()
        with tempfile.TemporaryDirectory() as d:
            res = refrun.run(spec, opts, d, all_data=spec["species"], threads=os.cpu_count(), verbose=True)
        outs = res["outputs"]
        last = outs[-1]
        fields = np.stack([last["fields"][sp] for sp in spec["species"]])
        lat, win = samples(fields, spec)
        nd, ns = len(spec["domains"]), len(spec["species"])
        scal = np.full((len(outs), nd, ns, 3), np.nan)
        for k, o in enumerate(outs):
            for (dname, sp), v in o["scalars"].items():
                scal[k, spec["domains"].index(dname), spec["species"].index(sp)] = v
        arrays = {"scalars": scal, "time_index": np.array([o["time_index"] for o in outs], dtype=np.int64),
                  "time": np.array([o["time"] for o in outs]), "lattice": lat.astype(np.float32),
                  "window": win.astype(np.float32)}
        for bname, st in last["discrete"].items():
            arrays[f"discrete_{bname}"] = st.astype(np.int8)
        meta = dict(case=case, shape=list(spec["voxels"].shape), h=opts["h"], model_sha1=model_digest(spec),
                    stride=lattice_stride(fields.shape[1:]), window=list(window(spec)),
                    mainloop_s=res["mainloop_s"], threads=os.cpu_count(),
                    reference_cmd=" ".join(os.path.basename(c) if i == 0 else c for i, c in enumerate(res["cmd"])))
        os.makedirs(OUT, exist_ok=True)
        np.savez_compressed(os.path.join(OUT, f"{case}.npz"), meta=json.dumps(meta), **arrays)
        print(case, "steps", arrays["time_index"][-1], "outputs", len(outs), "lattice", lat.shape, "window",
              win.shape, f"{time.time() - t:.0f} s", flush=True)


if __name__ == "__main__":
    main(sys.argv[1:] or list(CASES))
