"""Generate the golden fixtures of the GPU parity tests by running the reference program.

    python tests/golden/make_golden.py

Each case builds a model with hpc-ca-phospattern_b200.synth, runs the reference
program (oracle/_ref, compiled from the reference's own sources by oracle/Makefile.ref)
on it with every channel forced (-O / -C, deterministic), and stores the reference's
output at its last output step: every species field (--all_data, stored as float32),
the per-domain min / max / average and the channel states.  The GPU tests rebuild the
same model from the case parameters and compare against these arrays.
"""
import importlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
synth = importlib.import_module("hpc-ca-phospattern_b200.synth")
DT = 0.95 * 36 / (6 * 220000.0)

# name -> (synth builder kwargs, spec overrides, options)
CASES = {
    "forced_12x12x16": (dict(shape=(12, 12, 16)), {},
                        dict(h=6.0, tstop=0.005, dt_save=0.0025, seed=1, open_states={"ryr": [0, 3], "p_ryr": [1]},
                             t_close={"ryr": 0.004, "p_ryr": 0.006})),
    "subdiv_8x8x10_h12": (dict(shape=(8, 8, 10)), {"h": 12.0},
                          dict(h=6.0, tstop=0.004, dt_save=0.002, seed=1, open_states={"ryr": [0, 2], "p_ryr": [0]},
                               t_close={"ryr": 1.0, "p_ryr": 1.0})),
    "dirichlet_fixed_substeps": (dict(shape=(12, 12, 16)), {"fixed_domain_species": [(3, 0)]},
                                 dict(h=6.0, tstop=0.006, dt_save=0.003, seed=4, force_dirichlet=True,
                                      dt_update_react=3.5 * DT, dt_update_stoch=2 * DT,
                                      open_states={"ryr": [1, 4], "p_ryr": [1]}, t_close={"ryr": 0.003, "p_ryr": 1.0})),
    "long_20x20x24": (dict(shape=(20, 20, 24)), {},
                      dict(h=6.0, tstop=0.03, dt_save=0.015, seed=2, open_states={"ryr": [0, 1, 2, 3], "p_ryr": [0, 1]},
                           t_close={"ryr": 0.02, "p_ryr": 0.025})),
}


def build(case):
    kw, over, opts = CASES[case]
    spec = synth.tiny(**kw)
    spec.update(over)
    return spec, opts


def main():
    from oracle import refrun
    for case in CASES:
        spec, opts = build(case)
        with tempfile.TemporaryDirectory() as d:
            res = refrun.run(spec, opts, d, all_data=spec["species"])
        o = res["outputs"][-1]
        arrays = {f"field_{sp}": o["fields"][sp].astype(np.float32) for sp in spec["species"]}
        for bname, st in o["discrete"].items():
            arrays[f"discrete_{bname}"] = st.astype(np.int8)
        scal = {f"{d}/{sp}": v for (d, sp), v in o["scalars"].items()}
        meta = dict(case=case, time_index=o["time_index"], time=o["time"], scalars=scal,
                    reference_cmd=" ".join(os.path.basename(c) if i == 0 else c for i, c in enumerate(res["cmd"])))
        np.savez_compressed(os.path.join(HERE, f"{case}.npz"), meta=json.dumps(meta), **arrays)
        print(case, o["time_index"], {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
