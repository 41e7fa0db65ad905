"""Input generators: the files either side of the calcium_sparks path.

    python -m hpc-ca-phospattern_b200.generate phospho GEOMETRY PATTERN.npy OUT.h5 [--offset K]
    python -m hpc-ca-phospattern_b200.generate synth CONFIG GEOMETRY_OUT SPECIES_OUT [--index R] [--seed S]

phospho -- the phosphorylated geometries the reference's run scripts use
(Run_scripts/G*/{inner,outer,uniform}_*) from its geometry with one "ryr" discrete
boundary and a 2-D channel map (createdgeometries/G*/G*_<pattern>.npy: 0 = no channel,
1 = RyR, 2 = pRyR): every pair of /boundaries/ryr whose map entry is 2 moves to a new
discrete boundary "p_ryr" (the name the phosphorylation parameter files use), in its
original order; the other boundaries are copied.  Channel (x, y) reads map entry
(x + K, y + K), K = (map size - geometry size) / 2 by default (42 for the 84^3 G1 and a
168x168 map, 0 for the 168^3 geometries).

synth -- the benchmark's synthetic inputs (configs 1-4 of the workload: one spark
100x100x50 at 6 nm; 200x200x100 with 100 channels, 20 % pRyR; one realisation R of the
256-member ensemble; one realisation R of the uneven ensemble), in the reference's formats.
"""
import argparse
import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
if os.path.dirname(HERE) not in sys.path:
    sys.path.insert(0, os.path.dirname(HERE))
h5m = importlib.import_module("hpc-ca-phospattern_b200.h5model")
synth = importlib.import_module("hpc-ca-phospattern_b200.synth")


def phospho(geometry_file, pattern, out_file, offset=None):
    """Split the ryr boundary of a geometry by a channel map; returns (n_ryr, n_pryr)."""
    spec = h5m.read_geometry(geometry_file)
    pat = np.load(pattern) if isinstance(pattern, str) else np.asarray(pattern)
    names = [b["name"] for b in spec["boundaries"]]
    if "ryr" not in names:
        raise ValueError(f"{geometry_file}: no boundary named 'ryr'")
    if "p_ryr" in names:
        raise ValueError(f"{geometry_file}: already has a 'p_ryr' boundary")
    bi = names.index("ryr")
    ryr = spec["boundaries"][bi]
    if ryr["type"] != "discrete":
        raise ValueError("the 'ryr' boundary is not discrete")
    if offset is None:
        n = spec["voxels"].shape[0]
        if pat.shape[0] < n or (pat.shape[0] - n) % 2:
            raise ValueError(f"map of {pat.shape} does not centre on a geometry of {spec['voxels'].shape}")
        offset = (pat.shape[0] - n) // 2
    pairs = np.asarray(ryr["pairs"]).reshape(-1, 6)
    xi, yi = pairs[:, 0].astype(int) + offset, pairs[:, 1].astype(int) + offset
    if (xi < 0).any() or (yi < 0).any() or (xi >= pat.shape[0]).any() or (yi >= pat.shape[1]).any():
        raise ValueError("channel outside the map")
    val = pat[xi, yi]
    if (val == 0).any():
        raise ValueError(f"{int((val == 0).sum())} channels have no entry in the map")
    keep, moved = pairs[val == 1], pairs[val == 2]
    bounds = []
    for k, b in enumerate(spec["boundaries"]):
        if k == bi:
            bounds.append(dict(name="ryr", type="discrete", pairs=keep))
            bounds.append(dict(name="p_ryr", type="discrete", pairs=moved))
        else:
            bounds.append(b)
    spec["boundaries"] = bounds
    h5m.write_geometry(spec, out_file)
    return int(len(keep)), int(len(moved))


def synth_config(config, index=0, seed=None):
    if config == 1:
        return synth.config1()
    if config == 2:
        return synth.config2(**({"seed": seed} if seed is not None else {}))
    if config == 3:
        specs, opts = synth.config3(n=index + 1, **({"seed": seed} if seed is not None else {}))
        return specs[index], opts[index]
    if config == 4:
        specs, opts = synth.config4(n=index + 1, **({"seed": seed} if seed is not None else {}))
        return specs[index], opts[index]
    raise ValueError(f"no synthetic config {config}")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m hpc-ca-phospattern_b200.generate", description=__doc__,
                                 formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="cmd", required=True)
    p = sub.add_parser("phospho", help="split the ryr boundary by a RyR/pRyR map")
    p.add_argument("geometry")
    p.add_argument("pattern")
    p.add_argument("out")
    p.add_argument("--offset", type=int, default=None)
    q = sub.add_parser("synth", help="write a synthetic benchmark input")
    q.add_argument("config", type=int, choices=[1, 2, 3, 4])
    q.add_argument("geometry_out")
    q.add_argument("species_out")
    q.add_argument("--index", type=int, default=0)
    q.add_argument("--seed", type=int, default=None)
    a = ap.parse_args(argv)
    if a.cmd == "phospho":
        n1, n2 = phospho(a.geometry, a.pattern, a.out, a.offset)
        print(f"{a.out}: ryr {n1} channels, p_ryr {n2} channels")
    else:
        res = synth_config(a.config, a.index, a.seed)
        spec = res[0] if isinstance(res, tuple) else res
        h5m.write_model(spec, a.geometry_out, a.species_out)
        opts = res[1] if isinstance(res, tuple) else None
        print(f"{a.geometry_out}, {a.species_out}: {spec['voxels'].shape} voxels at {spec['h']} nm"
              + (f"; options {opts}" if opts else ""))
    return 0


if __name__ == "__main__":
    sys.exit(main())
