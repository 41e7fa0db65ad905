"""Run the reference program (oracle/_ref, built by oracle/Makefile.ref) on a model.

TEST INFRASTRUCTURE ONLY: used by tests/ (oracle pinning), tests/golden/make_golden.py
and bench.py's reference arm.  Writes the model in the reference's HDF5 formats, runs
calcium_sparks with the reference's command line, and reads back its output file.
"""
import importlib
import os
import re
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
h5m = importlib.import_module("hpc-ca-phospattern_b200.h5model")


def cpu_has(flag):
    try:
        with open("/proc/cpuinfo") as f:
            return any(flag in line.split() for line in f if line.startswith("flags"))
    except OSError:
        return False


def ref_binary():
    """Path of the reference build for this CPU, or None if it was not built."""
    for name, ok in (("calcium_sparks_avx512", cpu_has("avx512f")), ("calcium_sparks_avx2", cpu_has("avx2"))):
        p = os.path.join(HERE, "_ref", name)
        if ok and os.path.exists(p):
            return p
    return None


def cli_args(opts, all_data=(), casename="case", verbose=False):
    """The reference's command line (calcium_sparks.c:19-45) for an options dict."""
    a = ["-c", casename, "-h", repr(float(opts.get("h", 6.0))), "-t", repr(float(opts.get("tstop", 10.0))),
         "-o", repr(float(opts.get("dt_save", 0.5)))]
    if opts.get("dt", -1) > 0:
        a += ["-d", repr(float(opts["dt"]))]
    if opts.get("dt_update_react", -1) > 0:
        a += ["-T", repr(float(opts["dt_update_react"]))]
    if opts.get("dt_update_stoch", -1) > 0:
        a += ["-D", repr(float(opts["dt_update_stoch"]))]
    if opts.get("force_dirichlet"):
        a += ["-f"]
    if opts.get("seed") is not None:
        a += ["-S", str(int(opts["seed"]))]
    if opts.get("tabort"):
        a += ["-X", repr(float(opts["tabort"]))]
    if opts.get("open_states"):
        a += ["-O"]
        for name, idx in opts["open_states"].items():
            a += [name] + [str(int(i)) for i in idx]
    if opts.get("t_close"):
        a += ["-C"]
        for name, t in opts["t_close"].items():
            a += [name, repr(float(t))]
    if all_data:
        a += ["--all_data"] + list(all_data)
    if verbose:
        a += ["-v"]
    return a


def run(spec, opts, workdir, all_data=(), threads=None, verbose=False, binary=None, timeout=3600):
    """Run the reference; returns dict(outputs=[...], stdout=str, mainloop_s=float|None)."""
    os.makedirs(workdir, exist_ok=True)
    h5m.write_model(spec, os.path.join(workdir, "geom.h5"), os.path.join(workdir, "species.h5"))
    return run_files("geom.h5", "species.h5", opts, workdir, all_data, threads, verbose, binary, timeout)


def run_files(geom, species, opts, workdir, all_data=(), threads=None, verbose=False, binary=None, timeout=3600):
    binary = binary or ref_binary()
    if not binary:
        raise FileNotFoundError("oracle/_ref was not built (make -C oracle -f Makefile.ref)")
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(threads or 1)
    out_h5 = os.path.join(workdir, "case.h5")
    if os.path.exists(out_h5):
        os.remove(out_h5)
    cmd = [binary, "-g", geom, "-m", species] + cli_args(opts, all_data, "case", verbose)
    r = subprocess.run(cmd, cwd=workdir, env=env, capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError(f"reference failed ({r.returncode}): {r.stderr[-2000:]}")
    res = {"stdout": r.stdout, "outputs": read_output(out_h5), "cmd": cmd}
    m = re.search(r"Main Loop time\|\s*([0-9.eE+-]+)\|", r.stdout)
    res["mainloop_s"] = float(m.group(1)) if m else None
    return res


def read_output(path):
    """Every /data_%07d group of a calcium_sparks output file (species.c:2253-2298)."""
    outs = []
    with h5m.H5(path) as f:
        for is_group, name in f.list("/"):
            if not (is_group and name.startswith("data_")):
                continue
            g = "/" + name
            o = {"name": name, "time": float(np.atleast_1d(f.attr(g, "time"))[0]),
                 "time_index": int(np.atleast_1d(f.attr(g, "time_index"))[0]), "fields": {}, "scalars": {},
                 "discrete": {}}
            for sub_is_group, sub in f.list(g):
                if sub_is_group:
                    for _, sp in f.list(f"{g}/{sub}"):
                        o["scalars"][(sub, sp)] = tuple(float(np.atleast_1d(f.attr(f"{g}/{sub}/{sp}", k))[0])
                                                        for k in ("min", "max", "average"))
                elif sub.endswith("_all_data"):
                    o["fields"][sub[:-len("_all_data")]] = f.dset(f"{g}/{sub}")
                elif sub.startswith("discrete_"):
                    o["discrete"][sub[len("discrete_"):]] = f.dset(f"{g}/{sub}")
            outs.append(o)
    outs.sort(key=lambda o: o["name"])
    return outs
