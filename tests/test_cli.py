"""The calcium_sparks driver (bin/calcium_sparks) against the reference program.

CPU tests: command-line errors give the reference's message on stderr and exit status 1
(options.c, calcium_sparks.c:99-146).  GPU tests: both programs run on the same geometry
and species files with the same options; every /data_%07d group must match -- time,
time_index, per (domain, species) min / max / average, discrete channel states, the
--all_data fields, the -s sheets and the -l linescan -- with FP32 fields against the
reference's FP64 ones at relative error <= 1e-4 of each field's scale.  The -X abort rule
(evaluated on the channel states of the last output, species.c:3384-3486) must end both
runs after the same output.
"""
import importlib
import os
import subprocess

import numpy as np
import pytest

from oracle import refrun

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "hpc-ca-phospattern_b200", "bin", "calcium_sparks")
REF = refrun.ref_binary()
h5m = importlib.import_module("hpc-ca-phospattern_b200.h5model")
RTOL = 1e-4

needs_both = pytest.mark.skipif(not (os.path.exists(CLI) and REF), reason="CLI or oracle/_ref not built")


def model_files(synth, tmp_path, shape=(12, 12, 16)):
    spec = synth.tiny(shape)
    g, s = str(tmp_path / "geom.h5"), str(tmp_path / "species.h5")
    h5m.write_model(spec, g, s)
    return spec, g, s


def run(binary, args, cwd):
    return subprocess.run([binary] + args, cwd=cwd, capture_output=True, text=True, timeout=600)


BAD = [
    ["-t", "1"],                                                   # no geometry file
    ["-g", "geom.h5", "-t", "1"],                                  # no species file
    ["-g", "geom.h5", "-m", "species.h5", "-O", "ryr", "3", "1"],  # decreasing -O indices
    ["-g", "geom.h5", "-m", "species.h5", "-p", "AB"],             # bad -p plane
    ["-g", "geom.h5", "-m", "species.h5", "-l", "w", "Ca", "0", "0"],   # bad linescan axis
    ["-g", "geom.h5", "-m", "species.h5", "-O", "ryr", "0", "99"],      # -O index past the channels
]


@needs_both
@pytest.mark.parametrize("args", BAD, ids=["no-g", "no-m", "O-order", "p-plane", "l-axis", "O-range"])
def test_cli_errors_match_reference(synth, tmp_path, args):
    model_files(synth, tmp_path)
    ours = run(CLI, args, str(tmp_path))
    ref = run(REF, args, str(tmp_path))
    assert ref.returncode != 0
    assert ours.returncode == 1
    first = [ln for ln in ref.stderr.splitlines() if ln.strip()][0]
    assert first in ours.stderr, f"reference: {first!r}\nours: {ours.stderr!r}"


def compare_outputs(ours_path, ref_path, spec, fields=(), linescan=False, sheets=False):
    ours = refrun.read_output(ours_path)
    ref = refrun.read_output(ref_path)
    assert [o["name"] for o in ours] == [o["name"] for o in ref]
    scale = {}
    for o, r in zip(ours, ref):
        assert o["time_index"] == r["time_index"]
        assert o["time"] == pytest.approx(r["time"], rel=1e-12)
        assert set(o["scalars"]) == set(r["scalars"])
        for key, (rmn, rmx, ravg) in r["scalars"].items():
            omn, omx, oavg = o["scalars"][key]
            s = max([abs(v) for v in (rmx, rmn) if np.isfinite(v) and abs(v) < 3e38] + [1e-30])
            scale[key[1]] = max(scale.get(key[1], 0.0), s)
            for a, b in ((omn, rmn), (omx, rmx), (oavg, ravg)):
                if np.isnan(b):                                  # average of an empty domain: 0/0
                    assert np.isnan(a), f"{r['name']} {key}: {a} vs nan"
                elif abs(b) >= 3e38 or (0 < abs(b) < 1.2e-38):   # FLT_MAX / FLT_MIN of empty domains
                    assert a == b
                else:
                    assert abs(a - b) <= RTOL * s, f"{r['name']} {key}: {a} vs {b}"
        assert set(o["discrete"]) == set(r["discrete"])
        for b, st in r["discrete"].items():
            np.testing.assert_array_equal(o["discrete"][b], st)
        for sp in fields:
            a, b = o["fields"][sp], r["fields"][sp]
            err = np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-30)
            assert err <= RTOL, f"{r['name']} {sp}_all_data: rel err {err:.2e}"
    return ours, ref


def read_extra(path, prefix):
    out = {}
    with h5m.H5(path) as f:
        for is_group, name in f.list("/"):
            if not (is_group and name.startswith("data_")):
                continue
            for sub_is_group, sub in f.list("/" + name):
                if not sub_is_group and sub.startswith(prefix):
                    out[(name, sub)] = f.dset(f"/{name}/{sub}")
    return out


@needs_both
@pytest.mark.gpu
def test_cli_matches_reference_outputs(synth, tmp_path):
    spec, g, s = model_files(synth, tmp_path)
    args = ["-g", g, "-m", s, "-c", "case", "-h", "6", "-t", "0.006", "-o", "0.002", "-S", "3",
            "-O", "ryr", "0", "3", "p_ryr", "1", "-C", "ryr", "0.004", "p_ryr", "0.005",
            "--all_data", "Ca", "Fluo", "-s", "Ca", "-z", "42", "66", "-x", "30",
            "-l", "x", "Ca", "-1", "2"]
    ours_dir, ref_dir = tmp_path / "ours", tmp_path / "ref"
    ours_dir.mkdir()
    ref_dir.mkdir()
    ro = run(CLI, args, str(ours_dir))
    assert ro.returncode == 0, ro.stderr[-2000:]
    rr = run(REF, args, str(ref_dir))
    assert rr.returncode == 0, rr.stderr[-2000:]
    compare_outputs(str(ours_dir / "case.h5"), str(ref_dir / "case.h5"), spec, fields=("Ca", "Fluo"))
    # sheets and linescan datasets: same names, values within tolerance
    for prefix in ("Ca_z_sheet", "Ca_x_sheet", "linescan_"):
        a = read_extra(str(ours_dir / "case.h5"), prefix)
        b = read_extra(str(ref_dir / "case.h5"), prefix)
        assert a.keys() == b.keys() and len(b) > 0, (prefix, sorted(a), sorted(b))
        for key in b:
            err = np.max(np.abs(a[key] - b[key])) / max(np.max(np.abs(b[key])), 1e-30)
            assert err <= RTOL, f"{key}: rel err {err:.2e}"
    # console: the per-output channel tables are identical
    chan_o = [ln for ln in ro.stdout.splitlines() if "|" in ln and ":" in ln]
    chan_r = [ln for ln in rr.stdout.splitlines() if "|" in ln and ":" in ln]
    assert chan_o == chan_r


@needs_both
@pytest.mark.gpu
def test_cli_abort_rule_matches_reference(synth, tmp_path):
    """-X: channels forced closed at 1.5 ms; both runs end after the same output."""
    spec, g, s = model_files(synth, tmp_path)
    args = ["-g", g, "-m", s, "-c", "case", "-h", "6", "-t", "0.05", "-o", "0.0005", "-S", "5",
            "-O", "ryr", "0", "p_ryr", "0", "-C", "ryr", "0.0015", "p_ryr", "0.0015", "-X", "0.002"]
    ours_dir, ref_dir = tmp_path / "ours", tmp_path / "ref"
    ours_dir.mkdir()
    ref_dir.mkdir()
    ro = run(CLI, args, str(ours_dir))
    assert ro.returncode == 0, ro.stderr[-2000:]
    rr = run(REF, args, str(ref_dir))
    assert rr.returncode == 0, rr.stderr[-2000:]
    ours, ref = compare_outputs(str(ours_dir / "case.h5"), str(ref_dir / "case.h5"), spec)
    total = round(0.05 / (0.95 * 36 / (6 * 220000.0)))
    assert ref[-1]["time_index"] < total * 0.5, "the reference run did not abort"


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
@pytest.mark.gpu
def test_cli_verbose_timing_buckets(synth, tmp_path):
    """-v: the reference's timing table (utils.c:11-75) with the step's buckets filled from
    the library's per-phase device times: every step counted in Diffusion stencil,
    Boundary fluxes and Stochastic evaluation, their times within the main loop's."""
    spec, g, s = model_files(synth, tmp_path)
    args = ["-g", g, "-m", s, "-c", "case", "-h", "6", "-t", "0.004", "-o", "0.002", "-S", "3",
            "-O", "ryr", "0", "-v"]
    r = run(CLI, args, str(tmp_path))
    assert r.returncode == 0, r.stderr[-2000:]
    rows = {}
    for ln in r.stdout.splitlines():
        parts = ln.split("|")
        if len(parts) == 5:
            rows[parts[0].strip()] = (float(parts[1]), int(parts[4]))
    steps = round(0.004 / (0.95 * 36 / (6 * 220000.0)))
    for name in ("Diffusion stencil", "Boundary fluxes", "Stochastic evaluation", "Diffusion Total"):
        assert abs(rows[name][1] - steps) <= 1, (name, rows[name], steps)
    main = rows["Main Loop time"][0]
    assert rows["Diffusion stencil"][0] + rows["Boundary fluxes"][0] + rows["Stochastic evaluation"][0] <= main + 0.1
