"""Parity at the benchmark configurations: the CUDA path against the reference program.

The fixtures (tests/golden/configs/*.npz, made by tests/golden/make_config_parity.py)
hold the reference program's own FP64 run (oracle/_ref, every channel forced with -O/-C,
so deterministic) of:

  config1_full      100x100x50, the full 2 ms (77,192 steps);
  config2_short     200x200x100 with its 10x10 lattice and 20 % pRyR, 0.5 ms;
  config3_r0        realisation 0 of the batched ensemble, 1 ms;
  config4_largest   the largest grid of the uneven ensemble (204x246x120 at 9.9 nm,
                    dt_update_react = 5 dt), 2,000 steps.

CPU: the builders still make the models the fixtures were run on (SHA-1 of voxels and
boundary pairs).  GPU: the FP32 path through the C ABI is advanced output by output; at
every output the per-(domain, species) min / max / average must lie within 1e-4 of that
pair's scale (species.c:2785-2880), and at the last output every species field, on the
stored voxel sets, must meet the FP32 accuracy bar of tests/parity.py (per-species
max |diff| / max |ref| <= 1e-4 and pointwise |diff| <= 1e-4 |ref| + 1e-7 max |ref|); channel
states must be equal.
"""
import glob
import importlib
import json
import os
import sys

import numpy as np
import pytest

from parity import RTOL, assert_close

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
mcp = importlib.import_module("make_config_parity")
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(mcp.OUT, "*.npz")))


def load(case):
    z = np.load(os.path.join(mcp.OUT, f"{case}.npz"))
    meta = json.loads(str(z["meta"]))
    spec, opts = mcp.build(case)
    return spec, opts, meta, z


def test_every_configuration_has_a_fixture():
    assert CASES == sorted(mcp.CASES), CASES


@pytest.mark.parametrize("case", CASES)
def test_builders_make_the_fixture_models(case):
    spec, opts, meta, z = load(case)
    assert mcp.model_digest(spec) == meta["model_sha1"]
    assert list(spec["voxels"].shape) == meta["shape"]
    lat, win = mcp.samples(np.zeros((len(spec["species"]),) + spec["voxels"].shape), spec)
    assert lat.shape == z["lattice"].shape and win.shape == z["window"].shape
    assert z["scalars"].shape == (len(z["time_index"]), len(spec["domains"]), len(spec["species"]), 3)
    assert np.all(np.diff(z["time_index"]) > 0)


def check_scalars(case, k, spec, h, ref, mn, mx, tot):
    """Output k's per-(domain, species) min / max / average against the reference; the
    average is the total sum(u dV) over the domain's volume, dV = h^3 (subdivisions 1)."""
    worst = 0.0
    for di, dname in enumerate(spec["domains"]):
        nvox = np.count_nonzero(spec["voxels"] == di)
        for si, sp in enumerate(spec["species"]):
            rmn, rmx, ravg = ref[di, si]
            if nvox == 0:
                # the reference's FLT_MAX / FLT_MIN start values and 0/0 average (species.c:2808-2815, 3046)
                assert mn[di, si] == np.float32(rmn) and mx[di, si] == np.float32(rmx) and np.isnan(ravg)
                continue
            scale = max(abs(rmn), abs(rmx), 1e-30)
            avg = tot[di, si] / (nvox * h ** 3)
            for a, b in ((mn[di, si], rmn), (mx[di, si], rmx), (avg, ravg)):
                err = abs(a - b) / scale
                worst = max(worst, err)
                assert err <= RTOL, f"{case} output {k} {dname}/{sp}: {a} vs {b} (rel {err:.2e})"
    return worst


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_reference_at_configuration(case, pkg):
    spec, opts, meta, z = load(case)
    sim = pkg.Simulation(spec, opts)
    inf = sim.info()
    assert inf.subdivisions == 1 and abs(inf.h - meta["h"]) < 1e-12
    worst = 0.0
    for k, ti in enumerate(z["time_index"]):
        sim.advance(int(ti) - sim.info().step)
        assert sim.info().step == ti
        mn, mx, tot, _ = sim.outputs()
        worst = max(worst, check_scalars(case, k, spec, inf.h, z["scalars"][k], mn, mx, tot))
    lat, win = mcp.samples(sim.state(), spec)
    e_lat = assert_close(lat, z["lattice"].astype(np.float64), RTOL, what=f"{case} lattice")
    e_win = assert_close(win, z["window"].astype(np.float64), RTOL, what=f"{case} window")
    for bname in [k[len("discrete_"):] for k in z.files if k.startswith("discrete_")]:
        bi = [b["name"] for b in spec["boundaries"]].index(bname)
        np.testing.assert_array_equal(sim.channels(bi), z[f"discrete_{bname}"].astype(np.int32))
    sim.close()
    print(f"\n{case}: {int(z['time_index'][-1])} steps, per-species rel err lattice {np.array2string(e_lat, precision=2)}"
          f" window {np.array2string(e_win, precision=2)}, worst output scalar {worst:.2e}")
