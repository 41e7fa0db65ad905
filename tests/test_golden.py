"""Golden vectors produced by the reference program itself (tests/golden/make_golden.py).

CPU: the FP64 oracle reproduces them (fields stored as float32, so to float32 precision).
GPU: the CUDA path, through the C ABI, matches them at the FP32 accuracy bar (per-species
relative error <= 1e-4), with bit-exact channel states.
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
make_golden = importlib.import_module("make_golden")
# reference runs written by make_golden.py (they carry a "meta" record); other fixtures in
# the folder (the spark statistics) belong to their own tests
CASES = sorted(os.path.basename(p)[:-4] for p in glob.glob(os.path.join(HERE, "golden", "*.npz"))
               if "meta" in np.load(p).files)


def load(case):
    z = np.load(os.path.join(HERE, "golden", f"{case}.npz"))
    meta = json.loads(str(z["meta"]))
    spec, opts = make_golden.build(case)
    fields = np.stack([z[f"field_{sp}"].astype(np.float64) for sp in spec["species"]])
    disc = {k[len("discrete_"):]: z[k].astype(np.int32) for k in z.files if k.startswith("discrete_")}
    return spec, opts, meta, fields, disc


def check_scalars(spec, meta, mn, mx, tot, rtol):
    for key, (rmin, rmax, ravg) in meta["scalars"].items():
        dname, sp = key.split("/")
        di, si = spec["domains"].index(dname), spec["species"].index(sp)
        nvox = np.count_nonzero(spec["voxels"] == di)
        if nvox == 0:
            continue
        vol = nvox * spec["h"] ** 3
        np.testing.assert_allclose([mn[di, si], mx[di, si], tot[di, si] / vol], [rmin, rmax, ravg], rtol=rtol,
                                   atol=1e-9 * max(abs(rmax), 1.0))


def test_golden_cases_present():
    assert len(CASES) >= 4


@pytest.mark.parametrize("case", CASES)
def test_oracle_reproduces_reference_golden(case, oracle_mod):
    spec, opts, meta, ref, disc = load(case)
    orc = oracle_mod.Oracle(spec, opts)
    orc.step(meta["time_index"])
    u = orc.state()
    for s in range(ref.shape[0]):
        err = np.max(np.abs(u[s] - ref[s])) / np.max(np.abs(ref[s]))
        assert err < 1e-6, (case, s, err)
    for bname, st in disc.items():
        bi = [b["name"] for b in spec["boundaries"]].index(bname)
        np.testing.assert_array_equal(orc.channels(bi), st)
    mn, mx, tot = orc.outputs()
    check_scalars(spec, meta, mn, mx, tot, 1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", [0, 1])
@pytest.mark.parametrize("case", CASES)
def test_gpu_matches_reference_golden(case, kernel, pkg):
    spec, opts, meta, ref, disc = load(case)
    sim = pkg.Simulation(spec, opts)
    sim.set_kernel(kernel)
    sim.advance(meta["time_index"])
    assert sim.info().step == meta["time_index"]
    assert_close(sim.state(), ref, RTOL, what=f"{case} vs reference")
    for bname, st in disc.items():
        bi = [b["name"] for b in spec["boundaries"]].index(bname)
        np.testing.assert_array_equal(sim.channels(bi), st)
    mn, mx, tot, _ = sim.outputs()
    check_scalars(spec, meta, mn, mx, tot, RTOL)
