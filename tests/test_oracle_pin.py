"""Pin the FP64 oracle to the reference program itself (CPU, no GPU).

The reference ships no tests or golden vectors, so the reference's own sources are built
here (oracle/Makefile.ref: single-rank MPI stub + HDF5 shim) and run on the same models;
its --all_data fields, per-domain min/max/average and channel states must match the
oracle's to FP64 rounding.  Cases cover forced channels (-O/-C), subdivisions, Dirichlet
faces (-f), fixed domain species, reaction / channel substeps (-T/-D), and the
reference's own G1 geometry with its parameter file.
"""
import os

import numpy as np
import pytest

from oracle import refrun
from oracle.refsrc import reference_file

BIN = refrun.ref_binary()
pytestmark = pytest.mark.skipif(BIN is None, reason="oracle/_ref not built")
DT = 0.95 * 36 / (6 * 220000.0)


def compare(spec, opts, tmp_path, species=("Ca", "Fluo", "CMDN", "ATP", "TRPN"), tol=1e-11):
    from oracle.oracle import Oracle
    res = refrun.run(spec, opts, str(tmp_path), all_data=species)
    orc = Oracle(spec, opts)
    prev = 0
    assert res["outputs"], "reference wrote no output"
    names = spec["species"]
    for o in res["outputs"]:
        orc.step(o["time_index"] - prev)
        prev = o["time_index"]
        u = orc.state()
        for sp, ref in o["fields"].items():
            si = names.index(sp)
            err = np.max(np.abs(ref - u[si])) / max(np.max(np.abs(ref)), 1e-300)
            assert err < tol, f"{o['name']} {sp}: oracle vs reference rel diff {err:.3e}"
        mn, mx, tot = orc.outputs()
        for (dname, sp), (rmin, rmax, ravg) in o["scalars"].items():
            di, si = spec["domains"].index(dname), names.index(sp)
            vol = np.count_nonzero(spec["voxels"] == di) * spec["h"] ** 3
            if vol == 0:
                assert rmin == np.float32(3.4028235e38) and rmax == np.float32(1.1754944e-38)
                continue
            np.testing.assert_allclose([mn[di, si], mx[di, si], tot[di, si] / vol], [rmin, rmax, ravg], rtol=1e-9,
                                       atol=1e-12)
        for bname, states in o["discrete"].items():
            bi = [b["name"] for b in spec["boundaries"]].index(bname)
            np.testing.assert_array_equal(orc.channels(bi), states.astype(np.int32))
    return res


def test_pin_forced_channels(synth, tmp_path):
    spec = synth.tiny((12, 12, 16))
    opts = dict(h=6.0, tstop=0.005, dt_save=0.0025, seed=1, open_states={"ryr": [0, 3], "p_ryr": [1]},
                t_close={"ryr": 0.004, "p_ryr": 0.006})
    compare(spec, opts, tmp_path)


def test_pin_subdivisions(synth, tmp_path):
    spec = synth.tiny((8, 8, 10))
    spec["h"] = 12.0
    opts = dict(h=6.0, tstop=0.004, dt_save=0.002, seed=1, open_states={"ryr": [0, 2], "p_ryr": [0]},
                t_close={"ryr": 1.0, "p_ryr": 1.0})
    compare(spec, opts, tmp_path)


def test_pin_dirichlet_fixed_substeps(synth, tmp_path):
    spec = synth.tiny((12, 12, 16))
    spec["fixed_domain_species"] = [(3, 0)]
    opts = dict(h=6.0, tstop=0.006, dt_save=0.003, seed=4, force_dirichlet=True, dt_update_react=3.5 * DT,
                dt_update_stoch=2 * DT, open_states={"ryr": [1, 4], "p_ryr": [1]}, t_close={"ryr": 0.003, "p_ryr": 1.0})
    compare(spec, opts, tmp_path)


def test_pin_forced_dt_odd_sizes(synth, tmp_path):
    spec = synth.tiny((11, 9, 13), serca=False)
    opts = dict(h=6.0, dt=2e-5, tstop=0.003, dt_save=0.0015, seed=9, open_states={"ryr": [4], "p_ryr": [0]},
                t_close={"ryr": 1.0, "p_ryr": 1.0})
    compare(spec, opts, tmp_path)


G1 = reference_file("createdgeometries", "G1", "G1_nonP_0.h5")
P55 = reference_file("parameters", "nonP_blanket", "parameters_sr1100_ryr55.h5")


@pytest.mark.skipif(not (G1 and P55), reason="reference input files absent")
def test_pin_reference_g1_geometry(tmp_path):
    """The reference's own G1 geometry (84^3 at 12 nm) and parameter file."""
    import importlib
    from oracle.oracle import Oracle
    h5m = importlib.import_module("hpc-ca-phospattern_b200.h5model")
    spec = h5m.read_model(G1, P55)
    opts = dict(h=12.0, tstop=2.5e-3, dt_save=1.2e-3, seed=1, open_states={"ryr": list(range(10))},
                t_close={"ryr": 2e-3})
    res = refrun.run_files(G1, P55, opts, str(tmp_path), all_data=("Ca", "CMDN-CSQN"), threads=8)
    orc = Oracle(spec, opts)
    prev = 0
    for o in res["outputs"]:
        orc.step(o["time_index"] - prev)
        prev = o["time_index"]
        u = orc.state()
        for sp, ref in o["fields"].items():
            si = spec["species"].index(sp)
            err = np.max(np.abs(ref - u[si])) / np.max(np.abs(ref))
            assert err < 1e-11, f"G1 {o['name']} {sp}: {err:.3e}"
        np.testing.assert_array_equal(orc.channels(1), o["discrete"]["ryr"].astype(np.int32))
