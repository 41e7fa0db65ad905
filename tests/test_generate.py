"""Input generators (hpc-ca-phospattern_b200/generate.py), CPU only.

* phospho: the reference's G1 geometry split by its inner_10 channel map gives 40 RyR and
  10 pRyR channels (the README's "inner 20 %"), every channel on its map value, the other
  boundaries untouched; the reference program accepts the file with its own
  phosphorylation parameter file, and the FP64 oracle reproduces its run;
* synth: the written files read back to the model they were written from.
"""
import importlib
import os

import numpy as np
import pytest

from oracle import refrun
from oracle.refsrc import reference_file

gen = importlib.import_module("hpc-ca-phospattern_b200.generate")
h5m = importlib.import_module("hpc-ca-phospattern_b200.h5model")
G1 = reference_file("createdgeometries", "G1", "G1_nonP_0.h5")
MAP = reference_file("createdgeometries", "G1", "G1_inner_10.npy")
PHOS = reference_file("parameters", "phosphorylation", "parameters_sr1100_ryr55_pryr25.h5")
have_ref = bool(G1 and MAP and PHOS)


@pytest.mark.skipif(not have_ref, reason="reference input files absent")
def test_phospho_split_of_g1(tmp_path):
    out = str(tmp_path / "G1_inner_10.h5")
    n_ryr, n_p = gen.phospho(G1, MAP, out)
    assert (n_ryr, n_p) == (40, 10)
    src, new = h5m.read_geometry(G1), h5m.read_geometry(out)
    assert [b["name"] for b in new["boundaries"]] == ["serca", "ryr", "p_ryr", "sr_cleft"]
    np.testing.assert_array_equal(new["voxels"], src["voxels"])
    old = {b["name"]: np.asarray(b["pairs"]) for b in src["boundaries"]}
    nb = {b["name"]: np.asarray(b["pairs"]) for b in new["boundaries"]}
    for name in ("serca", "sr_cleft"):
        np.testing.assert_array_equal(nb[name], old[name])
    m = np.load(MAP)
    assert np.all(m[nb["ryr"][:, 0] + 42, nb["ryr"][:, 1] + 42] == 1)
    assert np.all(m[nb["p_ryr"][:, 0] + 42, nb["p_ryr"][:, 1] + 42] == 2)
    merged = np.concatenate([nb["ryr"], nb["p_ryr"]])
    assert sorted(map(tuple, merged)) == sorted(map(tuple, old["ryr"]))


@pytest.mark.skipif(not (have_ref and refrun.ref_binary()), reason="reference program or files absent")
def test_phospho_geometry_runs_in_reference_and_oracle(tmp_path):
    from oracle.oracle import Oracle
    geo = str(tmp_path / "G1_inner_10.h5")
    gen.phospho(G1, MAP, geo)
    opts = dict(h=12.0, tstop=1.2e-3, dt_save=6e-4, seed=1, open_states={"ryr": [0, 5], "p_ryr": [2]},
                t_close={"ryr": 1e-3, "p_ryr": 1e-3})
    res = refrun.run_files(geo, PHOS, opts, str(tmp_path), all_data=("Ca",), threads=8)
    spec = h5m.read_model(geo, PHOS)
    orc = Oracle(spec, opts)
    prev = 0
    pb = [b["name"] for b in spec["boundaries"]].index("p_ryr")
    for o in res["outputs"]:
        orc.step(o["time_index"] - prev)
        prev = o["time_index"]
        err = np.max(np.abs(o["fields"]["Ca"] - orc.state()[0])) / np.max(np.abs(o["fields"]["Ca"]))
        assert err < 1e-11, f"{o['name']}: {err:.2e}"
        assert len(o["discrete"]["p_ryr"]) == 10
        np.testing.assert_array_equal(orc.channels(pb), o["discrete"]["p_ryr"].astype(np.int32))


def test_synth_files_read_back(tmp_path):
    g, s = str(tmp_path / "g.h5"), str(tmp_path / "s.h5")
    assert gen.main(["synth", "3", g, s, "--index", "2"]) == 0
    spec, _ = gen.synth_config(3, 2)
    back = h5m.read_model(g, s)
    np.testing.assert_array_equal(back["voxels"], spec["voxels"])
    assert [b["name"] for b in back["boundaries"]] == [b["name"] for b in spec["boundaries"]]
    for a, b in zip(back["boundaries"], spec["boundaries"]):
        np.testing.assert_array_equal(np.asarray(a["pairs"]), np.asarray(b["pairs"]).reshape(-1, 6))
    assert back["species"] == spec["species"]


def test_h5lite_incremental_flushes(tmp_path):
    """A created file is written incrementally: a later flush appends the new datasets'
    data and rewrites only the metadata; everything reads back, attributes included."""
    p = str(tmp_path / "inc.h5")
    a = np.arange(200_000, dtype=np.float64)
    b = np.linspace(0.0, 1.0, 5000)
    with h5m.H5(p, "w") as f:
        f.put_group("/data_0000000")
        f.put_attr("/data_0000000", "time", np.array([0.5]))
        f.put_dset("/data_0000000/Ca_all_data", a)
        f.flush()
        s1 = os.path.getsize(p)
        f.put_group("/data_0000001")
        f.put_dset("/data_0000001/Ca_all_data", b)
        f.flush()
        s2 = os.path.getsize(p)
    assert s1 > a.nbytes
    assert 0 < s2 - s1 < b.nbytes + 8192, (s1, s2)
    with h5m.H5(p) as f:
        np.testing.assert_array_equal(f.dset("/data_0000000/Ca_all_data"), a)
        np.testing.assert_array_equal(f.dset("/data_0000001/Ca_all_data"), b)
        assert float(np.ravel(f.attr("/data_0000000", "time"))[0]) == 0.5
        assert sorted(n for _, n in f.list("/")) == ["data_0000000", "data_0000001"]


def test_h5lite_incremental_then_append(tmp_path):
    """A file written by incremental flushes, reopened for appending (whole rewrite),
    keeps every dataset and attribute."""
    p = str(tmp_path / "app.h5")
    a = np.arange(1000, dtype=np.float64)
    with h5m.H5(p, "w") as f:
        f.put_group("/g")
        f.put_dset("/g/a", a)
        f.flush()
        f.put_attr("/g", "n", np.array([7], dtype=np.int32))
    with h5m.H5(p, "a") as f:
        f.put_dset("/g/b", 2 * a)
    with h5m.H5(p) as f:
        np.testing.assert_array_equal(f.dset("/g/a"), a)
        np.testing.assert_array_equal(f.dset("/g/b"), 2 * a)
        assert int(np.ravel(f.attr("/g", "n"))[0]) == 7
