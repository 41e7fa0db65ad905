"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle.

Every case runs the same model and options through libcsparks_cuda.so and through the
oracle, and compares every species field (per-species relative error <= 1e-4, the FP32
accuracy bar), the channel states (bit-exact) and the output reductions.
"""
import numpy as np
import pytest

from parity import RTOL, assert_close, species_rel_err

pytestmark = pytest.mark.gpu

KERNELS = [0, 1]   # 0 = TMA-staged, 1 = direct


def run_pair(pkg, oracle_mod, spec, opts, nsteps, kernel=1, chunks=1):
    sim = pkg.Simulation(spec, opts)
    sim.set_kernel(kernel)
    orc = oracle_mod.Oracle(spec, opts)
    per = nsteps // chunks
    for _ in range(chunks):
        sim.advance(per)
        orc.step(per)
    return sim, orc


def discrete_boundaries(spec):
    return [i for i, b in enumerate(spec["boundaries"]) if b["type"] == "discrete"]


def check_channels(sim, orc, spec, r=0):
    for b in discrete_boundaries(spec):
        np.testing.assert_array_equal(sim.channels(b, r), orc.channels(b))


@pytest.mark.parametrize("kernel", KERNELS)
def test_forced_channels_parity(pkg, oracle_mod, synth, kernel):
    spec = synth.tiny((12, 12, 16))
    opts = dict(h=6.0, tstop=5.0, seed=1, open_states={"ryr": [0, 3], "p_ryr": [1]},
                t_close={"ryr": 0.004, "p_ryr": 0.006})
    sim, orc = run_pair(pkg, oracle_mod, spec, opts, 400, kernel, chunks=4)
    assert sim.info().step == orc.info().step == 400
    assert_close(sim.state(), orc.state(), what="forced")
    check_channels(sim, orc, spec)


@pytest.mark.parametrize("kernel", KERNELS)
def test_stochastic_parity(pkg, oracle_mod, synth, kernel):
    """Same Philox draws on both sides: identical channel trajectories."""
    spec = synth.tiny((12, 12, 16))
    opts = dict(h=6.0, tstop=5.0, seed=7, open_states={"ryr": [0]})
    sim = pkg.Simulation(spec, opts)
    sim.set_kernel(kernel)
    orc = oracle_mod.Oracle(spec, opts)
    for _ in range(10):
        sim.advance(50)
        orc.step(50)
        check_channels(sim, orc, spec)
    assert_close(sim.state(), orc.state(), what="stochastic")


def test_kernels_bitwise_equal(pkg, synth):
    spec = synth.tiny((20, 18, 24))
    opts = dict(h=6.0, tstop=5.0, seed=3, open_states={"ryr": [0, 1, 2]})
    a = pkg.Simulation(spec, opts)
    b = pkg.Simulation(spec, opts)
    a.set_kernel(0)
    b.set_kernel(1)
    a.advance(137)
    b.advance(137)
    np.testing.assert_array_equal(a.state(), b.state())


def test_batched_equals_single(pkg, oracle_mod, synth):
    rng = np.random.default_rng(5)
    specs = []
    for k, shape in enumerate([(12, 12, 16), (16, 10, 12), (10, 14, 20)]):
        specs.append(synth.tiny(shape, pryr=(k != 1)))
    opts = [dict(h=6.0, tstop=5.0, seed=11, open_states={"ryr": [k]}) for k in range(3)]
    batch = pkg.Simulation(specs, opts)
    batch.advance(120)
    for r in range(3):
        single = pkg.Simulation(specs[r], opts[r])
        single.advance(120)
        orc = oracle_mod.Oracle(specs[r], opts[r], realisation=r)
        orc.step(120)
        # realisation r of the batch draws the Philox stream of index r
        np.testing.assert_array_equal(batch.channels(0, r), orc.channels(0))
        assert_close(batch.state(r), orc.state(), what=f"batch r={r}")
        if r == 0:
            np.testing.assert_array_equal(batch.state(0), single.state(0))
    _ = rng


@pytest.mark.parametrize("kernel", KERNELS)
def test_subdivisions(pkg, oracle_mod, synth, kernel):
    """Geometry at 12 nm simulated at 6 nm: every geometry voxel becomes 2^3 voxels;
    density pairs expand to 4 pairs, discrete ones sit at the sub-voxel centre."""
    spec = synth.tiny((8, 8, 10))
    spec["h"] = 12.0
    opts = dict(h=6.0, tstop=5.0, seed=2, open_states={"ryr": [0, 2], "p_ryr": [0]})
    sim, orc = run_pair(pkg, oracle_mod, spec, opts, 200, kernel)
    assert sim.info().subdivisions == 2
    assert_close(sim.state(), orc.state(), what="subdivisions")


@pytest.mark.parametrize("kernel", KERNELS)
def test_dirichlet_fixed_and_substeps(pkg, oracle_mod, synth, kernel):
    spec = synth.tiny((12, 12, 16))
    spec["fixed_domain_species"] = [(3, 0)]          # nsr Ca fixed
    dt = 0.95 * 36 / (6 * 220000.0)
    opts = dict(h=6.0, tstop=5.0, seed=4, force_dirichlet=True, dt_update_react=3.5 * dt,
                dt_update_stoch=2 * dt, open_states={"ryr": [1, 4]}, t_close={"ryr": 0.003})
    sim, orc = run_pair(pkg, oracle_mod, spec, opts, 300, kernel, chunks=3)
    inf = sim.info()
    assert inf.reaction_substep == 3 and inf.stochastic_substep == 2
    assert_close(sim.state(), orc.state(), what="dirichlet/fixed/substeps")
    check_channels(sim, orc, spec)


def test_forced_dt_and_odd_sizes(pkg, oracle_mod, synth):
    """-d forcing the time step, a grid with planes that are not multiples of 4 and a
    z extent of 9 (below the reference's vector width + 1)."""
    spec = synth.tiny((9, 11, 9), serca=False)
    opts = dict(h=6.0, dt=2e-5, tstop=1.0, seed=9, open_states={"ryr": [4]})
    sim, orc = run_pair(pkg, oracle_mod, spec, opts, 250, 1)
    assert abs(sim.info().dt - 2e-5) < 1e-20
    assert_close(sim.state(), orc.state(), what="odd sizes")
    sim0, _ = run_pair(pkg, oracle_mod, spec, opts, 250, 0)
    np.testing.assert_array_equal(sim0.state(), sim.state())


def test_outputs_match_oracle(pkg, oracle_mod, synth):
    spec = synth.tiny((12, 12, 16))
    opts = dict(h=6.0, tstop=5.0, seed=1, open_states={"ryr": [0]})
    sim, orc = run_pair(pkg, oracle_mod, spec, opts, 100)
    mn, mx, tot, op = sim.outputs()
    omn, omx, otot = orc.outputs()
    present = [d for d in range(len(spec["domains"])) if np.any(spec["voxels"] == d)]
    for d in present:
        np.testing.assert_allclose(mn[d], omn[d], rtol=RTOL, atol=1e-9)
        np.testing.assert_allclose(mx[d], omx[d], rtol=RTOL, atol=1e-9)
        np.testing.assert_allclose(tot[d], otot[d], rtol=RTOL, atol=1e-6)
    # an empty domain keeps the reference's FLT_MAX / FLT_MIN initial values
    tt = spec["domains"].index("tt")
    assert mn[tt, 0] == np.float32(3.4028235e38) and mx[tt, 0] == np.float32(1.1754944e-38)
    assert list(op) == list(np.concatenate([orc.channels(b) for b in discrete_boundaries(spec)]))


def test_abort_rule(pkg, oracle_mod, synth):
    """All channels forced closed at t_close; the run stops tabort ms later."""
    spec = synth.tiny((12, 12, 16))
    dt = 0.95 * 36 / (6 * 220000.0)
    opts = dict(h=6.0, tstop=5.0, seed=1, open_states={"ryr": [0], "p_ryr": []},
                t_close={"ryr": 50 * dt, "p_ryr": 50 * dt}, tabort=30 * dt)
    sim = pkg.Simulation(spec, opts)
    orc = oracle_mod.Oracle(spec, opts)
    flags = sim.advance(200)
    orc.step(200)
    assert flags[0] == 1
    assert sim.info().step == orc.info().step
    assert 70 < sim.info().step < 90
    assert_close(sim.state(), orc.state(), what="abort")


def test_state_roundtrip_and_channels(pkg, synth):
    spec = synth.tiny((12, 12, 16))
    sim = pkg.Simulation(spec, dict(h=6.0, tstop=1.0, seed=1))
    u = sim.state()
    rng = np.random.default_rng(0)
    v = u * (1 + 0.01 * rng.standard_normal(u.shape))
    sim.set_state(v)
    # the device keeps each value as an FP32 deviation from its domain's base: one FP32
    # rounding of the deviation, so within FP32 precision of the value
    np.testing.assert_allclose(sim.state(), v, rtol=2.0 ** -22, atol=0)
    st = np.array([1, 0, 1, 1, 0, 0, 1], dtype=np.int32)
    sim.set_channels(0, st)
    np.testing.assert_array_equal(sim.channels(0), st)


def test_errors_are_codes_not_aborts(pkg, synth):
    spec = synth.tiny((12, 12, 16))
    with pytest.raises(pkg.CspError) as e:
        pkg.Simulation(spec, dict(h=6.0, open_states={"ryr": [99]}))
    assert e.value.code == -4
    import copy
    bad = copy.deepcopy(spec)
    bad["domain_species"]["cyt"]["buffers"][0]["species"] = [7, 0]   # no species 7
    with pytest.raises(pkg.CspError) as e:
        pkg.Simulation(bad, dict(h=6.0))
    assert e.value.code == -1
    bad = copy.deepcopy(spec)
    bad["voxels"] = bad["voxels"].copy()
    bad["voxels"][0, 0, 0] = 6                                        # domain id >= num_domains
    with pytest.raises(pkg.CspError) as e:
        pkg.Simulation(bad, dict(h=6.0))
    assert e.value.code == -1
    sim = pkg.Simulation(spec, dict(h=6.0, tstop=1.0))
    with pytest.raises(pkg.CspError):
        sim.state(3)
    with pytest.raises(pkg.CspError):
        sim.channels(2)   # serca is a density boundary


def test_equilibrium_is_steady_full_size(pkg, synth):
    """Config-3-sized realisation with every channel closed and no SERCA: the initial
    state is the buffer equilibrium, so it must stay (up to FP32 rounding)."""
    spec = synth.spark_model((100, 100, 50), serca=False)
    sim = pkg.Simulation(spec, dict(h=6.0, tstop=10.0, seed=1, open_states={"ryr": []},
                                    t_close={"ryr": 1e-9}))
    u0 = sim.state()
    sim.advance(64)
    u1 = sim.state()
    err = species_rel_err(u1, u0)
    assert np.all(err < 1e-5), err


def test_mass_conservation_full_size(pkg, synth):
    """Closed system (no SERCA, channels open only between jSR and cleft): total calcium,
    free plus bound, is conserved; the FP64 sums must agree to FP32 precision."""
    spec = synth.spark_model((100, 100, 50), serca=False)
    sim = pkg.Simulation(spec, dict(h=6.0, tstop=10.0, seed=1, open_states={"ryr": list(range(25))}))

    def total_ca():
        _, _, tot, _ = sim.outputs()
        return tot.sum()  # Ca + every bound form: each buffer binds one Ca

    t0 = total_ca()
    sim.advance(200)
    t1 = total_ca()
    assert abs(t1 - t0) / t0 < 2e-5, (t0, t1)
    u = sim.state()
    assert np.all(np.isfinite(u))
    # the cleft under open channels is far above rest
    lay = spec["layout"]
    assert u[0, 50, 50, lay["cleft_z"][1] - 1] > 10.0


def rotate_spec(spec, order):
    """The same model with the physical axes permuted (voxels and boundary pairs)."""
    import copy
    out = copy.copy(spec)
    out["voxels"] = np.ascontiguousarray(np.transpose(spec["voxels"], order))
    bl = []
    for b in spec["boundaries"]:
        p = np.asarray(b["pairs"])
        q = p[:, [order[0], order[1], order[2], 3 + order[0], 3 + order[1], 3 + order[2]]]
        bl.append(dict(b, pairs=np.ascontiguousarray(q)))
    out["boundaries"] = bl
    return out


@pytest.mark.parametrize("order", [(2, 0, 1), (1, 2, 0), (0, 2, 1)])
@pytest.mark.parametrize("kernel", KERNELS)
def test_axis_orders(pkg, oracle_mod, synth, order, kernel):
    """Domain sheets perpendicular to each physical axis: the device axis order chosen
    from the geometry changes, the fields (in the reference's x,y,z order) do not."""
    spec = rotate_spec(synth.tiny((12, 10, 16)), order)
    opts = dict(h=6.0, tstop=5.0, seed=5, open_states={"ryr": [0, 4], "p_ryr": [1]})
    sim, orc = run_pair(pkg, oracle_mod, spec, opts, 150, kernel)
    assert_close(sim.state(), orc.state(), what=f"axes {order}")
    check_channels(sim, orc, spec)


def test_density_pair_bookkeeping(pkg, synth):
    """Every boundary pair is handled exactly once: channel voxels (and density pairs not
    evaluated inside the voxel kernels) are rows of the boundary kernel."""
    spec = synth.tiny((12, 12, 16))
    sim = pkg.Simulation(spec, dict(h=6.0, tstop=1.0, seed=1))
    inf = sim.info()
    nserca = len(spec["boundaries"][[b["name"] for b in spec["boundaries"]].index("serca")]["pairs"])
    nch = sum(len(b["pairs"]) for b in spec["boundaries"] if b["type"] == "discrete")
    assert 0 <= inf.fused_pairs <= nserca
    unfused = nserca - inf.fused_pairs
    assert 2 * nch <= inf.flux_rows <= 2 * nch + 2 * unfused
    if inf.fused_pairs == 0:
        assert inf.flux_rows > nserca


def test_autotune_keeps_fields_bitwise(pkg, synth):
    """The autotuner only changes the staged kernel's tiling: fields stay bitwise equal."""
    specs = [synth.tiny((16, 14, 20)), synth.tiny((12, 12, 16))]
    opts = [dict(h=6.0, tstop=5.0, seed=3, open_states={"ryr": [0, 2]}, t_close={"ryr": 5.0})] * 2
    a = pkg.Simulation(specs, opts)
    b = pkg.Simulation(specs, opts)
    a.advance(30)
    b.advance(30)
    rep = b.autotune(repeats=2)
    assert rep["chosen"]["ms"] > 0 and len(rep["candidates"]) >= 4
    a.advance(50)
    b.advance(50)
    for r in range(2):
        np.testing.assert_array_equal(a.state(r), b.state(r))


def test_uneven_ensemble_matches_oracle(pkg, oracle_mod, synth):
    """Config 4 in small: different shapes and resolutions (so different dt and step
    counts) in one batch, dt_update_react = 5 dt; every realisation against its own oracle,
    run to its own last step."""
    cases = [((14, 12, 18), 6.0), ((10, 16, 12), 8.5), ((12, 10, 14), 10.0)]
    specs, opts = [], []
    for k, (shape, h) in enumerate(cases):
        spec = synth.tiny(shape, pryr=(k != 1))
        spec["h"] = h
        dt = 0.95 * h * h / (6 * 220000.0)
        specs.append(spec)
        opts.append(dict(h=h, tstop=0.004, seed=21, dt_update_react=5 * dt, open_states={"ryr": [k]},
                         t_close={"ryr": 0.003}))
    sim = pkg.Simulation(specs, opts)
    totals = [sim.info(r).total_steps for r in range(3)]
    assert len(set(totals)) == 3, totals
    flags = sim.advance(max(totals) + 10)
    assert all(flags)
    for r in range(3):
        assert sim.info(r).step == totals[r]
        orc = oracle_mod.Oracle(specs[r], opts[r], realisation=r)
        orc.step(totals[r])
        assert_close(sim.state(r), orc.state(), what=f"uneven r={r}")
        np.testing.assert_array_equal(sim.channels(0, r), orc.channels(0))


def test_async_advance_and_snapshot(pkg, synth):
    """csp_advance_async / _wait give the fields of csp_advance; a snapshot started before
    an asynchronous advance holds the fields from before it (the conversion is ordered
    before the steps, the copy overlaps them); the species mask is honoured; misuse is an
    error code."""
    spec = synth.tiny((12, 12, 16))
    opts = dict(h=6.0, tstop=5.0, seed=3, open_states={"ryr": [0, 2]})
    a = pkg.Simulation(spec, opts)
    b = pkg.Simulation(spec, opts)
    a.advance(40)
    b.advance_async(40)
    b.advance_wait()
    np.testing.assert_array_equal(a.state(), b.state())
    u40 = b.state()
    b.snapshot_async()
    b.advance_async(30)
    snap = b.snapshot_wait()
    b.advance_wait()
    np.testing.assert_array_equal(snap, u40)
    a.advance(30)
    u70 = a.state()
    np.testing.assert_array_equal(u70, b.state())
    b.snapshot_async(species_mask=0b101)
    part = b.snapshot_wait()
    np.testing.assert_array_equal(part[[0, 2]], u70[[0, 2]])
    b.advance_async(1)
    with pytest.raises(pkg.CspError):
        b.advance(1)
    b.advance_wait()
    with pytest.raises(pkg.CspError):
        b.advance_wait()
    with pytest.raises(pkg.CspError):
        b.snapshot_wait()
    a.advance(1)
    np.testing.assert_array_equal(a.state(), b.state())


def test_batched_state_transfers(pkg, synth):
    """csp_upload_states / csp_download_states equal the per-realisation calls."""
    specs = [synth.tiny((12, 12, 16)), synth.tiny((10, 14, 12))]
    opts = [dict(h=6.0, tstop=5.0, seed=5, open_states={"ryr": [0]})] * 2
    a = pkg.Simulation(specs, opts)
    a.advance(20)
    u = [a.state(r) for r in range(2)]
    rng = np.random.default_rng(3)
    new = [np.ascontiguousarray(x * (1.0 + 0.01 * rng.random(x.shape))) for x in u]
    a.set_states(new)
    got = [np.empty_like(x) for x in u]
    a.states_into(got)
    for r in range(2):
        np.testing.assert_array_equal(got[r], a.state(r))
        np.testing.assert_allclose(got[r], new[r], rtol=2.0 ** -22, atol=0)


def test_fp32_transfers_and_pipelined_run(pkg, synth):
    """csp_upload_states_f32 / csp_download_states_f32 move the FP64 calls' values;
    csp_run_states (upload, nsteps steps, download, pipelined by realisation groups) gives
    bitwise the fields, channel states and step counts of upload + csp_advance + download,
    with FP32 and FP64 host arrays, for more realisations than groups and uneven sizes; its
    per-step stop flags show each realisation stopping at its own last step."""
    shapes = [(12, 12, 16), (10, 14, 12), (14, 10, 12), (12, 12, 20), (10, 10, 16), (16, 12, 12), (12, 14, 14),
              (10, 12, 18), (12, 10, 16), (14, 12, 10), (10, 16, 12)]
    specs = [synth.tiny(s, pryr=(k % 3 != 1)) for k, s in enumerate(shapes)]
    dt = 0.95 * 36 / (6 * 220000.0)
    opts = [dict(h=6.0, tstop=(20 + 2 * k) * dt, seed=17, open_states={"ryr": [k % 7]}) for k in range(len(shapes))]
    a = pkg.Simulation(specs, opts)
    b = pkg.Simulation(specs, opts)
    a.advance(5)
    b.advance(5)
    u64 = [a.state(r) for r in range(a.n)]
    u32 = [np.ascontiguousarray(x.astype(np.float32)) for x in u64]
    got = [np.empty_like(x) for x in u32]
    a.set_states_f32(u32)
    a.states_into_f32(got)
    for r in range(a.n):
        # an FP32 download is the FP64 download rounded; both within FP32 precision of the input
        np.testing.assert_array_equal(got[r], a.state(r).astype(np.float32))
        np.testing.assert_allclose(got[r], u32[r], rtol=2.0 ** -22, atol=0)
    # reference sequence on a: FP64 upload, 40 steps, download
    a.set_states(u64)
    fa = a.advance(40)
    ref = [a.state(r) for r in range(a.n)]
    out = [np.zeros_like(x) for x in u64]
    fb, sf = b.run_states(u64, 40, out, step_flags=True)
    np.testing.assert_array_equal(fa, fb)
    for r in range(a.n):
        np.testing.assert_array_equal(out[r], ref[r])
        assert b.info(r).step == a.info(r).step
        np.testing.assert_array_equal(b.channels(0, r), a.channels(0, r))
        last = b.info(r).total_steps
        col = sf[:, r]
        assert col[-1] == 1 and np.all(col[: last - 5 - 1] == 0) and np.all(col[last - 5 - 1:] == 1)
    # FP32 host arrays, output aliasing input, against FP32 upload + csp_advance
    c = pkg.Simulation(specs, opts)
    d = pkg.Simulation(specs, opts)
    c.advance(5)
    d.advance(5)
    d.set_states_f32(u32)
    d.advance(40)
    buf = [x.copy() for x in u32]
    c.run_states(buf, 40, buf)
    for r in range(c.n):
        np.testing.assert_array_equal(buf[r], d.state(r).astype(np.float32))
