"""CPU checks of the FP64 oracle itself (no GPU).

The oracle is pinned to the reference program in test_oracle_pin.py; these tests check
its invariants and cross-check it against a second, loop-level restatement of the
reference step on a grid small enough for pure Python.
"""
import numpy as np
import pytest


def py_step(spec, state, info, open_by_boundary, time_ind, dt, h):
    """One reference step (species.c:1501-1702, 1704-1810, 1080-1121) in plain Python
    loops, FP64, on one rank; channels fixed (no gating); no Dirichlet / fixed values."""
    vox = spec["voxels"]
    nx, ny, nz = vox.shape
    doms = spec["domains"]
    nd = len(doms)
    ds = [spec["domain_species"][d] for d in doms]
    conn = np.asarray(spec["domain_connections"])
    u1 = state.copy()
    du = state.copy()
    update = set()
    max_sig = max(max(d.get("sigma", []) or [0]) for d in ds)
    diff_species = sorted({s for d in ds for s in d.get("diffusive", [])})
    for dsi, si in enumerate(diff_species):
        sub = info.substeps[dsi]
        if time_ind % sub:
            continue
        update.add(si)
        coef = np.zeros((5, 5))
        for di in range(nd):
            sa = ds[di].get("sigma", [])
            if not (dsi < len(sa) and sa[dsi] != 0):
                continue
            for dn in range(di):
                sb = ds[dn].get("sigma", [])
                if conn[di, dn] and dsi < len(sb) and sb[dsi] != 0:
                    coef[di, dn] = coef[dn, di] = dt * 0.5 * (sa[dsi] + sb[dsi]) / (h * h) * sub
            coef[di, di] = dt * sa[dsi] / (h * h) * sub
        for x in range(nx):
            for y in range(ny):
                for z in range(nz):
                    u = u1[si, x, y, z]
                    d = u
                    for (a, b, c) in ((0, 0, -1), (0, 0, 1), (0, -1, 0), (0, 1, 0), (-1, 0, 0), (1, 0, 0)):
                        xx, yy, zz = x + a, y + b, z + c
                        if 0 <= xx < nx and 0 <= yy < ny and 0 <= zz < nz:
                            d += coef[vox[x, y, z], vox[xx, yy, zz]] * (u1[si, xx, yy, zz] - u)
                    du[si, x, y, z] = d
    # boundary fluxes: RyR law only (the test models carry no SERCA)
    for bi, b in enumerate(spec["boundaries"]):
        if b["name"] not in ("ryr", "p_ryr"):
            continue
        p = spec[b["name"]]
        si = spec["species"].index(p["species"])
        update.add(si)
        K0 = np.exp(-2 * dt * 1e15 / (2 * 96485.) * p["i_unitary"] / (1300. - 0.1) / (h * h * h))
        for i, pr in enumerate(np.asarray(b["pairs"])):
            if not open_by_boundary[bi][i]:
                continue
            f, t = tuple(pr[:3]), tuple(pr[3:])
            J = (u1[si][f] - u1[si][t]) * (1 - K0) / 2
            du[si][t] += J
            du[si][f] -= J
    # reactions
    nbuf = len({b["species"][0] for d in ds for b in d.get("buffers", [])})
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                di = vox[x, y, z]
                bufs = ds[di].get("buffers", [])
                for bi in range(nbuf):
                    if bi < len(bufs):
                        bf = bufs[bi]
                        s0, s1, kon, koff, tot = bf["species"][0], bf["species"][1], bf["k_on"], bf["k_off"], bf["tot"]
                    else:
                        s0 = s1 = 0
                        kon = koff = tot = 0.0
                    b0, b1 = u1[s0, x, y, z], u1[s1, x, y, z]
                    J = kon * (tot - b0) * b1 - koff * b0
                    if s0 in update:
                        du[s0, x, y, z] += dt * J
                    else:
                        du[s0, x, y, z] = b0 + dt * J
                    if s1 in update:
                        du[s1, x, y, z] -= dt * J
                    else:
                        du[s1, x, y, z] = b1 - dt * J
    for di in range(nd):
        for bf in ds[di].get("buffers", [])[:nbuf]:
            update.add(bf["species"][0])
            update.add(bf["species"][1])
        if len(ds[di].get("buffers", [])) < nbuf:
            update.add(0)
    out = state.copy()
    for s in update:
        out[s] = du[s]
    return out


def test_oracle_matches_loop_restatement(synth, oracle_mod):
    spec = synth.tiny((6, 5, 7), serca=False, pryr=True)
    opts = dict(h=6.0, tstop=1.0, seed=1, open_states={"ryr": [0, 2], "p_ryr": [1]})
    orc = oracle_mod.Oracle(spec, opts)
    inf = orc.info()
    st = orc.state()
    rng = np.random.default_rng(1)
    st = st * (1 + 0.05 * rng.random(st.shape))       # leave equilibrium
    orc.set_state(st)
    opens = {0: orc.channels(0), 1: orc.channels(1)}
    for t in range(1, 13):
        st = py_step(spec, st, inf, opens, t, inf.dt, inf.h)
        orc.step(1)
    np.testing.assert_allclose(orc.state(), st, rtol=1e-12, atol=1e-12)


def test_oracle_equilibrium_and_conservation(synth, oracle_mod):
    spec = synth.spark_model((16, 16, 12), serca=False, patch_frac=0.5, margin=2, jsr_voxels=3,
                             channels=[(8, 8), (6, 8)])
    orc = oracle_mod.Oracle(spec, dict(h=6.0, tstop=1.0, open_states={"ryr": []}))
    u0 = orc.state()
    orc.step(50)
    np.testing.assert_allclose(orc.state(), u0, rtol=1e-12, atol=1e-12)
    orc2 = oracle_mod.Oracle(spec, dict(h=6.0, tstop=1.0, open_states={"ryr": [0, 1]}))
    tot0 = orc2.outputs()[2].sum()
    orc2.step(100)
    tot1 = orc2.outputs()[2].sum()
    assert abs(tot1 - tot0) / tot0 < 1e-12
    assert orc2.state()[0].max() > u0[0][spec["voxels"] == 1].max() * 10


def test_oracle_time_constants(synth, oracle_mod):
    spec = synth.tiny((12, 12, 16))
    orc = oracle_mod.Oracle(spec, dict(h=6.0, tstop=2.0))
    inf = orc.info()
    dt = 0.95 * 36 / (6 * 220000.0)
    assert inf.dt == pytest.approx(dt, rel=1e-15)
    # Ca and ATP every step, Fluo floor(220000/20000)=11, CMDN floor(220000/22000)=10
    assert list(inf.substeps)[:4] == [1, 11, 10, 1]
    n = 0
    t = 0.0
    while t < 2.0:
        t += dt
        n += 1
    assert inf.total_steps == n
    inf2 = oracle_mod.Oracle(spec, dict(h=6.0, dt_update_react=5 * dt, dt_update_stoch=2.5 * dt)).info()
    assert (inf2.reaction_substep, inf2.stochastic_substep) == (5, 2)
    # a 12 nm geometry at -h 5 has subdivisions floor(12/5) = 2 and h = 6
    spec12 = dict(spec, h=12.0)
    inf3 = oracle_mod.Oracle(spec12, dict(h=5.0)).info()
    assert inf3.subdivisions == 2 and inf3.h == 6.0 and list(inf3.n) == [24, 24, 32]


def test_oracle_forced_close_and_abort(synth, oracle_mod):
    spec = synth.tiny((12, 12, 16))
    dt = 0.95 * 36 / (6 * 220000.0)
    orc = oracle_mod.Oracle(spec, dict(h=6.0, tstop=5.0, open_states={"ryr": [0, 1], "p_ryr": [0]},
                                       t_close={"ryr": 20 * dt, "p_ryr": 20 * dt}, tabort=10 * dt))
    orc.step(10)
    assert orc.channels(0)[:2].tolist() == [1, 1]
    orc.step(200)
    assert orc.channels(0).sum() == 0 and orc.channels(1).sum() == 0
    assert orc.info().stopped == 1
    assert 25 < orc.info().step < 35


def test_philox_known_answer(oracle_mod):
    """Philox4x32-10 against the published known-answer vectors (Random123 kat_vectors)."""
    import ctypes
    # the oracle exposes it only through channel draws; restate the block function here
    def philox(ctr, key):
        c = list(ctr)
        k0, k1 = key
        for _ in range(10):
            p0 = 0xD2511F53 * c[0]
            p1 = 0xCD9E8D57 * c[2]
            c = [((p1 >> 32) ^ c[1] ^ k0) & 0xffffffff, p1 & 0xffffffff,
                 ((p0 >> 32) ^ c[3] ^ k1) & 0xffffffff, p0 & 0xffffffff]
            k0 = (k0 + 0x9E3779B9) & 0xffffffff
            k1 = (k1 + 0xBB67AE85) & 0xffffffff
        return c
    assert philox([0, 0, 0, 0], [0, 0]) == [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert philox([0xffffffff] * 4, [0xffffffff] * 2) == [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    _ = ctypes
