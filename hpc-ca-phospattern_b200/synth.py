"""Seeded synthetic calcium-spark inputs in the reference's model layout.

No input of the benchmark configurations exists in the reference repository, so these
builders make them: a box of cytosol with a junctional-SR patch, the dyadic cleft under
it, a network-SR sheet around it and a RyR / pRyR cluster on a 30 nm lattice between
jSR and cleft.  The species model is the reference's 5-domain, 5-species model
(parameters/phosphorylation/parameters_sr1100_ryr55_pryr25.h5: Ca, Fluo, CMDN/CSQN,
ATP, TRPN) with the concentrations of the benchmark configurations (Ca 0.14 uM cytosol /
1300 uM SR, CSQN 30 mM, D_SR = 60 um^2/s).  Buffers start at equilibrium with Ca.

A model description is a plain dict (see spark_model); abi.make_model turns it into the
C csp_model, h5model.write_model into the reference's HDF5 files.
"""
import numpy as np

DOMAINS = ["cyt", "cleft", "jsr", "nsr", "tt"]
SPECIES = ["Ca", "Fluo", "CMDN", "ATP", "TRPN"]
CYT, CLEFT, JSR, NSR, TT = range(5)

RYR = dict(Kd_open=55.0, k_min_open=5e-6, k_max_open=0.9, n_open=2.7,
           Kd_close=35.0, k_min_close=0.9, k_max_close=3.0, n_close=-0.5,
           i_unitary=0.235, boundary="ryr", species="Ca")
P_RYR = dict(RYR, Kd_open=25.0, boundary="p_ryr")
SERCA = dict(v_cyt_to_A_sr=307.0, density=0.013, scale=1.0, boundary="serca", species="Ca")


def _bound(tot, k_on, k_off, ca):
    return tot * ca / (ca + k_off / k_on)


def species_model(ca_cyt=0.14, ca_sr=1300.0, sigma_ca=220000.0, sigma_ca_sr=60000.0,
                  csqn_tot=30000.0, trpn_tot=70.0, fluo_tot=50.0):
    """Per-domain species tables (the /<domain> groups of the species file).

    Global diffusive order Ca, Fluo, CMDN, ATP; every domain lists a prefix of it, as
    the reference's coefficient tables require (species.c:1547-1560).
    """
    cyt_bufs = [dict(species=[1, 0], k_on=0.08, k_off=0.09, tot=fluo_tot),    # Fluo-4
                dict(species=[2, 0], k_on=0.034, k_off=0.238, tot=24.0),      # CMDN
                dict(species=[3, 0], k_on=0.255, k_off=45.0, tot=455.0),      # ATP
                dict(species=[4, 0], k_on=0.0327, k_off=0.0196, tot=trpn_tot)]  # TRPN
    cleft_bufs = [dict(b) for b in cyt_bufs]
    cleft_bufs[3]["tot"] = 47.0
    jsr_bufs = [dict(species=[1, 0], k_on=0.11, k_off=0.11, tot=2.5e-5),     # Fluo-5
                dict(species=[2, 0], k_on=0.102, k_off=65.0, tot=csqn_tot)]   # CSQN
    nsr_bufs = [dict(jsr_bufs[0])]

    def init(ca, bufs):
        v = [0.0] * len(SPECIES)
        v[0] = ca
        for b in bufs:
            v[b["species"][0]] = _bound(b["tot"], b["k_on"], b["k_off"], ca)
        return v

    cyt_sig = [sigma_ca, 20000.0, 22000.0, 140000.0]
    sr_sig = [sigma_ca_sr, 8000.0]
    return {
        "cyt": dict(diffusive=[0, 1, 2, 3], sigma=cyt_sig, init=init(ca_cyt, cyt_bufs), buffers=cyt_bufs),
        "cleft": dict(diffusive=[0, 1, 2, 3], sigma=cyt_sig, init=init(ca_cyt, cleft_bufs), buffers=cleft_bufs),
        "jsr": dict(diffusive=[0, 1], sigma=sr_sig, init=init(ca_sr, jsr_bufs), buffers=jsr_bufs),
        "nsr": dict(diffusive=[0, 1], sigma=sr_sig, init=init(ca_sr, nsr_bufs), buffers=nsr_bufs),
        "tt": dict(diffusive=[], sigma=[], init=[0.0] * len(SPECIES), buffers=[]),
    }


def connections():
    c = np.eye(len(DOMAINS), dtype=np.uint8)
    c[CYT, CLEFT] = c[CLEFT, CYT] = 1
    c[JSR, NSR] = c[NSR, JSR] = 1
    return c


def _adjacent_pairs(vox, a, b):
    """All face-adjacent voxel pairs (from in domain a, to in domain b), [n][6]."""
    out = []
    for axis in range(3):
        sl0 = [slice(None)] * 3
        sl1 = [slice(None)] * 3
        for sign in (1, -1):
            if sign == 1:
                sl0[axis] = slice(0, -1); sl1[axis] = slice(1, None)
            else:
                sl0[axis] = slice(1, None); sl1[axis] = slice(0, -1)
            m = (vox[tuple(sl0)] == a) & (vox[tuple(sl1)] == b)
            idx = np.argwhere(m)
            if idx.size == 0:
                continue
            frm = idx.copy()
            to = idx.copy()
            if sign == 1:
                to[:, axis] += 1
            else:
                frm[:, axis] += 1
            out.append(np.concatenate([frm, to], axis=1))
    if not out:
        return np.zeros((0, 6), dtype=np.uint16)
    p = np.concatenate(out).astype(np.uint16)
    order = np.lexsort((p[:, 5], p[:, 4], p[:, 3], p[:, 2], p[:, 1], p[:, 0]))
    return p[order]


def spark_model(shape=(100, 100, 50), h=6.0, channels=None, pryr_mask=None, serca=True,
                cleft_voxels=2, jsr_voxels=5, patch_frac=0.6, margin=5, **species_kw):
    """A calcium-spark geometry + species model.

    channels: (n, 2) lattice positions (x, y) of the RyR/pRyR cluster, in voxels;
    default a centred 5x5 lattice at 5-voxel (30 nm at 6 nm) pitch.
    pryr_mask: bool (n,) -- which channels are phosphorylated (boundary p_ryr).
    """
    nx, ny, nz = shape
    vox = np.full(shape, CYT, dtype=np.uint8)
    zc = nz // 2 - cleft_voxels           # cleft below the SR sheet
    zj = zc + cleft_voxels                # first jSR / nSR plane
    zt = min(nz, zj + jsr_voxels)
    px = max(2, int(round(nx * patch_frac)) // 2 * 2)
    py = max(2, int(round(ny * patch_frac)) // 2 * 2)
    x0, y0 = (nx - px) // 2, (ny - py) // 2
    if serca:
        vox[margin:nx - margin, margin:ny - margin, zj:zt] = NSR
    vox[x0:x0 + px, y0:y0 + py, zj:zt] = JSR
    vox[x0:x0 + px, y0:y0 + py, zc:zj] = CLEFT
    if channels is None:
        g = np.arange(5) * 5 - 10
        channels = np.array([(nx // 2 + a, ny // 2 + b) for a in g for b in g])
    channels = np.asarray(channels, dtype=np.int64).reshape(-1, 2)
    if pryr_mask is None:
        pryr_mask = np.zeros(len(channels), dtype=bool)
    pryr_mask = np.asarray(pryr_mask, dtype=bool)

    def chan_pairs(sel):
        c = channels[sel]
        p = np.zeros((len(c), 6), dtype=np.uint16)
        p[:, 0] = c[:, 0]; p[:, 1] = c[:, 1]; p[:, 2] = zj          # jSR voxel
        p[:, 3] = c[:, 0]; p[:, 4] = c[:, 1]; p[:, 5] = zj - 1      # cleft voxel
        return p

    boundaries = [dict(name="ryr", type="discrete", pairs=chan_pairs(~pryr_mask))]
    spec = dict(h=h, voxels=vox, domains=list(DOMAINS), domain_connections=connections(),
                species=list(SPECIES), domain_species=species_model(**species_kw),
                ryr=dict(RYR), fixed_domain_species=[])
    if pryr_mask.any():
        boundaries.append(dict(name="p_ryr", type="discrete", pairs=chan_pairs(pryr_mask)))
        spec["p_ryr"] = dict(P_RYR)
    if serca:
        boundaries.append(dict(name="serca", type="density", pairs=_adjacent_pairs(vox, CYT, NSR)))
        spec["serca"] = dict(SERCA)
    spec["boundaries"] = boundaries
    spec["global_size"] = [s * h for s in shape]
    spec["layout"] = dict(cleft_z=(zc, zj), sr_z=(zj, zt), patch=(x0, y0, px, py))
    return spec


def lattice_cluster(rng, n_channels, shape, pitch=5, kind="compact", patch=(20, 20, 60, 60)):
    """n lattice positions inside the jSR patch: compact, elongated or fragmented."""
    x0, y0, px, py = patch
    gx = np.arange(x0 + pitch // 2, x0 + px, pitch)
    gy = np.arange(y0 + pitch // 2, y0 + py, pitch)
    pts = np.array([(a, b) for a in gx for b in gy], dtype=np.float64)
    cx, cy = pts.mean(axis=0)
    if kind == "compact":
        d = (pts[:, 0] - cx) ** 2 + (pts[:, 1] - cy) ** 2
    elif kind == "elongated":
        ang = rng.uniform(0, np.pi)
        u = (pts[:, 0] - cx) * np.cos(ang) + (pts[:, 1] - cy) * np.sin(ang)
        v = -(pts[:, 0] - cx) * np.sin(ang) + (pts[:, 1] - cy) * np.cos(ang)
        d = (u / 3.0) ** 2 + v ** 2
    else:  # fragmented into 2-4 sub-clusters
        k = int(rng.integers(2, 5))
        centres = pts[rng.choice(len(pts), size=k, replace=False)]
        d = np.min(((pts[:, None, :] - centres[None]) ** 2).sum(-1), axis=1)
    d = d + rng.uniform(0, 1e-3, size=len(d))
    sel = np.argsort(d)[:min(n_channels, len(pts))]
    return pts[sel].astype(np.int64)


def config1():
    """Plain FP64 configuration: 100x100x50 at 6 nm, 5x5 RyR cluster, RyR 0 forced open."""
    spec = spark_model((100, 100, 50), serca=True)
    opts = dict(h=6.0, tstop=2.0, seed=1, open_states={"ryr": [0]})
    return spec, opts


def config2(seed=2):
    """200x200x100 at 6 nm; 10x10 lattice with 10 % vacancies, 20 % pRyR; dt_update_stoch = dt."""
    rng = np.random.default_rng(seed)
    g = np.arange(10) * 5 - 22
    pts = np.array([(100 + a, 100 + b) for a in g for b in g])
    keep = rng.random(len(pts)) >= 0.10
    pts = pts[keep]
    pmask = np.zeros(len(pts), dtype=bool)
    pmask[rng.choice(len(pts), size=int(round(0.2 * len(pts))), replace=False)] = True
    spec = spark_model((200, 200, 100), channels=pts, pryr_mask=pmask, serca=True)
    opts = dict(h=6.0, tstop=10.0, seed=seed, open_states={"ryr": [0]})
    return spec, opts


def config3_draws(n=256, seed=3, shape=(100, 100, 50)):
    """The random draws of config3 for every realisation (cheap: no geometry is built):
    cluster channel positions, pRyR mask and options, in the order config3 draws them."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(n):
        nch = int(rng.integers(16, 101))
        kind = ["compact", "elongated", "fragmented"][int(rng.integers(0, 3))]
        nx, ny, nz = shape
        px, py = int(round(nx * 0.6)) // 2 * 2, int(round(ny * 0.6)) // 2 * 2
        patch = ((nx - px) // 2, (ny - py) // 2, px, py)
        pts = lattice_cluster(rng, nch, shape, kind=kind, patch=patch)
        pfrac = rng.uniform(0.0, 0.5)
        pmask = rng.random(len(pts)) < pfrac
        pmask[0] = False                  # channel 0 of "ryr" is the forced-open trigger
        out.append(dict(shape=shape, h=6.0, channels=pts, pryr_mask=pmask,
                        opts=dict(h=6.0, tstop=10.0, seed=seed * 1000003 + r, tabort=1.5, open_states={"ryr": [0]})))
    return out


def config3(n=256, seed=3, shape=(100, 100, 50), only=None):
    """Batched ensemble: n realisations of 100x100x50, 16-100 RyRs, pRyR 0-50 %,
    compact / elongated / fragmented clusters drawn from the seed, abort 1.5 ms after
    all channels close.  only: build just these realisation indices (the draws of all n
    are still taken, so realisation i is the same whichever others are built)."""
    draws = config3_draws(n, seed, shape)
    idx = range(n) if only is None else only
    specs = [spark_model(shape, channels=draws[i]["channels"], pryr_mask=draws[i]["pryr_mask"], serca=True)
             for i in idx]
    return specs, [dict(draws[i]["opts"]) for i in idx]


def config4_draws(n=64, seed=4):
    """The random draws of config4 for every realisation (no geometry built): grid shape,
    resolution h and options."""
    rng = np.random.default_rng(seed)
    out = []
    for r in range(n):
        nx = int(rng.integers(64, 257)) // 2 * 2
        ny = int(rng.integers(64, 257)) // 2 * 2
        nz = int(rng.integers(64, 129)) // 2 * 2
        h = float(rng.uniform(6.0, 10.0))
        dt = 0.95 * h * h / (6 * 220000.0)
        out.append(dict(shape=(nx, ny, nz), h=h, opts=dict(h=h, tstop=10.0, seed=seed * 1000003 + r,
                                                              dt_update_react=5 * dt, open_states={"ryr": [0]})))
    return out


def config4(n=64, seed=4, only=None):
    """Uneven ensemble: grids from 64^3 to 256x256x128 at h = 6-10 nm, -T 5*dt."""
    draws = config4_draws(n, seed)
    idx = range(n) if only is None else only
    specs = [spark_model(draws[i]["shape"], h=draws[i]["h"], serca=True) for i in idx]
    return specs, [dict(draws[i]["opts"]) for i in idx]


def tiny(shape=(12, 12, 16), serca=True, pryr=True, **kw):
    """A small spark geometry for parity tests (runs in milliseconds on the oracle)."""
    nx, ny, nz = shape
    g = np.array([-2, 0, 2])
    pts = np.array([(nx // 2 + a, ny // 2 + b) for a in g for b in g])
    pmask = np.zeros(len(pts), dtype=bool)
    if pryr:
        pmask[[2, 5]] = True
    return spark_model(shape, channels=pts, pryr_mask=pmask, serca=serca, patch_frac=0.6,
                       margin=1, jsr_voxels=3, **kw)
