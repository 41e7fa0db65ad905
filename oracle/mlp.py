"""CPU restatement (FP64 numpy) of the reaction surrogate's mathematics.

TEST INFRASTRUCTURE ONLY: the checker of hpc-ca-phospattern_b200/csrc/csp_mlp.cuh.

* plain integrator: the reference's buffer reaction update (Species_step_reaction,
  species.c:1653-1702; kernel_generic.cpp:495-507: J = k_on (tot - b) Ca - k_off b,
  du[b] += dt J, du[Ca] -= dt J) applied n times at the step dt to one voxel, reaction only;
* the network: x[8] = [log10(Ca)/3, b_s/tot_s (s = 1..5), log10(dt_r)/4, domain/4],
  two ReLU layers of 64, outputs t_s; increment df_s = dt_r g_s/tot_s + S_s t_s with
  S_s = dt_r^2/2 (lambda_s |g_s| + k_on,s (tot_s - b_s) |sum_q g_q|) / tot_s,
  lambda_s = k_off,s + k_on,s Ca, and dCa = -sum_s tot_s df_s;
* acceptance: max_s |db_s - dt_r/2 (g_s(y0) + g_s(y1))| / tot_s <= tol;
* loss: mean squared error over samples and outputs, and its gradient.
Parameter layout: w1[8][64] b1[64] w2[64][64] b2[64] w3[64][5] b3[5].
"""
import numpy as np

NIN, NH, NOUT, NSLOT = 8, 64, 5, 5
NPARAM = NIN * NH + NH + NH * NH + NH + NH * NOUT + NOUT


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = []
    for shape in ((NIN, NH), (NH,), (NH, NH), (NH,), (NH, NOUT), (NOUT,)):
        n = int(np.prod(shape))
        out.append(p[o:o + n].reshape(shape))
        o += n
    return out


def forward(p, x):
    w1, b1, w2, b2, w3, b3 = unpack(p)
    h1 = np.maximum(x @ w1 + b1, 0.0)
    h2 = np.maximum(h1 @ w2 + b2, 0.0)
    return h2 @ w3 + b3, (h1, h2)


def loss_grad(p, x, t):
    """Mean squared error over samples and outputs, and its gradient (packed)."""
    x = np.asarray(x, dtype=np.float64)
    t = np.asarray(t, dtype=np.float64)
    w1, b1, w2, b2, w3, b3 = unpack(p)
    y, (h1, h2) = forward(p, x)
    n = x.shape[0]
    e = y - t
    scale = 1.0 / (n * NOUT)
    loss = float(np.sum(e * e) * scale)
    dy = 2.0 * e * scale
    gw3, gb3 = h2.T @ dy, dy.sum(0)
    d2 = (dy @ w3.T) * (h2 > 0)
    gw2, gb2 = h1.T @ d2, d2.sum(0)
    d1 = (d2 @ w2.T) * (h1 > 0)
    gw1, gb1 = x.T @ d1, d1.sum(0)
    return loss, np.concatenate([a.ravel() for a in (gw1, gb1, gw2, gb2, gw3, gb3)])


def constants(spec, d):
    """(kon, koff, tot) by slot (species 1..5) of domain d; zeros for absent slots."""
    ds = spec["domain_species"][spec["domains"][d]]
    kon, koff, tot = np.zeros(NSLOT), np.zeros(NSLOT), np.zeros(NSLOT)
    for bf in ds.get("buffers", []):
        s, lig = bf["species"]
        if lig != 0 or not 1 <= s <= NSLOT:
            raise ValueError("surrogate needs buffers bound to species 0 among species 1..5")
        kon[s - 1], koff[s - 1], tot[s - 1] = bf["k_on"], bf["k_off"], bf["tot"]
    return kon, koff, tot


def eligible(k, dtr, limit=0.25, ca_max=500.0):
    """Whether the network serves a domain with constants k at dt_r (not stiff)."""
    kon, koff, tot = k
    on = tot > 0
    if not on.any():
        return False
    return dtr * (np.sum(kon[on] * tot[on]) + np.max(koff[on] + ca_max * kon[on])) <= limit


def g(k, c, b):
    kon, koff, tot = k
    return np.where(tot > 0, kon * (tot - b) * c - koff * b, 0.0)


def plain(k, n, h, c, b):
    """n explicit reaction steps of h from (c, b); returns (dc, db)."""
    cc, bb = float(c), np.array(b, dtype=np.float64)
    for _ in range(n):
        gg = g(k, cc, bb)
        bb = bb + h * gg
        cc = cc - h * gg.sum()
    return cc - c, bb - np.asarray(b, dtype=np.float64)


def features(k, d, dtr, c, b):
    tot = k[2]
    x = np.zeros(NIN)
    x[0] = np.log10(max(c, 1e-3)) / 3.0
    x[1:6] = np.where(tot > 0, np.asarray(b) / np.where(tot > 0, tot, 1.0), 0.0)
    x[6] = np.log10(dtr) / 4.0
    x[7] = d / 4.0
    return x


def scale(k, dtr, c, b):
    kon, koff, tot = k
    gg = g(k, c, b)
    G = abs(gg.sum())
    lam = koff + kon * c
    return np.where(tot > 0, 0.5 * dtr * dtr * (lam * np.abs(gg) + kon * (tot - b) * G) / np.where(tot > 0, tot, 1.0),
                    0.0)


def increment(k, dtr, c, b, t):
    """(dc, db) of the network output t."""
    tot = k[2]
    b = np.asarray(b, dtype=np.float64)
    df = np.where(tot > 0, dtr * g(k, c, b) / np.where(tot > 0, tot, 1.0) + scale(k, dtr, c, b) * t, 0.0)
    db = tot * df
    return -db.sum(), db


def residual(k, dtr, c, b, dc, db):
    tot = k[2]
    g0, g1 = g(k, c, b), g(k, c + dc, np.asarray(b) + db)
    r = np.abs(db - 0.5 * dtr * (g0 + g1)) / np.where(tot > 0, tot, 1.0)
    return float(np.max(np.where(tot > 0, r, 0.0)))


def surrogate(p, k, d, dtr, c, b, tol):
    """(dc, db, accepted) of the network for one voxel, with the plain-integrator fallback
    left to the caller."""
    x = features(k, d, dtr, c, b)
    t, _ = forward(p, x[None, :])
    dc, db = increment(k, dtr, c, b, t[0])
    return dc, db, residual(k, dtr, c, b, dc, db) <= tol
