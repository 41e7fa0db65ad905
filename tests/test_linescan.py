"""csp_linescan against the reference's linescan sum evaluated directly.

The reference (Species_compute_convolution_with_gaussian_function_locally,
species.c:1960-2037, gauss utils.c:209-213) sums, for every index a of the scanned axis,
u * g(o_x - x h) g(o_y - y h) g(o_z - z h) over all species voxels with o_axis = a h; with
domains given on the command line it keeps voxels whose domain id is below their count.
Here that sum is evaluated term by term in numpy (FP64) on the library's own FP32 state,
so the check isolates the device reduction: relative error <= 1e-10.
"""
import numpy as np
import pytest


def gauss(x, s):
    return 1.0 / np.sqrt(2 * np.pi * s) * np.exp(-x * x / 2.0 / s)


def direct(u, dom, h, axis, offsets, conv, num_domains):
    n = u.shape
    coords = [np.arange(n[a]) * h for a in range(3)]
    keep = np.ones(n, bool) if num_domains == 0 else dom < num_domains
    out = np.zeros(n[axis])
    for a in range(n[axis]):
        w = []
        for ax in range(3):
            o = a * h if ax == axis else offsets[ax]
            w.append(gauss(o - coords[ax], conv[ax]))
        W = w[0][:, None, None] * w[1][None, :, None] * w[2][None, None, :]
        out[a] = np.sum(np.where(keep, u * W, 0.0))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("axis,num_domains", [(0, 0), (1, 2), (2, 0)])
def test_linescan_matches_direct_sum(pkg, synth, axis, num_domains):
    spec = synth.tiny((12, 10, 16))
    opts = dict(h=6.0, tstop=1.0, seed=2, open_states={"ryr": [0, 4]}, t_close={"ryr": 1.0})
    sim = pkg.Simulation(spec, opts)
    sim.advance(40)
    u = sim.state()[0]
    h = sim.info().h
    conv = [28853.9, 28853.9, 115415.6]
    offsets = [(n // 2 + d) * h for n, d in zip(u.shape, (-1, 2, 1))]
    got = sim.linescan(0, axis, offsets, conv, num_domains)
    want = direct(u, spec["voxels"], h, axis, offsets, conv, num_domains)
    np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12 * np.max(np.abs(want)))
    sim.close()
