"""The allocation-free reduction entry point against the handle's own reduction.

csp_reduce_field_noalloc serves callers that cannot allocate device memory (a plugin
inside a framework that reserved the device memory for its pool, or a latency-bound loop
where cudaMalloc's device synchronisation is not allowed).  Its block partials live in a
fixed device array inside the library.  This test passes it the device buffers of the
fields of a running simulation and checks, on two calls in a row, that it returns what
csp_reduce_outputs returns for the same fields.  It is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FLT_MAX = float(np.float32(3.4028235e38))
FLT_MIN = float(np.float32(1.1754944e-38))


def test_noalloc_reduction_matches_csp_reduce_outputs(pkg, synth):
    import torch
    spec = synth.tiny((12, 12, 16))
    sim = pkg.Simulation(spec, dict(h=6.0, tstop=1.0, seed=1, open_states={"ryr": [0, 3]}))
    sim.advance(40)
    mn, mx, tot, _ = sim.outputs()                      # the existing entry point
    u = sim.state()                                     # [species][x][y][z]
    nd = len(spec["domains"])
    dV = sim.info().h ** 3
    lib = pkg.load()
    dom = torch.tensor(np.ascontiguousarray(spec["voxels"]).ravel(), dtype=torch.uint8, device="cuda")
    n = dom.numel()
    present = [d for d in range(nd) if np.any(spec["voxels"] == d)]
    for call in range(2):                                # two calls in a row share the scratch
        for s in range(u.shape[0]):
            field = torch.tensor(u[s].ravel().astype(np.float32), device="cuda")
            out = torch.full((3 * nd,), -1.0, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            rc = lib.csp_reduce_field_noalloc(C.c_void_p(field.data_ptr()), C.c_void_p(dom.data_ptr()), n, nd,
                                              dV, C.c_void_p(out.data_ptr()), None)
            assert rc == 0
            torch.cuda.synchronize()
            o = out.cpu().numpy().reshape(3, nd)
            # the handle reduces its fields in FP64 (base + FP32 deviation); this call gets
            # the same fields rounded to FP32, so the two agree to FP32 precision
            for d in present:
                np.testing.assert_allclose(o[0, d], mn[d, s], rtol=2.0 ** -22)
                np.testing.assert_allclose(o[1, d], mx[d, s], rtol=2.0 ** -22)
                np.testing.assert_allclose(o[2, d], tot[d, s], rtol=2.0 ** -22)
            for d in set(range(nd)) - set(present):
                assert o[0, d] == FLT_MAX and o[1, d] == FLT_MIN and o[2, d] == 0.0


def test_noalloc_rejects_sizes_beyond_its_scratch(pkg):
    import torch
    lib = pkg.load()
    field = torch.zeros(16, dtype=torch.float32, device="cuda")
    dom = torch.zeros(16, dtype=torch.uint8, device="cuda")
    out = torch.zeros(3 * 8, dtype=torch.float64, device="cuda")
    rc = lib.csp_reduce_field_noalloc(C.c_void_p(field.data_ptr()), C.c_void_p(dom.data_ptr()), 16, 6, 1.0,
                                      C.c_void_p(out.data_ptr()), None)
    assert rc == -4          # CSP_ERANGE: more domains than the fixed scratch holds


def test_noalloc_reduction_large_field_on_a_stream(pkg):
    """A field larger than the fixed grid covers in one pass (592 blocks x 256 threads), on
    a non-default stream, with only negative values in one domain and domain bytes whose
    id (bits 0-2) is at or above num_domains or that carry the upper bits: against an FP64
    NumPy reduction with the reference's start values (species.c:2808-2815: max starts
    at FLT_MIN, so an all-negative domain reports FLT_MIN)."""
    import torch
    lib = pkg.load()
    rng = np.random.default_rng(11)
    n = 592 * 256 * 3 + 1234
    nd = 4
    dom = rng.integers(0, 256, size=n, dtype=np.uint8)
    val = rng.normal(5.0, 3.0, size=n).astype(np.float32)
    d = dom & 7
    val[d == 2] = -np.abs(val[d == 2]) - 0.5              # domain 2: negative only
    dV = 216.0
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        field = torch.from_numpy(val).to("cuda", non_blocking=False)
        dd = torch.from_numpy(dom).to("cuda", non_blocking=False)
        out = torch.full((3 * nd,), -1.0, dtype=torch.float64, device="cuda")
    s.synchronize()
    v64 = val.astype(np.float64)
    for call in range(2):
        rc = lib.csp_reduce_field_noalloc(C.c_void_p(field.data_ptr()), C.c_void_p(dd.data_ptr()), n, nd, dV,
                                          C.c_void_p(out.data_ptr()), C.c_void_p(s.cuda_stream))
        assert rc == 0
        s.synchronize()
        o = out.cpu().numpy().reshape(3, nd)
        for k in range(nd):
            m = d == k
            assert o[0, k] == min(FLT_MAX, v64[m].min())
            assert o[1, k] == max(FLT_MIN, v64[m].max())
            np.testing.assert_allclose(o[2, k], v64[m].sum() * dV, rtol=1e-11)
        assert o[1, 2] == FLT_MIN
