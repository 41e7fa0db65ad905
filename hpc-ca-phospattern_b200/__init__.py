"""B200 calcium_sparks time step -- Python host bindings of libcsparks_cuda.so.

The product is the C ABI of include/csparks.h (libcsparks_cuda.so, built in-tree by
build.py) and the C command-line driver bin/calcium_sparks.  This module is the thin
ctypes layer the tests and bench.py drive it through.  There is no CPU path: loading
fails loudly when the CUDA library is missing.
"""
import ctypes as C
import os

import numpy as np

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libcsparks_cuda.so")
_lib = None


class CspError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{abi.ERRORS.get(code, code)}: {msg}")
        self.code = code


def load():
    """Load the in-tree CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run build.py (or __graft_entry__.build())")
        lib = C.CDLL(LIB_PATH)
        abi.declare(lib)
        _lib = lib
    return _lib


def _status(lib, h):
    buf = C.create_string_buffer(512)
    lib.csp_status(h, buf, 512)
    return buf.value.decode(errors="replace")


def mlp_init(seed=1):
    """Initial surrogate parameters (csp_mlp_init)."""
    lib = load()
    p = np.zeros(abi.MLP_NPARAM, dtype=np.float32)
    lib.csp_mlp_init(int(seed), p.ctypes.data_as(C.POINTER(C.c_float)))
    return p


def mlp_gradient(params, x, t):
    """(loss, grad) of the mean squared error from the device training kernels."""
    lib = load()
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    t = np.ascontiguousarray(t, dtype=np.float32)
    g = np.zeros(abi.MLP_NPARAM, dtype=np.float32)
    loss = C.c_float()
    P = C.POINTER(C.c_float)
    rc = lib.csp_mlp_gradient(p.ctypes.data_as(P), x.ctypes.data_as(P), t.ctypes.data_as(P), int(x.shape[0]),
                              g.ctypes.data_as(P), C.byref(loss))
    if rc != 0:
        raise CspError(rc, _status(lib, None))
    return loss.value, g


def mlp_forward(params, x, tensor_cores=False):
    """Network outputs on device (csp_mlp_forward): FP32 (False / 0), TF32 warp mma.sync
    tiles (True / 1) or TF32 tcgen05 tiles with tensor-memory accumulators (2)."""
    lib = load()
    p = np.ascontiguousarray(params, dtype=np.float32)
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.zeros((x.shape[0], 5), dtype=np.float32)
    P = C.POINTER(C.c_float)
    rc = lib.csp_mlp_forward(p.ctypes.data_as(P), x.ctypes.data_as(P), int(x.shape[0]), int(tensor_cores),
                             y.ctypes.data_as(P))
    if rc != 0:
        raise CspError(rc, _status(lib, None))
    return y


def set_device(device):
    """Select the CUDA device for the handles created next by this thread."""
    lib = load()
    rc = lib.csp_set_device(int(device))
    if rc != 0:
        raise CspError(rc, _status(lib, None))


class Simulation:
    """One handle of libcsparks_cuda.so over n realisations.

    specs: list of model descriptions (synth.py format); options: list of dicts for
    abi.make_options (one per realisation, or one shared).
    """

    def __init__(self, specs, options):
        self.lib = load()
        if isinstance(specs, dict):
            specs = [specs]
        if isinstance(options, dict):
            options = [options] * len(specs)
        n = len(specs)
        self._keep = []
        models = (abi.csp_model * n)()
        opts = (abi.csp_options * n)()
        for i, (s, o) in enumerate(zip(specs, options)):
            m, k1 = abi.make_model(s)
            op, k2 = abi.make_options(**o)
            models[i] = m
            opts[i] = op
            self._keep += [k1, k2, m, op]
        self._keep += [models, opts]
        h = C.c_void_p()
        rc = self.lib.csp_create(models, opts, n, C.byref(h))
        if rc != 0:
            raise CspError(rc, _status(self.lib, None))
        self.h = h
        self.n = n
        self.specs = specs

    def _check(self, rc):
        if rc != 0:
            raise CspError(rc, _status(self.lib, self.h))

    def info(self, r=0):
        inf = abi.csp_info()
        self._check(self.lib.csp_get_info(self.h, r, C.byref(inf)))
        return inf

    def shape(self, r=0):
        inf = self.info(r)
        return (inf.num_species, inf.n[0], inf.n[1], inf.n[2])

    def state(self, r=0):
        u = np.empty(self.shape(r), dtype=np.float64)
        self._check(self.lib.csp_download_state(self.h, r, u.ctypes.data_as(C.POINTER(C.c_double))))
        return u

    def linescan(self, species, axis, offsets_nm, conv, num_domains=0, r=0):
        """Gaussian linescan of one species along one axis (csp_linescan)."""
        n = self.info(r).n[axis]
        out = np.zeros(n, dtype=np.float64)
        off = np.ascontiguousarray(offsets_nm, dtype=np.float64)
        cv = np.ascontiguousarray(conv, dtype=np.float64)
        P = C.POINTER(C.c_double)
        self._check(self.lib.csp_linescan(self.h, r, int(species), int(axis), off.ctypes.data_as(P),
                                          cv.ctypes.data_as(P), int(num_domains), out.ctypes.data_as(P)))
        return out

    def autotune(self, repeats=3):
        """Pick the staged kernel's tile shape by timing (csp_autotune); returns a dict."""
        rep = abi.csp_tune_report()
        self._check(self.lib.csp_autotune(self.h, int(repeats), C.byref(rep)))
        cands = [dict(threads=rep.threads[i], segment=rep.segment[i], ms=rep.ms[i]) for i in range(rep.n)]
        return {"chosen": cands[rep.chosen], "candidates": cands}

    # ---- learned reaction surrogate ----
    def mlp_train(self, params=None, r=0, samples=1_000_000, val_samples=65536, epochs=10, batch=16384, lr=1e-3,
                  tol=1e-4, seed=1, harvested=False):
        """Train the reaction surrogate on device (csp_mlp_train); returns (params, report dict).
        harvested=True: on the pairs taken by mlp_harvest instead of sampled states."""
        p = mlp_init(seed) if params is None else np.array(params, dtype=np.float32)
        cfg = abi.csp_mlp_config(samples=samples, val_samples=val_samples, epochs=epochs, batch=batch, lr=lr,
                                 tol=tol, seed=seed, source=1 if harvested else 0)
        rep = abi.csp_mlp_report()
        self._check(self.lib.csp_mlp_train(self.h, r, C.byref(cfg), p.ctypes.data_as(C.POINTER(C.c_float)),
                                           C.byref(rep)))
        return p, {f: getattr(rep, f) for f, _ in abi.csp_mlp_report._fields_}

    def mlp_harvest(self, n, seed=1, capacity=None):
        """Take about n training pairs from the current fields (csp_mlp_harvest); returns
        (taken, held)."""
        taken, held = C.c_int64(), C.c_int64()
        self._check(self.lib.csp_mlp_harvest(self.h, int(n), int(seed), int(capacity or n), C.byref(taken),
                                             C.byref(held)))
        return taken.value, held.value

    def mlp_harvested(self, first=0, n=None):
        """The held training pairs [first, first + n) as (x[n][8], t[n][5]) (csp_mlp_harvested)."""
        if n is None:
            n = self.mlp_harvest(0)[1] - first
        x = np.zeros((n, abi.MLP_IN), dtype=np.float32)
        t = np.zeros((n, abi.MLP_OUT), dtype=np.float32)
        P = C.POINTER(C.c_float)
        self._check(self.lib.csp_mlp_harvested(self.h, int(first), int(n), x.ctypes.data_as(P), t.ctypes.data_as(P)))
        return x, t

    def set_surrogate(self, params, tol=1e-4):
        """Use the surrogate with these parameters on reaction steps (None: switch off)."""
        if params is None:
            self._check(self.lib.csp_set_surrogate(self.h, None, float(tol)))
            return
        self._mlp = np.ascontiguousarray(params, dtype=np.float32)
        self._check(self.lib.csp_set_surrogate(self.h, self._mlp.ctypes.data_as(C.POINTER(C.c_float)), float(tol)))

    def set_surrogate_tensor_cores(self, kind):
        """The network tiles' tensor cores: 1 warp mma.sync (default), 2 tcgen05 with
        tensor-memory accumulators (csp_set_surrogate_tensor_cores)."""
        self._check(self.lib.csp_set_surrogate_tensor_cores(self.h, int(kind)))

    def surrogate_counts(self):
        """(voxel increments, network evaluations, plain-integrator fallbacks)."""
        vx, ev, fb = C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self.lib.csp_surrogate_counts(self.h, C.byref(vx), C.byref(ev), C.byref(fb)))
        return vx.value, ev.value, fb.value

    def state_into(self, u, r=0):
        """Download realisation r into a caller-owned C-contiguous float64 array."""
        if u.dtype != np.float64 or not u.flags.c_contiguous or u.shape != self.shape(r):
            raise ValueError("state_into needs a C-contiguous float64 array of the state shape")
        self._check(self.lib.csp_download_state(self.h, r, u.ctypes.data_as(C.POINTER(C.c_double))))
        return u

    def set_state(self, u, r=0):
        u = np.ascontiguousarray(u, dtype=np.float64)
        if u.shape != self.shape(r):
            raise ValueError(f"state shape {u.shape} != {self.shape(r)}")
        self._check(self.lib.csp_upload_state(self.h, r, u.ctypes.data_as(C.POINTER(C.c_double))))

    def _state_ptrs(self, arrays, dtype=np.float64):
        if len(arrays) != self.n:
            raise ValueError(f"{len(arrays)} states for {self.n} realisations")
        for r, u in enumerate(arrays):
            if u.dtype != dtype or not u.flags.c_contiguous or u.shape != self.shape(r):
                raise ValueError(f"state {r} must be a C-contiguous {np.dtype(dtype).name} array of shape "
                                 f"{self.shape(r)}")
        ct = C.c_double if dtype == np.float64 else C.c_float
        ptrs = (C.POINTER(ct) * self.n)(*[u.ctypes.data_as(C.POINTER(ct)) for u in arrays])
        return ptrs

    def set_states_f32(self, arrays):
        """Upload every realisation's state from FP32 host arrays (csp_upload_states_f32)."""
        self._check(self.lib.csp_upload_states_f32(self.h, self._state_ptrs(arrays, np.float32)))

    def states_into_f32(self, arrays):
        """Download every realisation's state into FP32 host arrays (csp_download_states_f32)."""
        self._check(self.lib.csp_download_states_f32(self.h, self._state_ptrs(arrays, np.float32)))
        return arrays

    def run_states(self, u_in, nsteps, u_out, step_flags=False):
        """Upload u_in, advance nsteps, download into u_out, pipelined by realisation groups
        (csp_run_states); FP32 or FP64 host arrays.  Returns the stop flags, and with
        step_flags=True also the [nsteps][n] stop flags after every step."""
        dtype = u_in[0].dtype
        if dtype not in (np.float32, np.float64):
            raise ValueError("host states must be float32 or float64")
        pin = C.cast(self._state_ptrs(u_in, dtype), C.POINTER(C.c_void_p))
        pout = C.cast(self._state_ptrs(u_out, dtype), C.POINTER(C.c_void_p))
        flags = np.zeros(self.n, dtype=np.int32)
        sf = np.zeros((int(nsteps), self.n), dtype=np.int32) if step_flags else None
        P = C.POINTER(C.c_int32)
        self._check(self.lib.csp_run_states(self.h, abi.HOST_F32 if dtype == np.float32 else abi.HOST_F64, pin,
                                            int(nsteps), pout, flags.ctypes.data_as(P),
                                            sf.ctypes.data_as(P) if sf is not None else None))
        return (flags, sf) if step_flags else flags

    def set_states(self, arrays):
        """Upload every realisation's state in one call (csp_upload_states)."""
        self._check(self.lib.csp_upload_states(self.h, self._state_ptrs(arrays)))

    def states_into(self, arrays):
        """Download every realisation's state into caller-owned arrays (csp_download_states)."""
        self._check(self.lib.csp_download_states(self.h, self._state_ptrs(arrays)))
        return arrays

    def advance(self, nsteps):
        flags = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.csp_advance(self.h, int(nsteps), flags.ctypes.data_as(C.POINTER(C.c_int32))))
        return flags

    def advance_async(self, nsteps):
        """Launch nsteps steps and return at once (csp_advance_async)."""
        self._check(self.lib.csp_advance_async(self.h, int(nsteps)))

    def advance_wait(self):
        """Wait for advance_async; returns the stop flags (csp_advance_wait)."""
        flags = np.zeros(self.n, dtype=np.int32)
        self._check(self.lib.csp_advance_wait(self.h, flags.ctypes.data_as(C.POINTER(C.c_int32))))
        return flags

    def snapshot_async(self, species_mask=None, r=0):
        """Start an asynchronous copy of realisation r's fields (csp_snapshot_async)."""
        if species_mask is None:
            species_mask = (1 << self.shape(r)[0]) - 1
        self._check(self.lib.csp_snapshot_async(self.h, r, int(species_mask)))
        self._snap_shape = self.shape(r)

    def snapshot_wait(self):
        """Wait for snapshot_async; returns a copy of the fields ([species][x][y][z], FP64)."""
        p = C.POINTER(C.c_double)()
        self._check(self.lib.csp_snapshot_wait(self.h, C.byref(p)))
        n = int(np.prod(self._snap_shape))
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(self._snap_shape).copy()

    def profile(self, nsteps):
        """Advance nsteps with per-kernel CUDA events: (voxel_ms, boundary_ms) summed."""
        a, b = C.c_float(), C.c_float()
        self._check(self.lib.csp_profile_advance(self.h, int(nsteps), C.byref(a), C.byref(b)))
        return a.value, b.value

    def last_ms(self):
        ms = C.c_float()
        self._check(self.lib.csp_last_advance_ms(self.h, C.byref(ms)))
        return ms.value

    def channels(self, boundary, r=0):
        n = self.info(r).num_channels[boundary]
        st = np.zeros(n, dtype=np.int32)
        self._check(self.lib.csp_get_channel_states(self.h, r, boundary, st.ctypes.data_as(C.POINTER(C.c_int32))))
        return st

    def set_channels(self, boundary, states, r=0):
        st = np.ascontiguousarray(states, dtype=np.int32)
        self._check(self.lib.csp_set_channel_states(self.h, r, boundary, st.ctypes.data_as(C.POINTER(C.c_int32))))

    def outputs(self, r=0):
        inf = self.info(r)
        nd = len(self.specs[r]["domains"])
        ns = inf.num_species
        mn = np.zeros(nd * ns)
        mx = np.zeros(nd * ns)
        tot = np.zeros(nd * ns)
        nch = sum(inf.num_channels[b] for b in range(abi.MAX_BOUNDARIES))
        op = np.zeros(max(nch, 1), dtype=np.int32)
        P = C.POINTER
        self._check(self.lib.csp_reduce_outputs(self.h, r, mn.ctypes.data_as(P(C.c_double)),
                                                mx.ctypes.data_as(P(C.c_double)),
                                                tot.ctypes.data_as(P(C.c_double)),
                                                op.ctypes.data_as(P(C.c_int32))))
        return mn.reshape(nd, ns), mx.reshape(nd, ns), tot.reshape(nd, ns), op[:nch]

    def set_kernel(self, which):
        self._check(self.lib.csp_set_kernel(self.h, int(which)))

    def stream(self):
        s = C.c_void_p()
        self._check(self.lib.csp_get_stream(self.h, C.byref(s)))
        return s.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.csp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
