"""ctypes binding of the FP64 CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's
cpu_baseline / --impl reference legs as the checker; never by the product.
"""
import ctypes as C
import importlib
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
ROOT = os.path.dirname(HERE)
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
abi = importlib.import_module("hpc-ca-phospattern_b200.abi")

_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "csparks_oracle.c")):
            build()
        lib = C.CDLL(LIB)
        P = C.POINTER
        lib.oracle_create.restype = C.c_void_p
        lib.oracle_create.argtypes = [P(abi.csp_model), P(abi.csp_options), C.c_uint32]
        lib.oracle_step.argtypes = [C.c_void_p, C.c_int64]
        lib.oracle_get_state.argtypes = [C.c_void_p, P(C.c_double)]
        lib.oracle_set_state.argtypes = [C.c_void_p, P(C.c_double)]
        lib.oracle_get_info.argtypes = [C.c_void_p, P(abi.csp_info)]
        lib.oracle_get_channel_states.argtypes = [C.c_void_p, C.c_int32, P(C.c_int32)]
        lib.oracle_set_channel_states.argtypes = [C.c_void_p, C.c_int32, P(C.c_int32)]
        lib.oracle_reduce.argtypes = [C.c_void_p, P(C.c_double), P(C.c_double), P(C.c_double)]
        lib.oracle_domain_volume.restype = C.c_double
        lib.oracle_domain_volume.argtypes = [C.c_void_p, C.c_int]
        lib.oracle_destroy.argtypes = [C.c_void_p]
        _lib = lib
    return _lib


class Oracle:
    """FP64 reference step for one realisation (same model/options as the GPU path)."""

    def __init__(self, spec, options, realisation=0):
        self.lib = load()
        self.m, k1 = abi.make_model(spec)
        self.o, k2 = abi.make_options(**options)
        self._keep = (k1, k2)
        # the Philox stream of the GPU path: batch index + stream_offset
        self.h = self.lib.oracle_create(C.byref(self.m), C.byref(self.o),
                                        realisation + int(options.get("stream_offset", 0)))
        if not self.h:
            raise RuntimeError("oracle_create failed")
        self.spec = spec

    def info(self):
        inf = abi.csp_info()
        self.lib.oracle_get_info(self.h, C.byref(inf))
        return inf

    def shape(self):
        inf = self.info()
        return (inf.num_species, inf.n[0], inf.n[1], inf.n[2])

    def step(self, n):
        self.lib.oracle_step(self.h, int(n))

    def state(self):
        u = np.empty(self.shape(), dtype=np.float64)
        self.lib.oracle_get_state(self.h, u.ctypes.data_as(C.POINTER(C.c_double)))
        return u

    def set_state(self, u):
        u = np.ascontiguousarray(u, dtype=np.float64)
        self.lib.oracle_set_state(self.h, u.ctypes.data_as(C.POINTER(C.c_double)))

    def channels(self, boundary):
        n = self.info().num_channels[boundary]
        st = np.zeros(n, dtype=np.int32)
        rc = self.lib.oracle_get_channel_states(self.h, boundary, st.ctypes.data_as(C.POINTER(C.c_int32)))
        if rc:
            raise IndexError(boundary)
        return st

    def set_channels(self, boundary, states):
        st = np.ascontiguousarray(states, dtype=np.int32)
        self.lib.oracle_set_channel_states(self.h, boundary, st.ctypes.data_as(C.POINTER(C.c_int32)))

    def outputs(self):
        nd = len(self.spec["domains"])
        ns = self.info().num_species
        mn, mx, tot = (np.zeros(nd * ns) for _ in range(3))
        P = C.POINTER(C.c_double)
        self.lib.oracle_reduce(self.h, mn.ctypes.data_as(P), mx.ctypes.data_as(P), tot.ctypes.data_as(P))
        return mn.reshape(nd, ns), mx.reshape(nd, ns), tot.reshape(nd, ns)

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
