"""The reference's HDF5 input formats <-> model descriptions (synth.py format).

Geometry file (read by geometry.c:92-344): root attributes h, global_size; group
/domains (attributes num, name_<i>, indices; datasets voxels [N0,N1,N2] uint8 and
domain_connections [n,n] uint8); group /boundaries (attributes num, name_<i>, type_<i>;
one uint16 [n,6] dataset per boundary).  Species file (read by species.c:103-258,
boundaryfluxes.c:377-527): root attributes num_domains, num_species, domain_name_<i>,
species_name_<i>, num_fixed_domain_species, fixed_domain_species, convolution_constants,
use_ryr, use_p_ryr, use_serca; one group per domain (num_diffusive, init, diffusive,
sigma, num_buffers, and buffer_<bi> subgroups with k_on, k_off, tot, species); groups
/ryr, /p_ryr, /serca.  Attribute types follow the reference's C fields, because
read_h5_attr copies the file's own type into them (utils.c:77-99).

Uses the project's HDF5-subset library (lib/libh5lite.so).
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libh5lite.so")
U8, U16, U32, U64, I8, I16, I32, I64, F32, F64, STR = range(1, 12)
NP = {U8: np.uint8, U16: np.uint16, U32: np.uint32, U64: np.uint64, I8: np.int8, I16: np.int16,
      I32: np.int32, I64: np.int64, F32: np.float32, F64: np.float64}
CODE = {np.dtype(v): k for k, v in NP.items()}
_lib = None


def _load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run build.py")
        lib = C.CDLL(LIB_PATH)
        P = C.POINTER
        lib.h5l_open.restype = C.c_void_p
        lib.h5l_open.argtypes = [C.c_char_p, C.c_int]
        lib.h5l_create.restype = C.c_void_p
        lib.h5l_create.argtypes = [C.c_char_p]
        lib.h5l_close.argtypes = [C.c_void_p]
        lib.h5l_flush.argtypes = [C.c_void_p]
        lib.h5l_error.restype = C.c_char_p
        lib.h5l_get_attr.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, P(C.c_int), P(C.c_size_t), P(C.c_int),
                                     P(C.c_uint64), P(C.c_void_p), P(C.c_size_t)]
        lib.h5l_get_dset.argtypes = [C.c_void_p, C.c_char_p, P(C.c_int), P(C.c_size_t), P(C.c_int), P(C.c_uint64),
                                     P(C.c_void_p), P(C.c_size_t)]
        lib.h5l_list.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t]
        lib.h5l_list_attrs.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_size_t]
        lib.h5l_put_attr.argtypes = [C.c_void_p, C.c_char_p, C.c_char_p, C.c_int, C.c_size_t, C.c_int,
                                     P(C.c_uint64), C.c_void_p]
        lib.h5l_put_dset.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, P(C.c_uint64), C.c_void_p]
        lib.h5l_put_group.argtypes = [C.c_void_p, C.c_char_p]
        _lib = lib
    return _lib


class H5:
    """An HDF5 file held in memory by h5lite (written on close when created)."""

    def __init__(self, path, mode="r"):
        self.lib = _load()
        self.path = path
        if mode == "w":
            self.f = self.lib.h5l_create(path.encode())
        else:
            self.f = self.lib.h5l_open(path.encode(), 1 if mode == "a" else 0)
        if not self.f:
            raise OSError(f"{path}: {self.lib.h5l_error().decode()}")

    def flush(self):
        """Write the file as it stands (created files: the new datasets' data and the metadata)."""
        if self.lib.h5l_flush(self.f):
            raise OSError(f"{self.path}: {self.lib.h5l_error().decode()}")

    def close(self):
        if self.f:
            rc = self.lib.h5l_close(self.f)
            self.f = None
            if rc:
                raise OSError(f"{self.path}: {self.lib.h5l_error().decode()}")

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def attr(self, obj, name):
        code, size, nd = C.c_int(), C.c_size_t(), C.c_int()
        dims = (C.c_uint64 * 8)()
        data, nb = C.c_void_p(), C.c_size_t()
        rc = self.lib.h5l_get_attr(self.f, obj.encode(), name.encode(), C.byref(code), C.byref(size), C.byref(nd), dims,
                                   C.byref(data), C.byref(nb))
        if rc:
            raise KeyError(self.lib.h5l_error().decode())
        raw = C.string_at(data, nb.value) if nb.value else b""
        if code.value == STR:
            return raw.split(b"\0")[0].decode()
        a = np.frombuffer(raw, dtype=NP[code.value]).copy()
        return a.reshape([dims[i] for i in range(nd.value)]) if nd.value else a[0]

    def dset(self, path):
        code, size, nd = C.c_int(), C.c_size_t(), C.c_int()
        dims = (C.c_uint64 * 8)()
        data, nb = C.c_void_p(), C.c_size_t()
        rc = self.lib.h5l_get_dset(self.f, path.encode(), C.byref(code), C.byref(size), C.byref(nd), dims,
                                   C.byref(data), C.byref(nb))
        if rc:
            raise KeyError(self.lib.h5l_error().decode())
        raw = C.string_at(data, nb.value) if nb.value else b""
        return np.frombuffer(raw, dtype=NP[code.value]).copy().reshape([dims[i] for i in range(nd.value)])

    def list(self, path="/"):
        buf = C.create_string_buffer(1 << 20)
        n = self.lib.h5l_list(self.f, path.encode(), buf, len(buf))
        if n < 0:
            raise KeyError(self.lib.h5l_error().decode())
        return [(l[0] == "g", l[1:]) for l in buf.value.decode().splitlines()]

    def attrs(self, path="/"):
        buf = C.create_string_buffer(1 << 16)
        n = self.lib.h5l_list_attrs(self.f, path.encode(), buf, len(buf))
        if n < 0:
            raise KeyError(self.lib.h5l_error().decode())
        return buf.value.decode().splitlines()

    def put_attr(self, obj, name, value, dtype=None):
        if isinstance(value, str):
            b = value.encode()
            dims = (C.c_uint64 * 8)()
            rc = self.lib.h5l_put_attr(self.f, obj.encode(), name.encode(), STR, len(b), 0, dims, C.c_char_p(b))
        else:
            a = np.ascontiguousarray(np.asarray(value, dtype=dtype))
            dims = (C.c_uint64 * 8)(*a.shape)
            rc = self.lib.h5l_put_attr(self.f, obj.encode(), name.encode(), CODE[a.dtype], a.itemsize, a.ndim, dims,
                                       a.ctypes.data_as(C.c_void_p))
        if rc:
            raise OSError(self.lib.h5l_error().decode())

    def put_dset(self, path, value, dtype=None):
        a = np.ascontiguousarray(np.asarray(value, dtype=dtype))
        dims = (C.c_uint64 * 8)(*a.shape)
        if self.lib.h5l_put_dset(self.f, path.encode(), CODE[a.dtype], a.ndim, dims, a.ctypes.data_as(C.c_void_p)):
            raise OSError(self.lib.h5l_error().decode())

    def put_group(self, path):
        if self.lib.h5l_put_group(self.f, path.encode()):
            raise OSError(self.lib.h5l_error().decode())


RYR_FIELDS = ("Kd_open", "k_min_open", "k_max_open", "n_open", "Kd_close", "k_min_close", "k_max_close",
              "n_close", "i_unitary")


def write_model(spec, geometry_file, species_file):
    """Write a model description as the reference's geometry and species files."""
    write_geometry(spec, geometry_file)
    write_species(spec, species_file)


def write_geometry(spec, geometry_file):
    """The geometry file (geometry.c:96-344): root h / global_size, /domains, /boundaries."""
    doms = spec["domains"]
    with H5(geometry_file, "w") as g:
        g.put_attr("/", "h", float(spec["h"]), np.float64)
        g.put_attr("/", "global_size", np.asarray(spec.get("global_size", [s * spec["h"] for s in spec["voxels"].shape]),
                                                  dtype=np.float64))
        g.put_group("/domains")
        g.put_attr("/domains", "num", len(doms), np.uint8)
        for i, d in enumerate(doms):
            g.put_attr("/domains", f"name_{i}", d)
        g.put_attr("/domains", "indices", np.arange(len(doms), dtype=np.uint8))
        g.put_dset("/domains/voxels", spec["voxels"], np.uint8)
        g.put_dset("/domains/domain_connections", spec["domain_connections"], np.uint8)
        g.put_group("/boundaries")
        bl = spec.get("boundaries", [])
        g.put_attr("/boundaries", "num", len(bl), np.uint8)
        for i, b in enumerate(bl):
            g.put_attr("/boundaries", f"name_{i}", b["name"])
            g.put_attr("/boundaries", f"type_{i}", b["type"])
            g.put_dset(f"/boundaries/{b['name']}", np.asarray(b["pairs"]).reshape(-1, 6), np.uint16)


def write_species(spec, species_file):
    """The species file (species.c:103-258, boundaryfluxes.c:377-527)."""
    doms = spec["domains"]
    with H5(species_file, "w") as s:
        sp = spec["species"]
        s.put_attr("/", "num_domains", len(doms), np.uint8)
        s.put_attr("/", "num_species", len(sp), np.uint8)
        for i, d in enumerate(doms):
            s.put_attr("/", f"domain_name_{i}", d)
        for i, n in enumerate(sp):
            s.put_attr("/", f"species_name_{i}", n)
        fixed = spec.get("fixed_domain_species", [])
        s.put_attr("/", "num_fixed_domain_species", len(fixed), np.uint8)
        if fixed:
            s.put_attr("/", "fixed_domain_species", np.asarray(fixed, dtype=np.uint8).ravel())
        s.put_attr("/", "convolution_constants",
                   np.asarray(spec.get("convolution_constants", [28853.9, 28853.9, 115415.6]), dtype=np.float64))
        for key in ("ryr", "p_ryr", "serca"):
            s.put_attr("/", f"use_{key}", 1 if key in spec else 0, np.uint8)
        for d in doms:
            ds = spec["domain_species"][d]
            s.put_group("/" + d)
            diff = ds.get("diffusive", [])
            s.put_attr("/" + d, "num_diffusive", len(diff), np.uint8)
            s.put_attr("/" + d, "init", np.asarray(ds["init"], dtype=np.float64))
            if diff:
                s.put_attr("/" + d, "diffusive", np.asarray(diff, dtype=np.uint8))
                s.put_attr("/" + d, "sigma", np.asarray(ds["sigma"], dtype=np.float64))
            bufs = ds.get("buffers", [])
            s.put_attr("/" + d, "num_buffers", len(bufs), np.uint8)
            for bi, b in enumerate(bufs):
                grp = f"/{d}/buffer_{bi}"
                s.put_group(grp)
                for f in ("k_off", "k_on", "tot"):
                    s.put_attr(grp, f, float(b[f]), np.float64)
                s.put_attr(grp, "species", np.asarray(b["species"], dtype=np.uint8))
        for key in ("ryr", "p_ryr"):
            if key in spec:
                s.put_group("/" + key)
                for f in RYR_FIELDS:
                    s.put_attr("/" + key, f, float(spec[key][f]), np.float64)
                s.put_attr("/" + key, "boundary", spec[key]["boundary"])
                s.put_attr("/" + key, "species", spec[key]["species"])
        if "serca" in spec:
            s.put_group("/serca")
            for f in ("v_cyt_to_A_sr", "density", "scale"):
                s.put_attr("/serca", f, float(spec["serca"][f]), np.float64)
            s.put_attr("/serca", "boundary", spec["serca"]["boundary"])


def _float(v):
    """One attribute value as a float (attributes are written as 1-element arrays)."""
    return float(np.ravel(v)[0])


def _int(v):
    return int(np.ravel(v)[0])


def read_geometry(geometry_file):
    """The geometry part of a model description."""
    spec = {}
    with H5(geometry_file) as g:
        spec["h"] = _float(g.attr("/", "h"))
        spec["global_size"] = [float(v) for v in np.atleast_1d(g.attr("/", "global_size"))]
        nd = _int(g.attr("domains", "num"))
        spec["domains"] = [g.attr("domains", f"name_{i}") for i in range(nd)]
        spec["voxels"] = g.dset("/domains/voxels").astype(np.uint8)
        spec["domain_connections"] = g.dset("/domains/domain_connections").astype(np.uint8)
        nb = _int(g.attr("boundaries", "num"))
        spec["boundaries"] = []
        for i in range(nb):
            name = g.attr("boundaries", f"name_{i}")
            spec["boundaries"].append(dict(name=name, type=g.attr("boundaries", f"type_{i}"),
                                           pairs=g.dset(f"/boundaries/{name}").astype(np.uint16).reshape(-1, 6)))
    return spec


def read_model(geometry_file, species_file):
    """Read the reference's geometry and species files into a model description."""
    spec = read_geometry(geometry_file)
    with H5(species_file) as s:
        ns = _int(s.attr("/", "num_species"))
        spec["species"] = [s.attr("/", f"species_name_{i}") for i in range(ns)]
        spec["domain_species"] = {}
        for d in spec["domains"]:
            ds = {"init": [float(v) for v in np.atleast_1d(s.attr(d, "init"))]}
            ndiff = _int(s.attr(d, "num_diffusive"))
            ds["diffusive"] = [int(v) for v in np.atleast_1d(s.attr(d, "diffusive"))] if ndiff else []
            ds["sigma"] = [float(v) for v in np.atleast_1d(s.attr(d, "sigma"))] if ndiff else []
            ds["buffers"] = []
            for bi in range(_int(s.attr(d, "num_buffers"))):
                grp = f"/{d}/buffer_{bi}/"
                ds["buffers"].append(dict(k_off=_float(s.attr(grp, "k_off")), k_on=_float(s.attr(grp, "k_on")),
                                          tot=_float(s.attr(grp, "tot")),
                                          species=[int(v) for v in np.atleast_1d(s.attr(grp, "species"))]))
            spec["domain_species"][d] = ds
        nf = _int(s.attr("/", "num_fixed_domain_species"))
        fx = np.atleast_1d(s.attr("/", "fixed_domain_species")) if nf else []
        spec["fixed_domain_species"] = [(int(fx[2 * i]), int(fx[2 * i + 1])) for i in range(nf)]
        spec["convolution_constants"] = [float(v) for v in np.atleast_1d(s.attr("/", "convolution_constants"))]
        for key in ("ryr", "p_ryr"):
            if _int(s.attr("/", f"use_{key}")):
                p = {f: _float(s.attr("/" + key, f)) for f in RYR_FIELDS}
                p["boundary"] = s.attr("/" + key, "boundary")
                p["species"] = s.attr("/" + key, "species")
                spec[key] = p
        if _int(s.attr("/", "use_serca")):
            p = {f: _float(s.attr("/serca", f)) for f in ("v_cyt_to_A_sr", "density", "scale")}
            p["boundary"] = s.attr("/serca", "boundary")
            # the reference takes the SERCA species from the /ryr group (boundaryfluxes.c:511)
            p["species"] = s.attr("/ryr", "species")
            spec["serca"] = p
    return spec
