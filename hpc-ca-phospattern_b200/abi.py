"""ctypes mirror of include/csparks.h (the C ABI of libcsparks_cuda.so).

The structures here are byte-for-byte the C structs; `Model` and `Options` keep the
numpy arrays they point into alive for as long as the ctypes structure exists.
"""
import ctypes as C

import numpy as np

MAX_DOMAINS = 5
MAX_SPECIES = 8
MAX_BUFFERS = 8
MAX_BOUNDARIES = 8
MAX_FIXED = 8
NAME_LEN = 20
HOST_F64, HOST_F32 = 0, 1    # csp_run_states host_dtype (CSP_HOST_F64, CSP_HOST_F32)
TUNE_MAX = 10                # CSP_TUNE_MAX

OK, EINVAL, ENOMEM, ECUDA, ERANGE, EDEVICE, ENOTSUP = 0, -1, -2, -3, -4, -5, -6
DENSITY, DISCRETE = 0, 1
ERRORS = {0: "CSP_OK", -1: "CSP_EINVAL", -2: "CSP_ENOMEM", -3: "CSP_ECUDA",
          -4: "CSP_ERANGE", -5: "CSP_EDEVICE", -6: "CSP_ENOTSUP"}

Name = C.c_char * NAME_LEN


class csp_boundary(C.Structure):
    _fields_ = [("name", Name), ("type", C.c_int32), ("num_pairs", C.c_int32),
                ("pairs", C.POINTER(C.c_uint16))]


class csp_domain_species(C.Structure):
    _fields_ = [("num_diffusive", C.c_int32),
                ("diffusive", C.c_uint8 * MAX_SPECIES),
                ("sigma", C.c_double * MAX_SPECIES),
                ("init", C.c_double * MAX_SPECIES),
                ("num_buffers", C.c_int32),
                ("k_on", C.c_double * MAX_BUFFERS),
                ("k_off", C.c_double * MAX_BUFFERS),
                ("tot", C.c_double * MAX_BUFFERS),
                ("bsp0", C.c_uint8 * MAX_BUFFERS),
                ("bsp1", C.c_uint8 * MAX_BUFFERS)]


class csp_ryr_params(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("Kd_open", "k_min_open", "k_max_open", "n_open",
                                          "Kd_close", "k_min_close", "k_max_close", "n_close",
                                          "i_unitary")] + [("boundary", Name), ("species", Name)]


class csp_serca_params(C.Structure):
    _fields_ = [("v_cyt_to_A_sr", C.c_double), ("density", C.c_double), ("scale", C.c_double),
                ("boundary", Name), ("species", Name)]


class csp_model(C.Structure):
    _fields_ = [("h_geom", C.c_double),
                ("global_size", C.c_double * 3),
                ("N", C.c_int32 * 3),
                ("num_domains", C.c_int32),
                ("domain_names", Name * MAX_DOMAINS),
                ("domain_indices", C.c_uint8 * MAX_DOMAINS),
                ("voxels", C.POINTER(C.c_uint8)),
                ("domain_connections", C.c_uint8 * (MAX_DOMAINS * MAX_DOMAINS)),
                ("num_boundaries", C.c_int32),
                ("boundaries", csp_boundary * MAX_BOUNDARIES),
                ("num_species", C.c_int32),
                ("species_names", Name * MAX_SPECIES),
                ("domain", csp_domain_species * MAX_DOMAINS),
                ("num_fixed_domain_species", C.c_int32),
                ("fixed_domain_species", C.c_uint8 * (2 * MAX_FIXED)),
                ("use_ryr", C.c_uint8), ("use_p_ryr", C.c_uint8), ("use_serca", C.c_uint8),
                ("ryr", csp_ryr_params), ("p_ryr", csp_ryr_params),
                ("serca", csp_serca_params),
                ("convolution_constants", C.c_double * 3)]


class csp_open_list(C.Structure):
    _fields_ = [("name", Name), ("count", C.c_int32), ("indices", C.POINTER(C.c_int32))]


class csp_t_close(C.Structure):
    _fields_ = [("name", Name), ("time", C.c_double)]


class csp_options(C.Structure):
    _fields_ = [("h", C.c_double), ("dt", C.c_double), ("tstop", C.c_double),
                ("dt_save", C.c_double), ("dt_update_react", C.c_double),
                ("dt_update_stoch", C.c_double), ("tabort", C.c_double),
                ("force_dirichlet", C.c_int32), ("seed_given", C.c_int32),
                ("seed", C.c_uint64),
                ("num_open_lists", C.c_int32), ("open", csp_open_list * MAX_BOUNDARIES),
                ("num_t_close", C.c_int32), ("t_close", csp_t_close * MAX_BOUNDARIES),
                ("stream_offset", C.c_int64)]


class csp_info(C.Structure):
    _fields_ = [("n", C.c_int32 * 3), ("subdivisions", C.c_int32), ("h", C.c_double),
                ("dt", C.c_double), ("num_species", C.c_int32), ("num_diffusive", C.c_int32),
                ("diffusive_species", C.c_int32 * MAX_SPECIES),
                ("substeps", C.c_int32 * MAX_SPECIES), ("num_buffers", C.c_int32),
                ("stochastic_substep", C.c_int32), ("reaction_substep", C.c_int32),
                ("total_steps", C.c_int64), ("step", C.c_int64),
                ("num_channels", C.c_int32 * MAX_BOUNDARIES), ("stopped", C.c_int32),
                ("fused_pairs", C.c_int64), ("flux_rows", C.c_int64)]


MLP_NPARAM = 5061
MLP_IN, MLP_OUT = 8, 5


class csp_mlp_config(C.Structure):
    _fields_ = [("samples", C.c_int64), ("val_samples", C.c_int64), ("epochs", C.c_int32), ("batch", C.c_int32),
                ("lr", C.c_float), ("tol", C.c_double), ("seed", C.c_uint64), ("source", C.c_int32)]


class csp_mlp_report(C.Structure):
    _fields_ = [("val_loss_first", C.c_float), ("val_loss_last", C.c_float), ("val_accept_rate", C.c_double),
                ("train_ms", C.c_float), ("steps", C.c_int32), ("samples", C.c_int64)]


class csp_tune_report(C.Structure):
    _fields_ = [("n", C.c_int32), ("threads", C.c_int32 * TUNE_MAX), ("segment", C.c_int32 * TUNE_MAX),
                ("ms", C.c_float * TUNE_MAX), ("chosen", C.c_int32)]


def _name(s):
    b = s.encode()
    if len(b) >= NAME_LEN:
        raise ValueError(f"name {s!r} longer than {NAME_LEN - 1} bytes")
    return b


def make_model(spec):
    """Build a csp_model from a plain-Python model description (see synth.py).

    Returns (csp_model, keepalive) -- keepalive holds the numpy arrays the struct points to.
    """
    m = csp_model()
    keep = []
    vox = np.ascontiguousarray(spec["voxels"], dtype=np.uint8)
    keep.append(vox)
    m.h_geom = float(spec["h"])
    m.global_size[:] = [float(v) for v in spec.get("global_size", [s * spec["h"] for s in vox.shape])]
    m.N[:] = list(vox.shape)
    doms = spec["domains"]
    m.num_domains = len(doms)
    for i, d in enumerate(doms):
        m.domain_names[i].value = _name(d)
        m.domain_indices[i] = i
    m.voxels = vox.ctypes.data_as(C.POINTER(C.c_uint8))
    conn = np.asarray(spec["domain_connections"], dtype=np.uint8).reshape(len(doms), len(doms))
    for a in range(len(doms)):
        for b in range(len(doms)):
            m.domain_connections[a * len(doms) + b] = int(conn[a, b])
    bnds = spec.get("boundaries", [])
    m.num_boundaries = len(bnds)
    for i, b in enumerate(bnds):
        pairs = np.ascontiguousarray(b["pairs"], dtype=np.uint16).reshape(-1, 6)
        keep.append(pairs)
        m.boundaries[i].name = _name(b["name"])
        m.boundaries[i].type = DISCRETE if b["type"] == "discrete" else DENSITY
        m.boundaries[i].num_pairs = pairs.shape[0]
        m.boundaries[i].pairs = pairs.ctypes.data_as(C.POINTER(C.c_uint16))
    species = spec["species"]
    m.num_species = len(species)
    for i, s in enumerate(species):
        m.species_names[i].value = _name(s)
    for di, dname in enumerate(doms):
        ds = spec["domain_species"][dname]
        dst = m.domain[di]
        diff = ds.get("diffusive", [])
        dst.num_diffusive = len(diff)
        for k, (si, sig) in enumerate(zip(diff, ds.get("sigma", []))):
            dst.diffusive[k] = si
            dst.sigma[k] = sig
        for k, v in enumerate(ds["init"]):
            dst.init[k] = v
        bufs = ds.get("buffers", [])
        dst.num_buffers = len(bufs)
        for k, bf in enumerate(bufs):
            dst.k_on[k] = bf["k_on"]
            dst.k_off[k] = bf["k_off"]
            dst.tot[k] = bf["tot"]
            dst.bsp0[k] = bf["species"][0]
            dst.bsp1[k] = bf["species"][1]
    fixed = spec.get("fixed_domain_species", [])
    m.num_fixed_domain_species = len(fixed)
    for k, (d, s) in enumerate(fixed):
        m.fixed_domain_species[2 * k] = d
        m.fixed_domain_species[2 * k + 1] = s
    for key in ("ryr", "p_ryr"):
        if key in spec:
            setattr(m, "use_" + key, 1)
            p = getattr(m, key)
            for f in ("Kd_open", "k_min_open", "k_max_open", "n_open", "Kd_close", "k_min_close",
                      "k_max_close", "n_close", "i_unitary"):
                setattr(p, f, float(spec[key][f]))
            p.boundary = _name(spec[key]["boundary"])
            p.species = _name(spec[key]["species"])
    if "serca" in spec:
        m.use_serca = 1
        for f in ("v_cyt_to_A_sr", "density", "scale"):
            setattr(m.serca, f, float(spec["serca"][f]))
        m.serca.boundary = _name(spec["serca"]["boundary"])
        # the reference takes the SERCA species from the /ryr group (boundaryfluxes.c:511)
        m.serca.species = _name(spec["ryr"]["species"] if "ryr" in spec else spec["serca"]["species"])
    m.convolution_constants[:] = spec.get("convolution_constants", [28853.9, 28853.9, 115415.6])
    return m, keep


def make_options(h=6.0, dt=-1.0, tstop=10.0, dt_save=0.5, dt_update_react=-1.0,
                 dt_update_stoch=-1.0, tabort=0.0, force_dirichlet=False, seed=None,
                 open_states=None, t_close=None, stream_offset=0):
    """csp_options with the reference defaults (options.c:502-542) unless overridden.

    open_states: {"ryr": [0, 3], ...} as -O; t_close: {"ryr": 2.0} as -C.
    """
    o = csp_options()
    keep = []
    o.h, o.dt, o.tstop, o.dt_save = h, dt, tstop, dt_save
    o.dt_update_react, o.dt_update_stoch, o.tabort = dt_update_react, dt_update_stoch, tabort
    o.force_dirichlet = 1 if force_dirichlet else 0
    o.seed_given = 1 if seed is not None else 0
    o.seed = int(seed or 0)
    for i, (name, idx) in enumerate((open_states or {}).items()):
        arr = np.ascontiguousarray(idx, dtype=np.int32)
        keep.append(arr)
        o.open[i].name = _name(name)
        o.open[i].count = arr.size
        o.open[i].indices = arr.ctypes.data_as(C.POINTER(C.c_int32))
    o.num_open_lists = len(open_states or {})
    for i, (name, t) in enumerate((t_close or {}).items()):
        o.t_close[i].name = _name(name)
        o.t_close[i].time = float(t)
    o.num_t_close = len(t_close or {})
    o.stream_offset = int(stream_offset)
    return o, keep


def declare(lib):
    """Attach argtypes / restypes of every csp_* symbol to a loaded CDLL."""
    P = C.POINTER
    h = C.c_void_p
    sig = {
        "csp_options_default": (None, [P(csp_options)]),
        "csp_set_device": (C.c_int, [C.c_int32]),
        "csp_create": (C.c_int, [P(csp_model), P(csp_options), C.c_int32, P(C.c_void_p)]),
        "csp_get_info": (C.c_int, [h, C.c_int32, P(csp_info)]),
        "csp_upload_state": (C.c_int, [h, C.c_int32, P(C.c_double)]),
        "csp_download_state": (C.c_int, [h, C.c_int32, P(C.c_double)]),
        "csp_upload_states": (C.c_int, [h, P(P(C.c_double))]),
        "csp_download_states": (C.c_int, [h, P(P(C.c_double))]),
        "csp_upload_states_f32": (C.c_int, [h, P(P(C.c_float))]),
        "csp_download_states_f32": (C.c_int, [h, P(P(C.c_float))]),
        "csp_run_states": (C.c_int, [h, C.c_int32, P(C.c_void_p), C.c_int64, P(C.c_void_p), P(C.c_int32),
                                     P(C.c_int32)]),
        "csp_advance": (C.c_int, [h, C.c_int64, P(C.c_int32)]),
        "csp_advance_async": (C.c_int, [h, C.c_int64]),
        "csp_advance_wait": (C.c_int, [h, P(C.c_int32)]),
        "csp_snapshot_async": (C.c_int, [h, C.c_int32, C.c_uint32]),
        "csp_snapshot_wait": (C.c_int, [h, P(P(C.c_double))]),
        "csp_reduce_outputs": (C.c_int, [h, C.c_int32, P(C.c_double), P(C.c_double), P(C.c_double), P(C.c_int32)]),
        "csp_get_channel_states": (C.c_int, [h, C.c_int32, C.c_int32, P(C.c_int32)]),
        "csp_linescan": (C.c_int, [h, C.c_int32, C.c_int32, C.c_int32, P(C.c_double), P(C.c_double), C.c_int32,
                                   P(C.c_double)]),
        "csp_set_channel_states": (C.c_int, [h, C.c_int32, C.c_int32, P(C.c_int32)]),
        "csp_status": (C.c_int, [h, C.c_char_p, C.c_size_t]),
        "csp_get_stream": (C.c_int, [h, P(C.c_void_p)]),
        "csp_last_advance_ms": (C.c_int, [h, P(C.c_float)]),
        "csp_set_kernel": (C.c_int, [h, C.c_int32]),
        "csp_test_wait_timeout": (C.c_int, [h, C.c_int32]),
        "csp_set_phase_timing": (C.c_int, [h, C.c_int32]),
        "csp_get_phase_times": (C.c_int, [h, P(C.c_double), P(C.c_int64)]),
        "csp_profile_advance": (C.c_int, [h, C.c_int64, P(C.c_float), P(C.c_float)]),
        "csp_reduce_field_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int64, C.c_int32, C.c_double,
                                               C.c_void_p, C.c_void_p]),
        "csp_mlp_init": (None, [C.c_uint64, P(C.c_float)]),
        "csp_mlp_train": (C.c_int, [h, C.c_int32, P(csp_mlp_config), P(C.c_float), P(csp_mlp_report)]),
        "csp_mlp_harvest": (C.c_int, [h, C.c_int64, C.c_uint64, C.c_int64, P(C.c_int64), P(C.c_int64)]),
        "csp_mlp_harvested": (C.c_int, [h, C.c_int64, C.c_int64, P(C.c_float), P(C.c_float)]),
        "csp_mlp_gradient": (C.c_int, [P(C.c_float), P(C.c_float), P(C.c_float), C.c_int64, P(C.c_float),
                                       P(C.c_float)]),
        "csp_mlp_forward": (C.c_int, [P(C.c_float), P(C.c_float), C.c_int64, C.c_int32, P(C.c_float)]),
        "csp_set_surrogate": (C.c_int, [h, P(C.c_float), C.c_double]),
        "csp_surrogate_counts": (C.c_int, [h, P(C.c_int64), P(C.c_int64), P(C.c_int64)]),
        "csp_set_surrogate_tensor_cores": (C.c_int, [h, C.c_int32]),
        "csp_autotune": (C.c_int, [h, C.c_int32, P(csp_tune_report)]),
        "csp_destroy": (None, [h]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return sig
