"""The C-ABI library loads and exports every symbol include/csparks.h declares (no GPU
calls), and the ctypes mirror has the C struct sizes."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "csparks.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(csp_[a-z_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol(pkg):
    lib = pkg.load()
    names = declared_functions()
    assert "csp_create" in names and "csp_advance" in names
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", pkg.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert re.search(rf"\bT {n}\b", out), f"{n} not exported"


def test_struct_layout_matches_c(pkg, tmp_path):
    abi = pkg.abi
    prog = tmp_path / "sz.c"
    prog.write_text('#include <stdio.h>\n#include "csparks.h"\nint main(){printf("%zu %zu %zu %zu %zu\\n",'
                    'sizeof(csp_model),sizeof(csp_options),sizeof(csp_info),sizeof(csp_domain_species),'
                    'sizeof(csp_boundary));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I" + os.path.join(ROOT, "include"), str(prog), "-o", str(exe)], check=True)
    sizes = list(map(int, subprocess.run([str(exe)], capture_output=True, text=True).stdout.split()))
    assert sizes == [C.sizeof(abi.csp_model), C.sizeof(abi.csp_options), C.sizeof(abi.csp_info),
                     C.sizeof(abi.csp_domain_species), C.sizeof(abi.csp_boundary)]


def test_options_default_matches_reference(pkg):
    lib = pkg.load()
    o = pkg.abi.csp_options()
    lib.csp_options_default(C.byref(o))   # host-only, no CUDA call
    assert (o.h, o.dt, o.tstop, o.dt_save, o.dt_update_react, o.dt_update_stoch) == (6.0, -1.0, 10.0, 0.5, -1.0, -1.0)


def test_status_without_handle(pkg):
    lib = pkg.load()
    buf = C.create_string_buffer(64)
    assert lib.csp_status(None, buf, 64) == 0


def test_make_model_rejects_long_names(pkg, synth):
    spec = synth.tiny()
    spec = dict(spec, species=["Ca" * 20] + spec["species"][1:])
    with pytest.raises(ValueError):
        pkg.abi.make_model(spec)
