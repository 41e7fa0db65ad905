"""Build libcsparks_cuda.so (sm_100a) and the calcium_sparks CLI in-tree.

    python hpc-ca-phospattern_b200/build.py [--force]

nvcc cross-compiles for sm_100a without a GPU.  Outputs go to
hpc-ca-phospattern_b200/lib and hpc-ca-phospattern_b200/bin (git-ignored, they travel
with the source tree).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC,-O2", "--expt-relaxed-constexpr"]

LIB_SOURCES = ["csp_runtime.cu", "csp_noalloc.cu"]
LIB_DEPS = ["csp_runtime.cu", "csp_noalloc.cu", "csp_device.cuh", "csp_kernels.cuh", "csp_staged.cuh", "csp_mlp.cuh",
            os.path.join("..", "..", "include", "csparks.h")]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def run(cmd):
    print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_lib(force=False):
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libcsparks_cuda.so")
    deps = [os.path.join(CSRC, d) for d in LIB_DEPS]
    if force or _stale(target, deps):
        run([NVCC] + NVFLAGS + ["-shared", "-o", target] + [os.path.join(CSRC, s) for s in LIB_SOURCES])
    return target


def build_cli(force=False):
    """bin/calcium_sparks: the reference's command line on top of the C ABI."""
    srcs = ["calcium_sparks.c", "csp_options.c", "csp_io.c", "h5lite.c"]
    if not all(os.path.exists(os.path.join(CSRC, s)) for s in srcs):
        return None
    os.makedirs(BIN, exist_ok=True)
    target = os.path.join(BIN, "calcium_sparks")
    deps = [os.path.join(CSRC, s) for s in srcs + ["h5lite.h", "csp_io.h", "csp_options.h"]]
    deps.append(os.path.join(LIB, "libcsparks_cuda.so"))
    if force or _stale(target, deps):
        run(["gcc", "-O2", "-std=gnu11", "-Wall", "-Wno-unused-result", "-I" + os.path.join(HERE, "..", "include"),
             "-o", target] + [os.path.join(CSRC, s) for s in srcs] +
            ["-L" + LIB, "-lcsparks_cuda", "-Wl,-rpath,$ORIGIN/../lib", "-lz", "-lm"])
    return target


def build_h5lite(force=False):
    """lib/libh5lite.so: the HDF5-subset reader/writer, for the Python input writers."""
    src = os.path.join(CSRC, "h5lite.c")
    if not os.path.exists(src):
        return None
    os.makedirs(LIB, exist_ok=True)
    target = os.path.join(LIB, "libh5lite.so")
    if force or _stale(target, [src, os.path.join(CSRC, "h5lite.h")]):
        run(["gcc", "-O2", "-std=gnu11", "-Wall", "-fPIC", "-shared", "-o", target, src, "-lz"])
    return target


def main(force=False):
    build_lib(force)
    build_h5lite(force)
    build_cli(force)


if __name__ == "__main__":
    main("--force" in sys.argv)
