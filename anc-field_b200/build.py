"""Builds the FDTD core in-tree for sm_100a.

Outputs (git-ignored, shipped with the source tree):
  lib/libafd.so     the C-ABI library of include/afd.h (static CUDA runtime)
  bin/anc-field     the command-line drop-in for the reference executable

Usage: python build.py [--force] [--verbose]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "build")
LIB = os.path.join(HERE, "lib")
BIN = os.path.join(HERE, "bin")
INC = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
# -fmad=false: no multiply-add contraction, so every rounding of the step
# arithmetic is the one the reference expression order gives.
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-fmad=false", "--expt-relaxed-constexpr",
              "-Xcompiler", "-fPIC,-ffp-contract=off", "-I" + INC] + ARCH
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-Wall", "-I" + INC]

CU_SOURCES = ["engine.cu", "filters.cu", "mlp.cu", "lms.cu", "geometry.cu", "selftest.cu"]
CXX_SOURCES = ["model.cpp", "api.cpp"]
HEADERS = ["device.cuh", "engine.hpp", "model.hpp", "filters.hpp", "fused.cuh", "tc.cuh", "geometry.hpp"]


def _nvcc():
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.exists(d) and os.path.getmtime(d) > t for d in deps)


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd[:3]) + " ...")
    if verbose and (r.stdout or r.stderr):
        sys.stderr.write(r.stdout + r.stderr)
    return r


def build(force=False, verbose=False):
    """Compiles every CUDA and C++ source; returns the library path."""
    for d in (OBJ, LIB, BIN):
        os.makedirs(d, exist_ok=True)
    hdrs = [os.path.join(SRC, h) for h in HEADERS] + [os.path.join(INC, "afd.h"), os.path.join(INC, "afd_surrogate.h"), os.path.join(INC, "afd_lms.h")]
    objs = []
    nvcc = _nvcc()
    for s in CU_SOURCES:
        src = os.path.join(SRC, s)
        if not os.path.exists(src):
            continue
        o = os.path.join(OBJ, s + ".o")
        if force or _stale(o, [src] + hdrs):
            _run([nvcc] + NVCC_FLAGS + ["-Xptxas", "-v", "-c", src, "-o", o], verbose)
        objs.append(o)
    for s in CXX_SOURCES:
        src = os.path.join(SRC, s)
        o = os.path.join(OBJ, s + ".o")
        if force or _stale(o, [src] + hdrs):
            _run(["g++"] + CXX_FLAGS + ["-c", src, "-o", o], verbose)
        objs.append(o)
    lib = os.path.join(LIB, "libafd.so")
    if force or _stale(lib, objs):
        _run([nvcc, "-shared", "-o", lib] + objs + ARCH + ["-Xcompiler", "-fPIC"], verbose)
    exe = os.path.join(BIN, "anc-field")
    repl_src = [os.path.join(SRC, "repl_main.cpp"), os.path.join(SRC, "model.cpp")]
    if force or _stale(exe, repl_src + [lib] + hdrs):
        _run(["g++"] + CXX_FLAGS + repl_src + ["-o", exe, "-L" + LIB, "-lafd",
                                                "-Wl,-rpath,$ORIGIN/../lib"], verbose)
    return lib


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="--verbose" in sys.argv)
    print("built", os.path.join(LIB, "libafd.so"), os.path.join(BIN, "anc-field"))
