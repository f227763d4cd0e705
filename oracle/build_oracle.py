"""Builds the CPU oracle (test infrastructure, never the product path).

  _build/liboracle.so   the restatement afd_oracle.c, FP32 and FP64 entry
                        points (ora_simulate_f32 / ora_simulate_f64 / ora_simulate_f16)
  _ref/libref32.so      the reference's own kernel sources compiled from
  _ref/libref64.so      where they lie (ref_harness.c), FP32 and FP64
                        (ref_simulate_f32 / ref_simulate_f64); built only
                        when the reference tree is present

Usage: python oracle/build_oracle.py [--force] [--reference DIR]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
REFERENCE = os.environ.get("ANC_FIELD_REFERENCE", "/root/reference")
FLAGS = ["-std=c11", "-O2", "-ffp-contract=off", "-fopenmp", "-fPIC", "-Wall", "-Wno-unused-function"]


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _cc(args):
    r = subprocess.run(["gcc"] + args, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stderr)
        raise RuntimeError("oracle build failed")


def build_restatement(force=False):
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "afd_oracle.c")
    out = os.path.join(BUILD, "liboracle.so")
    if force or _stale(out, [src]):
        o32 = os.path.join(BUILD, "ora32.o")
        o64 = os.path.join(BUILD, "ora64.o")
        _cc(FLAGS + ["-c", src, "-o", o32])
        _cc(FLAGS + ["-DORA_REAL=double", "-DORA_NAME=ora_simulate_f64", "-DORA_NO_F16", "-c", src, "-o", o64])
        _cc(["-shared", "-fopenmp", o32, o64, "-o", out, "-lm"])
    return out


def build_reference(force=False, reference=REFERENCE):
    ksrc = os.path.join(reference, "anc-field", "src")
    if not os.path.isdir(ksrc):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    kernels = {"LEAPFROG": "leapfrog.cl", "SOURCE": "source.cl", "MIC": "mic.cl", "PML": "pml.cl",
               "LRS1": "lrs_1.cl", "LRS2": "lrs_2.cl", "LRS3": "lrs_3.cl"}
    defs = ['-DKS_%s="%s"' % (k, os.path.join(ksrc, f)) for k, f in kernels.items()]
    src = os.path.join(HERE, "ref_harness.c")
    deps = [src, os.path.join(HERE, "classify.h")] + [os.path.join(ksrc, f) for f in kernels.values()]
    # the kernels carry a stray token after #ifndef and unused locals
    quiet = ["-w"]
    outs = []
    for name, extra in (("libref32.so", []), ("libref64.so", ["-DREF_FP64", "-DREF_NAME=ref_simulate_f64"])):
        out = os.path.join(REF_OUT, name)
        if force or _stale(out, deps):
            _cc(FLAGS + quiet + defs + extra + ["-shared", src, "-o", out, "-lm"])
        outs.append(out)
    return outs


if __name__ == "__main__":
    force = "--force" in sys.argv
    ref = REFERENCE
    if "--reference" in sys.argv:
        ref = sys.argv[sys.argv.index("--reference") + 1]
    print(build_restatement(force))
    print(build_reference(force, ref))
