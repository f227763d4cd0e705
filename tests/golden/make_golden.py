"""Generates the golden fixtures in this directory from the reference's own
kernel sources compiled on the CPU (oracle/_ref, see oracle/ref_harness.c).

Each case is a small seeded room run in the reference semantics; the
fixture holds the inputs' seeds and sizes (cases.json) and the receiver
signals plus the final pressure field (golden_<case>.npz). The tests rebuild
the inputs from cases.json and compare the oracle restatement with these
outputs bit for bit.

Usage (needs oracle/_ref built, i.e. the reference tree present):
    python tests/golden/make_golden.py
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
sys.path.insert(0, HERE)

import oracle  # noqa: E402
from cases import CASES, build_case  # noqa: E402


def main():
    if not oracle.available("ref", "f32"):
        raise SystemExit("oracle/_ref is not built (needs the reference tree)")
    for name, spec in CASES.items():
        inp = build_case(spec)
        out = {}
        for prec in ("f32", "f64"):
            rcv, field = oracle.simulate(impl="ref", precision=prec, want_field=True, **inp)
            out["rcv_" + prec] = rcv
            out["field_" + prec] = field
        np.savez_compressed(os.path.join(HERE, "golden_%s.npz" % name), **out)
        print(name, {k: v.shape for k, v in out.items()})
    with open(os.path.join(HERE, "cases.json"), "w") as f:
        json.dump(CASES, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
