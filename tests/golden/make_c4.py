"""Generates c4.npz: the receiver signals of the 160x120x100 room of the
FP16-storage workload (FIXED scheme, K = 2 wall filters, 12-cell PML on z+,
Gaussian-modulated 500 Hz pulse, 8 receivers, 20000 steps) from the FP64
restatement (oracle/afd_oracle.c built with double), stored as float32
(the storage rounding, about -140 dB, is far below the bounds the tests
apply), and the first 2000 steps of the FP16-storage restatement, against
which the GPU's FP16 path is compared bit for bit.

Usage:  python tests/golden/make_c4.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.join(HERE, "..", "..")
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402

STEPS = 20000
EXACT_STEPS = 2000


def c4_inputs(steps):
    import __graft_entry__ as ge
    W = ge.load().workloads
    cfg = W.config_c1("fixed", steps=steps)
    return cfg, dict(grid=cfg.dims, vox=cfg.vox, a=cfg.a, b=cfg.b, dx=cfg.dx, c=cfg.c, dt=cfg.dt, mode=1,
                     pml_width=cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi, sources=cfg.sources,
                     receivers=cfg.receivers, steps=steps)


def main():
    _, kw = c4_inputs(STEPS)
    r64, _ = oracle.simulate(precision="f64", **kw)
    _, kw2 = c4_inputs(EXACT_STEPS)
    r16, _ = oracle.simulate(precision="f16", **kw2)
    np.savez_compressed(os.path.join(HERE, "c4.npz"), rcv_f64=r64.astype(np.float32), rcv_f16_2000=r16)
    print("c4.npz", r64.shape, r16.shape)


if __name__ == "__main__":
    main()
