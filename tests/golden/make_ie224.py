"""Builds tests/golden/ie224.npz from the reference's shipped ie224 example:
the voxel grid and filters of examples/models/ie224 (loaded with this
library's Kerkythea reader, run-length encoded), and the first N samples of
the 14 receiver recordings in examples/ie224-impulse-results, which the
reference produced on a GPU with examples/ie224-impulse.py (two runs: noise
source and actuator, seven microphones each).

It also runs the reference's own kernels (oracle/_ref, CPU, REF semantics)
on the noise-source case for 2000 steps and stores their receiver signals
as ie224_ref_noise2000.npz (a few minutes on 8 cores).

Usage: python tests/golden/make_ie224.py [reference_root]
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
N = 4000
MICS = ["error", "reference_front", "reference_back", "reference_left", "reference_right",
        "reference_bottom", "reference_top"]


def load_pkg():
    spec = importlib.util.spec_from_file_location("ancfield_b200", os.path.join(ROOT, "anc-field_b200", "__init__.py"),
                                                  submodule_search_locations=[os.path.join(ROOT, "anc-field_b200")])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["ancfield_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main(ref=sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ANC_FIELD_REFERENCE", "/root/reference")):
    pkg = load_pkg()
    m = pkg.Model.load_kerkythea(os.path.join(ref, "examples", "models", "ie224", "model.xml"), 0.02)
    vox = m.voxels().ravel()
    change = np.flatnonzero(np.diff(vox)) + 1
    starts = np.concatenate([[0], change])
    values = vox[starts].astype(np.int8)
    lengths = np.diff(np.concatenate([starts, [vox.size]])).astype(np.int64)
    a, b = m.coefs()
    rec = {}
    for src in ("noise", "actuator"):
        rows = []
        for mic in MICS:
            path = os.path.join(ref, "examples", "ie224-impulse-results", "ie224-%s-to-%s.dat" % (src, mic))
            with open(path) as f:
                rows.append([float(next(f)) for _ in range(N)])
        rec[src] = np.array(rows, np.float64)
    (nx, ny, nz), _, _ = m.dims
    np.savez_compressed(os.path.join(HERE, "ie224.npz"), dims=np.array([nx, ny, nz]), rle_values=values,
                        rle_lengths=lengths, a=a, b=b, names=np.array(m.material_names()),
                        noise=rec["noise"], actuator=rec["actuator"])
    print("runs", len(values), "dims", (nx, ny, nz), "recordings", rec["noise"].shape)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    import test_gpu_ie224 as T
    n = 2000
    src = (5 * T.impulse(2000, T.N, 32000)).astype(np.float32)[:n]
    cell = lambda p: tuple(int(np.float32(v) / np.float32(0.02)) for v in p)
    rcv, _ = oracle.simulate(grid=(nx, ny, nz), vox=m.voxels(), a=a.astype(np.float64), b=b.astype(np.float64),
                             mode=0, sources=[(cell(T.SOURCES["noise"]), src)],
                             receivers=[cell(p) for p in T.MICS], steps=n, impl="ref")
    np.savez_compressed(os.path.join(HERE, "ie224_ref_noise2000.npz"), rcv=rcv)


if __name__ == "__main__":
    main()
