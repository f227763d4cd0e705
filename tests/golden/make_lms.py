"""Generates lms.npz: known answers of the reference's LMS impulse-response
estimator, EstimateIr of anc_field_py/ancutil.py:24-37 (16 epochs of
sample-serial LMS, FP64), imported from the reference tree and run on
seeded inputs. Each case stores its input, output, taps N, step size mu
and the returned weights.

Usage (needs the reference tree):  python tests/golden/make_lms.py
"""
import importlib.util
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("ANC_FIELD_REFERENCE", "/root/reference"), "anc_field_py", "ancutil.py")

# (name, input length, output length, taps, mu, seed, kind)
CASES = [("fir4", 400, 400, 16, 1e-3, 1, "white"), ("odd", 257, 257, 33, 5e-3, 2, "white"),
         ("short_out", 300, 250, 12, 2e-3, 3, "white"), ("room", 2000, 2000, 128, 1e-3, 4, "colored")]


def case_inputs(n_in, n_out, N, seed, kind):
    rng = np.random.default_rng(seed)
    x = rng.standard_normal(n_in)
    if kind == "colored":
        x = np.convolve(x, [1.0, 0.6, 0.2])[:n_in]
    h = rng.standard_normal(N) * np.exp(-np.arange(N) / (N / 4))
    y = np.convolve(x, h)[:n_out] + 1e-3 * rng.standard_normal(n_out)
    return x, y


def main():
    spec = importlib.util.spec_from_file_location("ancutil", REF)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    out = {}
    for name, n_in, n_out, N, mu, seed, kind in CASES:
        x, y = case_inputs(n_in, n_out, N, seed, kind)
        out[name + "_x"] = x
        out[name + "_y"] = y
        out[name + "_w"] = mod.EstimateIr(x, y, N, mu)
        out[name + "_meta"] = np.array([N, mu])
        print(name, out[name + "_w"][:4])
    np.savez_compressed(os.path.join(HERE, "lms.npz"), **out)


if __name__ == "__main__":
    main()
