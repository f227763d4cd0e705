"""The GPU LMS estimator (include/afd_lms.h) against the reference's own
EstimateIr outputs (tests/golden/lms.npz) and the CPU restatement. The GPU
evaluates the reference recursion in blocks of 128 samples, which changes
only the order of floating-point additions: bar 1e-10 relative L2."""
import os

import numpy as np
import pytest

import lms_oracle

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TOL = 1e-10


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", ["fir4", "odd", "short_out", "room"])
def test_gpu_equals_reference_outputs(pkg, name):
    g = np.load(os.path.join(HERE, "golden", "lms.npz"))
    N, mu = g[name + "_meta"]
    got = pkg.lms.EstimateIr(g[name + "_x"], g[name + "_y"], int(N), float(mu))
    assert rel(got, g[name + "_w"]) < TOL


def test_gpu_many_tap_chunks_equals_restatement(pkg):
    """More taps than one CTA of the y0 pass handles (2048), several blocks."""
    rng = np.random.default_rng(9)
    N, steps = 3000, 700
    x = rng.standard_normal(steps)
    h = rng.standard_normal(N) * np.exp(-np.arange(N) / 300.0)
    d = np.convolve(x, h)[:steps]
    want = lms_oracle.estimate(x, d, N, 2e-4, epochs=2)
    got = pkg.lms.estimate_ir(x, d, N, 2e-4, epochs=2)
    assert rel(got, want) < TOL


def test_gpu_identifies_a_known_response(pkg):
    """Noise-free identification of a 200-tap response from 20000 samples of
    white noise: the reference's 16 passes converge to it."""
    rng = np.random.default_rng(10)
    h = rng.standard_normal(200) * np.exp(-np.arange(200) / 40.0)
    x = rng.standard_normal(20000)
    d = np.convolve(x, h)[:20000]
    w = pkg.lms.EstimateIr(x, d, 200, 1e-3)
    assert rel(w, h) < 1e-6
