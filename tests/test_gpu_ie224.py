"""Known-answer pin against the reference's shipped results: the ie224
impulse responses of examples/ie224-impulse-results, which the reference's
OpenCL kernels produced on a GPU (examples/ie224-impulse.py: model
examples/models/ie224, 416x160x576 cells, 1.06 M boundary faces, K = 1).

The fixture (tests/golden/ie224.npz, made by make_ie224.py) holds the
voxel grid, the filters and the first 4000 samples of the 14 recordings,
plus the reference's own kernels' output for the noise run (2000 steps,
oracle/_ref on the CPU, ie224_ref_noise2000.npz).

Measured: the first 1200 samples (direct sound and the first wall
reflections) agree with the recordings to about 1.2e-6 relative L2, the
level of their 6-significant-digit text. Later the recordings drift away
(7e-5 over samples 1200-2000, about 6e-4 over 4000); the reference's
shipped kernels show the same drift (this engine matches them bit for bit
on the full case), and a build with multiply-add contraction gives the
same figures, so the recordings were made by a model or code state other
than the shipped one. Bars: bit equality with the shipped kernels; 5e-6
on samples 0-1200 and 1e-3 over 4000 against the recordings.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
N = 4000
MICS = [(4, 1.6, 5.3), (4, 1.6, 4.5), (4, 1.6, 6.5), (3, 1.6, 5.5), (5, 1.6, 5.5), (4, 0.6, 5.5), (4, 2.6, 5.5)]
SOURCES = {"noise": (4, 1.6, 1.0), "actuator": (4, 1.6, 5.5)}
EARLY_TOL = 5e-6   # samples 0-1200: text-rounding level
TOTAL_TOL = 1e-3   # samples 0-4000: the recordings' drift (see above)


def impulse(bw, length, fs):
    """Band-limited unit impulse at index 1: Kaiser-window low-pass FIR with an
    80 dB stop band and a 100 Hz transition (anc_field_py/ancutil.py:49-79)."""
    from scipy import signal
    nyq = fs / 2.0
    n, beta = signal.kaiserord(80.0, 100.0 / nyq)
    taps = signal.firwin(n, bw / nyq, window=("kaiser", beta))
    x = np.zeros(length)
    x[1] = 1.0
    return signal.lfilter(taps, 1.0, x)


@pytest.fixture(scope="module")
def ie224():
    d = np.load(os.path.join(HERE, "golden", "ie224.npz"))
    nx, ny, nz = (int(v) for v in d["dims"])
    vox = np.repeat(d["rle_values"].astype(np.int32), d["rle_lengths"]).reshape(nz, ny, nx)
    return d, vox


@pytest.mark.parametrize("run", ["noise", "actuator"])
def test_ie224_recordings(pkg, ie224, run):
    d, vox = ie224
    sim = pkg.Simulation()  # reference constants, REF semantics
    sim.SetModel(pkg.Model.from_voxels(vox, d["a"], d["b"]))
    assert sim.info().n_boundary == 1056333 + 6760 + 22
    sim.AddSource(SOURCES[run], (5 * impulse(2000, N, 32000)).astype(np.float32))
    for m in MICS:
        sim.AddMic(m)
    sim.Run(N)
    got = sim.mics().astype(np.float64)
    want = d[run]
    errs = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
    print(run, "relative L2 per microphone:", " ".join("%.2e" % e for e in errs))
    early = np.linalg.norm(got[:, :1200] - want[:, :1200]) / np.linalg.norm(want[:, :1200])
    total = np.linalg.norm(got - want) / np.linalg.norm(want)
    print(run, "relative L2 samples 0-1200: %.2e, 0-4000: %.2e" % (early, total))
    assert early < EARLY_TOL, early
    assert total < TOTAL_TOL, total
    if run == "noise":
        ref = np.load(os.path.join(HERE, "golden", "ie224_ref_noise2000.npz"))["rcv"]
        assert np.array_equal(got[:, :2000].astype(np.float32), ref)
    # the first arrival is where the shipped data has it
    first = np.argmax(np.abs(want) > 1e-6, axis=1)
    assert np.array_equal(np.argmax(np.abs(got) > 1e-6, axis=1), first)
