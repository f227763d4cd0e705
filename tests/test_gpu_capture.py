"""Headless visualisation (afd_set_capture / afd_get_frames): the plane
copied on the device after every `every`-th step of each run, the way the
reference copies the y plane after every third step for its MJPEG stream
(simulation.hpp:393-400, copy_plane.cl:29-34). Frames are checked against
the oracle's field after the same number of steps, bit for bit."""
import numpy as np
import pytest

import oracle
from test_gpu_parity import small_room

pytestmark = pytest.mark.gpu


def sim_for(pkg, vox, a, b, sig, **params):
    sim = pkg.Simulation(mode=1, **params)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    sim.AddSourceCell((12, 14, 10), sig)
    return sim


def oracle_plane(vox, a, b, sig, steps, axis, index):
    nz, ny, nx = vox.shape
    _, f = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=[((12, 14, 10), sig)], receivers=[],
                           steps=steps, want_field=True)
    return {0: f[:, :, index], 1: f[:, index, :], 2: f[index, :, :]}[axis]


@pytest.mark.parametrize("axis,index", [(1, 10), (0, 7), (2, 20)])
def test_frames_follow_the_run_local_step_rule(pkg, axis, index):
    vox, a, b = small_room(K=2, seed=21)
    sig = np.random.default_rng(1).standard_normal(40).astype(np.float32)
    sim = sim_for(pkg, vox, a, b, sig)
    sim.set_capture(axis, index, every=3, max_frames=16)
    sim.Run(5)
    sim.Run(7)
    frames, steps = sim.frames()
    # run 1 (steps 0-4): run-local 0, 3; run 2 (steps 5-11): run-local 0, 3, 6
    assert list(steps) == [0, 3, 5, 8, 11]
    for fr, g in zip(frames, steps):
        assert np.array_equal(fr, oracle_plane(vox, a, b, sig, int(g) + 1, axis, index))
    assert np.array_equal(frames[-1], sim.plane(axis, index))


def test_ring_keeps_the_newest_frames(pkg):
    vox, a, b = small_room(K=2, seed=22)
    sig = np.random.default_rng(2).standard_normal(40).astype(np.float32)
    sim = sim_for(pkg, vox, a, b, sig)
    sim.set_capture(1, 12, every=2, max_frames=3)
    sim.Run(20)
    frames, steps = sim.frames()
    assert list(steps) == [14, 16, 18]
    assert np.array_equal(frames[-1], oracle_plane(vox, a, b, sig, 19, 1, 12))


def test_capture_with_fp16_storage_and_batch(pkg):
    vox, a, b = small_room(K=2, seed=23)
    sig = np.random.default_rng(3).standard_normal(40).astype(np.float32)
    sim = pkg.Simulation(mode=1, storage=1, batch=2)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    sim.AddSourceCell((12, 14, 10), sig, batch=0)
    sim.AddSourceCell((20, 10, 8), 100.0 * sig, batch=1)
    sim.set_capture(1, 9, every=4, max_frames=8, batch=1)
    sim.Run(10)
    frames, steps = sim.frames()
    assert list(steps) == [0, 4, 8]
    sim.Run(1)  # run-local step 0 of a new run: captured
    frames2, steps2 = sim.frames()
    assert list(steps2) == [0, 4, 8, 10]
    assert np.array_equal(frames2[-1], sim.plane(1, 9, batch=1))


def test_capture_off_and_bad_plane(pkg):
    vox, a, b = small_room(K=2, seed=24)
    sig = np.ones(4, np.float32)
    sim = sim_for(pkg, vox, a, b, sig)
    sim.set_capture(1, 500, every=2)
    with pytest.raises(pkg.AfdError) as ei:
        sim.Run(4)
    assert ei.value.status == pkg.afd.ERR_ARG
    sim.set_capture(1, 5, every=0)
    sim.Run(4)
    frames, steps = sim.frames()
    assert len(frames) == 0
