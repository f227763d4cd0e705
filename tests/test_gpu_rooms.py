"""Uneven rooms in one launch: rooms of different sizes packed into one grid
(workloads.pack_rooms), advanced by one simulation, each equal bit for bit
to its own run (the oracle's, FIXED scheme with a z+ PML per room). The
streaming kernel skips the work items that only hold the solid filler."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu


def test_packed_rooms_equal_their_own_runs(pkg):
    W = pkg.workloads
    a, b = W.passive_filters(3, 2, 77)
    rooms, parts = [], []
    for k, (nx, ny, nz) in enumerate([(40, 32, 28), (56, 44, 36), (36, 60, 30)]):
        vox = W.room(nx, ny, nz, 63 & ~W.FACE_ZP, n_boxes=1, nmat=3, seed=40 + k, box_min=4, box_max=8)
        src = W.air_cells(vox, 1, 50 + k, margin=2, near_wall=True)[0]
        rcv = W.air_cells(vox, 3, 60 + k, margin=3)
        rooms.append(vox)
        parts.append((vox, src, rcv))
    packed, offsets = W.pack_rooms(rooms)
    gz, gy, gx = packed.shape
    width = 6
    sig = W.gaussian_pulse(220, 32000.0)
    sim = pkg.Simulation(mode=1)
    sim.SetModel(pkg.Model.from_voxels(packed, a, b))
    sim.SetPml(width, faces=W.FACE_ZP, ksi=W.ksi_arrays((gx, gy, gz), width, W.FACE_ZP, kmax=6000.0))
    for (vox, s, r), (ox, oy, oz) in zip(parts, offsets):
        sim.AddSourceCell((s[0] + ox, s[1] + oy, s[2] + oz), sig)
        for q in r:
            sim.AddMicCell((q[0] + ox, q[1] + oy, q[2] + oz))
    sim.Run(220)
    got = sim.mics()
    for k, ((vox, s, r), (ox, oy, oz)) in enumerate(zip(parts, offsets)):
        nz, ny, nx = vox.shape
        want, _ = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, pml_width=width, faces=W.FACE_ZP,
                                  ksi=W.ksi_arrays((nx, ny, nz), width, W.FACE_ZP, kmax=6000.0),
                                  sources=[(s, sig)], receivers=r, steps=220)
        assert np.abs(want).max() > 0
        assert np.array_equal(got[3 * k:3 * k + 3], want), k


def test_thick_solid_regions_are_skipped_without_changing_results(pkg):
    """One room inside a grid that is mostly solid: the run with the work
    list equals the oracle's run of the whole grid on every air cell."""
    W = pkg.workloads
    a, b = W.passive_filters(2, 2, 78)
    inner = W.room(40, 36, 30, 63, n_boxes=1, nmat=2, seed=45, box_min=4, box_max=8)
    vox = np.zeros((46, 120, 200), np.int32)
    vox[8:38, 40:76, 100:140] = inner
    sig = W.gaussian_pulse(150, 32000.0)
    src = (112, 50, 20)
    rcv = [(120, 60, 25), (135, 70, 12)]
    sim = pkg.Simulation(mode=1)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    sim.AddSourceCell(src, sig)
    for r in rcv:
        sim.AddMicCell(r)
    sim.Run(150)
    want, field = oracle.simulate((200, 120, 46), vox, a, b, mode=1, sources=[(src, sig)], receivers=rcv,
                                  steps=150, want_field=True)
    assert np.array_equal(sim.mics(), want)
    air = vox == -1
    assert np.array_equal(sim.field()[air], field[air])
