"""Batch sharding on the GPU (anc-field_b200/sharding.py): the members of a
sharded batch run equal their own single-source runs bit for bit (one rank
here; the gather across ranks is covered on gloo ranks in test_sharding.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_sharded_members_equal_single_source_runs(pkg):
    W = pkg.workloads
    a, b = W.passive_filters(3, 2, 81)
    vox = W.room(48, 40, 36, 63 & ~W.FACE_ZP, n_boxes=2, nmat=3, seed=82, box_min=3, box_max=7)
    nz, ny, nx = vox.shape
    srcs = W.air_cells(vox, 3, 83, margin=2, near_wall=True)
    rcvs = W.air_cells(vox, 4, 84, margin=3)
    sig = W.gaussian_pulse(300, 32000.0)
    width = 6
    ksi = W.ksi_arrays((nx, ny, nz), width, W.FACE_ZP, kmax=6000.0)

    def make_sim(batch):
        sim = pkg.Simulation(mode=1, batch=batch)
        sim.SetModel(pkg.Model.from_voxels(vox, a, b))
        sim.SetPml(width, faces=W.FACE_ZP, ksi=ksi)
        for r in rcvs:
            sim.AddMicCell(r)
        return sim

    members = [[(tuple(int(v) for v in s), sig)] for s in srcs]
    y, run_s = pkg.sharding.run_batch_sharded(pkg, make_sim, members, 300)
    assert y.shape == (3, 4, 300) and run_s > 0
    for m, s in enumerate(srcs):
        one = make_sim(1)
        one.AddSourceCell(tuple(int(v) for v in s), sig)
        one.Run(300)
        assert np.array_equal(y[m], one.mics())
        one.close()
