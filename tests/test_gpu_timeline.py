"""Step timeline (afd_set_timeline / afd_get_timeline): the kernels of the
armed steps record the start of their first and the end of their last block
on the device clock, kinds that do not run stay empty, and recording changes
no result."""
import numpy as np
import pytest

from test_gpu_parity import small_room

pytestmark = pytest.mark.gpu


def make(pkg, storage, timeline):
    W = pkg.workloads
    vox, a, b = small_room(nx=64, ny=48, nz=40, K=2, seed=5)
    vox[-1] = np.where(vox[-1] >= 0, -1, vox[-1])  # open z+ for the PML
    vox = W.close_gaps(vox)
    nz, ny, nx = vox.shape
    sim = pkg.Simulation(mode=1, storage=storage)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    sim.SetPml(8, faces=W.FACE_ZP, ksi=W.ksi_arrays((nx, ny, nz), 8, W.FACE_ZP, kmax=6000.0))
    sim.AddSourceCell((20, 20, 10), W.gaussian_pulse(300, 32000.0))
    sim.AddMicCell((40, 30, 25))
    if timeline:
        sim.set_timeline(100, 16)
    return sim


@pytest.mark.parametrize("storage", [0, 1])
def test_timeline_records_and_changes_nothing(pkg, storage):
    out = []
    for tl in (False, True):
        sim = make(pkg, storage, tl)
        sim.Run(300)
        out.append(sim.mics())
        if tl:
            t = sim.timeline()
            K = sim.TIMELINE_KINDS
            assert t.shape == (16, len(K), 2)
            for k in ("interior_stream", "boundary", "pml_pressure", "pml_aux_z", "source_receiver"):
                s, e = t[:, K.index(k), 0], t[:, K.index(k), 1]
                assert np.all(np.isfinite(s)) and np.all(e >= s), k
            for k in ("pml_aux_x", "pml_aux_y"):  # PML on z+ only
                assert np.all(np.isnan(t[:, K.index(k)]))
            st = t[:, K.index("interior_stream"), 0]
            assert st[0] == 0.0 and np.all(np.diff(st) > 0)
            # serial plan in this chunk: the boundary kernel follows the
            # streaming kernel, the auxiliary update the PML pressure
            assert np.all(t[:, K.index("boundary"), 0] >= t[:, K.index("interior_stream"), 1])
            assert np.all(t[:, K.index("pml_aux_z"), 0] >= t[:, K.index("pml_pressure"), 1])
        sim.close()
    assert np.array_equal(out[0], out[1])


def test_timeline_off_and_arguments(pkg):
    sim = make(pkg, 0, False)
    sim.Run(50)
    assert sim.timeline().shape[0] == 0
    with pytest.raises(pkg.AfdError):
        sim.set_timeline(0, 5000)
    sim.set_timeline(10, 4)  # steps already done: nothing recorded
    sim.Run(20)
    assert np.all(np.isnan(sim.timeline()))
    sim.close()
