"""z-slab decomposition on one GPU: the grid split into two and three
slabs, each a simulation of its planes plus two halo planes, stepped in
halves with the halo planes exchanged between them (slabs.run_local), equals
the undivided run bit for bit -- receivers and the whole field -- with PML
slabs that cross the slab interfaces (x+ with z+, and every face with psi
kept) and sources and receivers in different slabs."""
import numpy as np
import pytest

from test_gpu_parity import small_room

pytestmark = pytest.mark.gpu


def _room(pkg, faces):
    W = pkg.workloads
    vox, a, b = small_room(nx=72, ny=56, nz=60, K=3, seed=41)
    vox[18:30, 20:34, 40:52] = 2  # a second box, near the slab interfaces
    if faces & 32:
        vox[-1] = -1
    if faces & 16:
        vox[0] = -1
    if faces & 2:
        vox[:, :, -1] = -1
    if faces & 1:
        vox[:, :, 0] = -1
    if faces & 8:
        vox[:, -1] = -1
    if faces & 4:
        vox[:, 0] = -1
    return W.close_gaps(vox), a, b


@pytest.mark.parametrize("faces", [2 | 32, 63])
@pytest.mark.parametrize("parts", [2, 3])
def test_slabs_equal_undivided_run(pkg, faces, parts):
    W, S = pkg.workloads, pkg.slabs
    vox, a, b = _room(pkg, faces)
    nz, ny, nx = vox.shape
    ksi = W.ksi_arrays((nx, ny, nz), 8, faces, kmax=6000.0)
    steps = 260
    rng = np.random.default_rng(9)
    sources = [(0, (20, 25, 9), W.gaussian_pulse(steps, 32000.0)),
               (0, (50, 30, 47), 0.5 * rng.standard_normal(steps).astype(np.float32))]
    receivers = [(30, 28, 5), (40, 20, 20), (33, 30, 29), (33, 30, 30), (60, 40, 45), (10, 10, 55)]

    ref = pkg.Simulation(mode=1, graphs=0)
    ref.SetModel(pkg.Model.from_voxels(vox, a, b))
    ref.SetPml(8, faces=faces, ksi=ksi)
    for _, cell, sig in sources:
        ref.AddSourceCell(cell, sig)
    for r in receivers:
        ref.AddMicCell(r)
    ref.Run(steps)
    want, wfield = ref.mics(), ref.field()
    psi_on = bool(faces & 3 and faces & 12 and faces & 48)
    ref.close()

    plist = [S.make_part(pkg, vox, a, b, lo, hi, nz, sources, receivers, pml=(8, faces, ksi))
             for lo, hi in S.split_planes(nz, parts)]
    S.run_local(plist, steps, faces, psi_on)
    got = S.gather_receivers(plist, len(receivers), steps)
    field = np.zeros_like(wfield)
    for p in plist:
        field[p.a:p.b] = p.sim.field()[1:-1]
        assert p.sim.info().steps_done == steps
    for p in plist:
        p.sim.close()
    assert np.abs(want).max() > 0
    assert np.array_equal(got, want)
    assert np.array_equal(field[1:-1], wfield[1:-1])


def test_slab_arguments_are_checked(pkg):
    sim = pkg.Simulation(mode=0)
    with pytest.raises(pkg.AfdError):
        sim.set_slab(3, 40)  # REF scheme
    sim.close()
    sim = pkg.Simulation(mode=1)
    sim.SetMinSize(0.6, 0.6, 0.6)
    with pytest.raises(pkg.AfdError):
        sim.step_phase(2)  # no open step
    sim.step_phase(1)
    with pytest.raises(pkg.AfdError):
        sim.step_phase(1)  # phase 2 is due
    sim.step_phase(2)
    with pytest.raises(pkg.AfdError):
        sim.halo(0, 0, 0, 0, 1)  # buffer too small
    sim.close()
