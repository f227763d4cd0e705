"""The streaming plan's online autotuner and the FIXED-scheme launch order
with the boundary and PML kernels beside the streaming kernel: a run long
enough to try every candidate plan (and switch plans, tile shapes among
them, between chunks) equals the serial run without graphs bit for bit, in
FP32 and FP16."""
import numpy as np
import pytest

from test_gpu_parity import small_room

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("storage", [0, 1])
def test_tuned_run_equals_serial_run(pkg, storage):
    W = pkg.workloads
    vox, a, b = small_room(nx=96, ny=72, nz=64, K=3, seed=31)
    vox[-1] = np.where(vox[-1] >= 0, -1, vox[-1])  # open z+ for the PML
    vox = W.close_gaps(vox)
    nz, ny, nx = vox.shape
    ksi = W.ksi_arrays((nx, ny, nz), 8, W.FACE_ZP, kmax=6000.0)
    sig = W.gaussian_pulse(3600, 32000.0)
    out = []
    for graphs in (1, 0):
        sim = pkg.Simulation(mode=1, graphs=graphs, storage=storage)
        sim.SetModel(pkg.Model.from_voxels(vox, a, b))
        sim.SetPml(8, faces=W.FACE_ZP, ksi=ksi)
        sim.AddSourceCell((30, 30, 20), sig)
        for r in [(50, 40, 30), (80, 20, 55), (10, 60, 10)]:
            sim.AddMicCell(r)
        sim.Run(3401)
        sim.Run(199)
        info = sim.info()
        assert bool(info.tuned) == bool(graphs)
        out.append((sim.mics(), sim.field()))
        sim.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])


@pytest.mark.parametrize("storage", [1, 0])
def test_tuned_batch_equals_serial_run(pkg, storage):
    """A 16-member batch (the 256x192x160 secondary-path room, every member
    a unit impulse at its own wall-adjacent cell): its z-chunk rule gives a
    half-depth candidate too, and a tuned run that tries every candidate
    equals the serial run without graphs bit for bit, member by member."""
    W = pkg.workloads
    cfg = W.config_c3(steps=3400)
    out = []
    for graphs in (1, 0):
        sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt, batch=16, graphs=graphs, storage=storage)
        sim.SetModel(pkg.Model.from_voxels(cfg.vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
        sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi)
        for m in range(16):
            for cell, sig in cfg.batch_sources[m]:
                sim.AddSourceCell(cell, sig, batch=m)
        for r in cfg.receivers:
            sim.AddMicCell(r)
        sim.Run(3400)
        assert bool(sim.info().tuned) == bool(graphs)
        out.append(np.stack([sim.mics(batch=m) for m in range(16)]))
        sim.close()
    assert np.array_equal(out[0], out[1])


@pytest.mark.parametrize("storage", [0, 1])
def test_every_plan_twice_equals_serial_run(pkg, storage):
    """Every streaming plan, forced with afd_set_plan and run twice from the
    start, equals the serial run without graphs bit for bit (a result that
    changed between two runs of one plan would be a race): tile shapes,
    the rule's z-chunk depth or a quarter of it, and (FP32) the boundary/PML
    pressure kernels beside the streaming kernel or in its tail warps, on
    the 16-member secondary-path batch (FP16 storage keeps a scale per
    member)."""
    W = pkg.workloads
    cfg = W.config_c3(steps=600)

    def run(graphs, plan=None):
        sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt, batch=16, graphs=graphs, storage=storage)
        sim.SetModel(pkg.Model.from_voxels(cfg.vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
        sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi)
        if plan is not None:
            sim.set_plan(**plan)
        for m in range(16):
            for cell, sig in cfg.batch_sources[m]:
                sim.AddSourceCell(cell, sig, batch=m)
        for r in cfg.receivers:
            sim.AddMicCell(r)
        sim.Run(600)
        info = sim.info()
        if plan is not None:
            assert bool(info.stream_beside) == plan.get("beside", False)
            assert (info.tile_x, info.tile_y) == plan.get("tile", (64 * (2 if storage else 1), 16))
            assert bool(info.stream_tail) == plan.get("tail", False)
        out = np.stack([sim.mics(batch=m) for m in range(16)]), sim.field(batch=7)
        sim.close()
        return out

    serial = run(0)
    wide = 2 if storage else 1  # FP16 storage doubles the tile width in cells
    plans = [dict(), dict(dz=8), dict(tile=(32 * wide, 32))]
    if not storage:
        plans += [dict(beside=True), dict(beside=True, per_sm=1), dict(tile=(128, 8), dz=8), dict(tail=True),
                  dict(tail=True, tile=(128, 8), dz=8)]
    else:
        # FP16: beside plans and the 64x32 tile with 8-plane chunks, the two
        # configurations whose runs differed before the stage-release fence
        plans += [dict(beside=True), dict(beside=True, per_sm=1), dict(tile=(64, 32), dz=16),
                  dict(tile=(64, 32), dz=8)]
    for plan in plans:
        for _ in range(2):
            got = run(1, plan)
            assert np.array_equal(got[0], serial[0]), plan
            assert np.array_equal(got[1], serial[1]), plan
