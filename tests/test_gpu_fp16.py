"""FP16 field storage (AFD_STORE_FP16, FIXED scheme): the CUDA path against
the FP16-storage restatement in oracle/afd_oracle.c bit for bit, and the
receiver error of the 160x120x100 workload over 20000 steps against the
FP64 restatement and against the FP32 path, as a dB bound.

Bounds (relative L2 over all receiver samples, 20 log10):
  FP16 vs FP64   <= -40 dB over all receivers, <= -35 dB for each one
  FP16 vs FP32   <= -40 dB
  FP32 vs FP64   <= -80 dB (the plain form's own error, for comparison)
Measured when the bounds were set: -45.2 dB (worst receiver -39.6 dB) for
FP16 and -88.2 dB for FP32.
"""
import os

import numpy as np
import pytest

import oracle
from test_gpu_parity import rel_l2, run_gpu, small_room

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FP16 = 1


def db(got, want):
    return 20.0 * np.log10(max(rel_l2(np.asarray(got, np.float64), np.asarray(want, np.float64)), 1e-30))


def pml_room(faces, seed=7, K=3):
    import ancfield_b200.workloads as W
    vox, a, b = small_room(nx=48, ny=40, nz=36, K=K, seed=seed)
    if faces & 32:
        vox[-1] = np.where(vox[-1] >= 0, -1, vox[-1])
    if faces & 2:
        vox[:, :, -1] = -1
    vox = W.close_gaps(vox)
    nz, ny, nx = vox.shape
    ksi = W.ksi_arrays((nx, ny, nz), 8, faces, kmax=6000.0)
    return vox, a, b, ksi


@pytest.mark.parametrize("faces", [32, 2 | 32, 63])
def test_fp16_bitexact(pkg, faces):
    import ancfield_b200.workloads as W
    vox, a, b, ksi = pml_room(faces)
    nz, ny, nx = vox.shape
    sig = W.gaussian_pulse(300, 32000.0)
    srcs, rcv = [((12, 14, 10), sig)], [(24, 20, 30), (44, 20, 18), (6, 6, 6)]
    got, field, sim = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, 300, mode=1, pml=(8, faces, ksi),
                              storage=FP16)
    assert sim.info().storage == FP16
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, pml_width=8, faces=faces, ksi=ksi,
                                   sources=srcs, receivers=rcv, steps=300, want_field=True, precision="f16")
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)


@pytest.mark.parametrize("graphs,fused", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_fp16_launch_paths(pkg, graphs, fused):
    vox, a, b = small_room(K=2, seed=11)
    nz, ny, nx = vox.shape
    sig = np.random.default_rng(4).standard_normal(450).astype(np.float32)
    srcs, rcv = [((7, 8, 9), sig)], [(20, 16, 14), (1, 1, 1)]
    got, field, _ = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, 450, mode=1, graphs=graphs, fused=fused,
                            storage=FP16)
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=srcs, receivers=rcv, steps=450,
                                   want_field=True, precision="f16")
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)


def test_fp16_consecutive_runs(pkg):
    vox, a, b = small_room(K=3, seed=12)
    nz, ny, nx = vox.shape
    sig = np.random.default_rng(5).standard_normal(700).astype(np.float32)
    srcs, rcv = [((7, 8, 9), sig)], [(20, 16, 14), (30, 20, 10)]
    got, field, _ = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, None, mode=1, runs=[1, 250, 449],
                            storage=FP16)
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=srcs, receivers=rcv,
                                   runs=[1, 250, 449], want_field=True, precision="f16")
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)


def test_fp16_batch_members_keep_their_own_scales(pkg):
    """Members whose sources differ by 60 dB each equal their own run."""
    vox, a, b = small_room(K=2, seed=13)
    nz, ny, nx = vox.shape
    rng = np.random.default_rng(6)
    sigs = [g * rng.standard_normal(200).astype(np.float32) for g in (1.0, 1000.0, 1e-3)]
    cells = [(5, 5, 5), (20, 10, 12), (33, 25, 20)]
    rcv = [(20, 16, 14), (10, 20, 6)]
    sim = pkg.Simulation(mode=1, batch=3, storage=FP16)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    for m in range(3):
        sim.AddSourceCell(cells[m], sigs[m], batch=m)
    for r in rcv:
        sim.AddMicCell(r)
    sim.Run(200)
    for m in range(3):
        want, _ = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=[(cells[m], sigs[m])],
                                  receivers=rcv, steps=200, precision="f16")
        assert np.array_equal(sim.mics(batch=m), want)


def c4_sim(pkg, cfg, storage):
    sim = pkg.Simulation(mode=1, dx=cfg.dx, c=cfg.c, dt=cfg.dt, storage=storage)
    sim.SetModel(pkg.Model.from_voxels(cfg.vox, cfg.a.astype(np.float32), cfg.b.astype(np.float32)))
    sim.SetPml(cfg.pml_width, faces=cfg.pml_faces, ksi=cfg.ksi)
    sim.AddSourceCell(cfg.sources[0][0], cfg.sources[0][1])
    for r in cfg.receivers:
        sim.AddMicCell(r)
    return sim


def test_fp16_c4_error_bound(pkg):
    """160x120x100 room, 20000 steps: bit equality with the FP16 restatement
    over the first 2000 steps, and the dB bounds of the module docstring."""
    W = pkg.workloads
    d = np.load(os.path.join(HERE, "golden", "c4.npz"))
    r64 = d["rcv_f64"].astype(np.float64)
    steps = r64.shape[1]
    cfg = W.config_c1("fixed", steps=steps)
    s16 = c4_sim(pkg, cfg, FP16)
    s16.Run(steps)
    y16 = s16.mics()
    s32 = c4_sim(pkg, cfg, 0)
    s32.Run(steps)
    y32 = s32.mics()
    assert np.array_equal(y16[:, :2000], d["rcv_f16_2000"])
    e16, e32, e1632 = db(y16, r64), db(y32, r64), db(y16, y32)
    per = [db(y16[m], r64[m]) for m in range(len(r64))]
    print("FP16 vs FP64 %.1f dB (worst receiver %.1f dB), FP16 vs FP32 %.1f dB, FP32 vs FP64 %.1f dB"
          % (e16, max(per), e1632, e32))
    assert e16 <= -40.0
    assert max(per) <= -35.0
    assert e1632 <= -40.0
    assert e32 <= -80.0


def test_fp16_energy_close_to_conserved(pkg):
    """Rigid box without walls or PML: the FP64 energy of the FP16 levels
    stays within the storage rounding of its initial value."""
    sim = pkg.Simulation(mode=1, storage=FP16)
    sim.SetMinSize(0.6, 0.6, 0.6)
    pulse = np.zeros(40, np.float32)
    pulse[:5] = [0.2, 1.0, 0.5, -0.3, 0.1]
    sim.AddSourceCell((16, 16, 16), pulse)
    sim.Run(50)
    e0 = sim.energy()
    sim.Run(400)
    e1 = sim.energy()
    assert e0 > 0
    assert abs(e1 - e0) / e0 < 1e-2


def test_fp16_unstable_run_is_reported(pkg):
    """A time step above the stability limit grows until the FP16 range is
    left; the kernels flag it and Run raises (no fault, no NaN returned)."""
    vox, a, b = small_room(K=1, seed=2, obstacle=False)
    sim = pkg.Simulation(mode=1, storage=FP16, dt=2.0 * 3.125e-5)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    sim.AddSourceCell((10, 10, 10), np.ones(4, np.float32))
    sim.AddMicCell((20, 16, 14))
    with pytest.raises(pkg.AfdError) as ei:
        sim.Run(6000)
    assert ei.value.status == pkg.afd.ERR_NUMERIC
    assert "FP16" in str(ei.value)
