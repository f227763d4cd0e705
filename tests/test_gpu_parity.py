"""CUDA engine vs the CPU oracle (afd_oracle.c) on the same seeded inputs.

Tolerance: relative L2 <= 1e-5 over all receiver samples (the north-star
bar). The FP32 paths are additionally expected to match the oracle bit for
bit: both evaluate the reference expressions in the same order with no
multiply-add contraction.
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel_l2(got, want):
    return float(np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-30))


def small_room(nx=40, ny=32, nz=28, K=2, seed=0, obstacle=True):
    rng = np.random.default_rng(seed)
    vox = -np.ones((nz, ny, nx), np.int32)
    vox[0], vox[-1] = 0, 1
    vox[:, 0], vox[:, -1] = 2, 0
    vox[:, :, 0], vox[:, :, -1] = 1, 2
    if obstacle:
        vox[8:13, 10:16, 12:20] = 1
    a = np.zeros((3, K), np.float32)
    b = np.zeros((3, K), np.float32)
    for m in range(3):
        a[m] = rng.uniform(0.02, 0.5, K) * np.array([1.0] + [0.3] * (K - 1))
        b[m] = np.array([1.0] + list(rng.uniform(-0.4, 0.4, K - 1)))
    return vox, a, b


def run_gpu(pkg, dims, vox, a, b, sources, receivers, steps, mode=0, pml=None, runs=None, dx=0.02,
            c=340.0, dt=3.125e-5, **params):
    sim = pkg.Simulation(mode=mode, dx=dx, c=c, dt=dt, **params)
    if vox is not None:
        sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    if pml is not None:
        width, faces, ksi = pml
        sim.SetPml(width, faces=faces, ksi=ksi)
    for cell, sig in sources:
        sim.AddSourceCell(cell, sig)
    for r in receivers:
        sim.AddMicCell(r)
    for n in (runs or [steps]):
        sim.Run(n)
    return sim.mics(), sim.field(), sim


@pytest.mark.parametrize("K", [1, 2, 3, 4])
def test_ref_boundary_bitexact(pkg, K):
    vox, a, b = small_room(K=K, seed=K)
    nz, ny, nx = vox.shape
    rng = np.random.default_rng(10 + K)
    sig = rng.standard_normal(250).astype(np.float32)
    srcs = [((5, 6, 7), sig), ((30, 20, 15), 0.5 * sig[::-1].copy())]
    rcv = [(20, 12, 10), (1, 1, 1), (38, 30, 26), (14, 12, 9)]
    got, field, sim = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, 300, mode=0)
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, sources=srcs, receivers=rcv, steps=300,
                                   want_field=True)
    assert rel_l2(got, want) <= TOL
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)
    counts = sim.info().group_counts[:]
    assert counts[25] >= 1  # the X_M_Y_M_Z_M corner is exercised


def test_ref_pml_bitexact(pkg):
    vox, a, b = small_room(K=2, seed=5)
    nz, ny, nx = vox.shape
    L = 8
    prof = np.linspace(6000.0, 0.0, L).astype(np.float32)
    sig = np.random.default_rng(3).standard_normal(200).astype(np.float32)
    srcs, rcv = [((10, 10, 10), sig)], [(20, 16, 14), (3, 3, 3)]
    sim = pkg.Simulation(mode=0)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    sim.SetPml(6, profile=prof)
    for cell, s in srcs:
        sim.AddSourceCell(cell, s)
    for r in rcv:
        sim.AddMicCell(r)
    sim.Run(250)
    k = []
    for n in (nx, ny, nz):
        kk = np.zeros(n, np.float32)
        for i in range(L):
            kk[i] = prof[L - 1 - i]
            kk[n - 1 - i] = prof[L - 1 - i]
        k.append(kk)
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, sources=srcs, receivers=rcv, steps=250,
                                   pml_width=6, ksi=k, want_field=True)
    got = sim.mics()
    assert rel_l2(got, want) <= TOL
    assert np.array_equal(got, want)
    assert np.array_equal(sim.field(), wfield)


@pytest.mark.parametrize("faces", [32, 2 | 32, 63])
def test_fixed_pml_bitexact_and_fp64(pkg, faces):
    import ancfield_b200.workloads as W
    vox, a, b = small_room(nx=48, ny=40, nz=36, K=3, seed=7)
    nz, ny, nx = vox.shape
    # open the PML faces
    if faces & 32:
        vox[-1] = np.where(vox[-1] >= 0, -1, vox[-1])
    if faces & 2:
        vox[:, :, -1] = -1
    vox = W.close_gaps(vox)
    ksi = W.ksi_arrays((nx, ny, nz), 8, faces, kmax=6000.0)
    sig = W.gaussian_pulse(300, 32000.0)
    srcs, rcv = [((12, 14, 10), sig)], [(24, 20, 30), (44, 20, 18), (6, 6, 6)]
    got, field, sim = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, 300, mode=1,
                              pml=(8, faces, ksi))
    assert sim.info().n_pml_cells > 0
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, pml_width=8, faces=faces, ksi=ksi,
                                   sources=srcs, receivers=rcv, steps=300, want_field=True)
    assert rel_l2(got, want) <= TOL
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)
    w64, _ = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, pml_width=8, faces=faces, ksi=ksi,
                             sources=srcs, receivers=rcv, steps=300, precision="f64")
    assert rel_l2(got, w64) < 1e-4


@pytest.mark.parametrize("graphs,fused", [(0, 0), (1, 0), (0, 1), (1, 1)])
def test_launch_paths_agree(pkg, graphs, fused):
    vox, a, b = small_room(K=2, seed=11)
    nz, ny, nx = vox.shape
    sig = np.random.default_rng(4).standard_normal(450).astype(np.float32)
    srcs, rcv = [((7, 8, 9), sig)], [(20, 16, 14)]
    got, field, _ = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, 450, mode=1, graphs=graphs, fused=fused)
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=srcs, receivers=rcv, steps=450,
                                   want_field=True)
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)


def test_consecutive_runs(pkg):
    """Several `run` commands continue the time index (simulation.hpp:432)."""
    vox, a, b = small_room(K=3, seed=12)
    nz, ny, nx = vox.shape
    sig = np.random.default_rng(5).standard_normal(700).astype(np.float32)
    srcs, rcv = [((7, 8, 9), sig)], [(20, 16, 14), (30, 20, 10)]
    got, field, _ = run_gpu(pkg, (nx, ny, nz), vox, a, b, srcs, rcv, None, mode=0, runs=[1, 250, 449])
    want, wfield = oracle.simulate((nx, ny, nz), vox, a, b, sources=srcs, receivers=rcv, runs=[1, 250, 449],
                                   want_field=True)
    assert got.shape == (2, 700)
    assert np.array_equal(got, want)
    assert np.array_equal(field, wfield)


def test_batch_members_independent(pkg):
    """Batch members share geometry; each equals its own single run."""
    vox, a, b = small_room(K=2, seed=13)
    nz, ny, nx = vox.shape
    rng = np.random.default_rng(6)
    sigs = [rng.standard_normal(200).astype(np.float32) for _ in range(3)]
    cells = [(5, 5, 5), (20, 10, 12), (33, 25, 20)]
    rcv = [(20, 16, 14), (10, 20, 6)]
    sim = pkg.Simulation(mode=1, batch=3)
    sim.SetModel(pkg.Model.from_voxels(vox, a, b))
    for m in range(3):
        sim.AddSourceCell(cells[m], sigs[m], batch=m)
    for r in rcv:
        sim.AddMicCell(r)
    sim.Run(200)
    for m in range(3):
        want, _ = oracle.simulate((nx, ny, nz), vox, a, b, mode=1, sources=[(cells[m], sigs[m])],
                                  receivers=rcv, steps=200)
        assert np.array_equal(sim.mics(batch=m), want)


def test_rigid_box_energy_conserved(pkg):
    """Without walls or PML the SLF energy is conserved (FP64 sum on the GPU)."""
    sim = pkg.Simulation(mode=1)
    sim.SetMinSize(0.6, 0.6, 0.6)  # 32^3 grid, Dirichlet faces only
    pulse = np.zeros(40, np.float32)
    pulse[:5] = [0.2, 1.0, 0.5, -0.3, 0.1]
    sim.AddSourceCell((16, 16, 16), pulse)
    sim.Run(50)
    e0 = sim.energy()
    sim.Run(400)
    e1 = sim.energy()
    assert e0 > 0
    assert abs(e1 - e0) / e0 < 1e-5


@pytest.mark.parametrize("storage", [0, 1])
def test_walled_box_energy(pkg, storage):
    """FIXED scheme, box-shaped room in one-cell walls, no PML: the GPU's
    FP64 energy equals the numpy restatement of the weighted energy on the
    same two levels, is constant for rigid walls and never increases for
    passive one-coefficient LRS walls."""
    from test_energy_weights import PULSE, walled_box, weighted_energy
    vox = walled_box(40, 32, 28)
    solid = vox != -1
    for a, rigid in ((np.zeros((3, 1), np.float32), True),
                     (np.array([[0.15], [0.4], [0.25]], np.float32), False)):
        sim = pkg.Simulation(mode=1, storage=storage)
        sim.SetModel(pkg.Model.from_voxels(vox, a, np.ones((3, 1), np.float32)))
        sim.AddSourceCell((12, 10, 9), PULSE)
        sim.Run(40)
        lam2 = float(sim.info().lambda2)
        energies = []
        for k in range(10):
            f0 = sim.field()
            sim.Run(1)
            e = sim.energy()
            if k in (0, 9):
                want = weighted_energy(sim.field(), f0, solid, lam2)
                assert abs(e - want) <= 1e-9 * want
            energies.append(e)
            sim.Run(39)
        sim.close()
        e = np.array(energies)
        assert e[0] > 0
        tol = 1e-6 if storage == 0 else 1e-2  # FP16 levels: storage rounding
        if rigid:
            assert np.ptp(e) / e[0] < tol
        else:
            assert np.all(e[1:] <= e[:-1] * (1 + tol))
            assert e[-1] < 0.1 * e[0]
