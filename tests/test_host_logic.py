"""Host-side logic without a GPU: seeded workloads, and the multi-rank
timing reduction of bench.py over a world of two gloo ranks."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_filters_are_stable_and_passive(pkg):
    W = pkg.workloads
    for K in (1, 2, 3, 4, 6):
        a, b = W.passive_filters(5, K, seed=K)
        assert (W.admittance_real_min(a, b) >= 0).all()
        if K > 1:
            assert max(np.abs(np.roots(b[m])).max() for m in range(5)) < 1.0


def test_rooms_are_physical_and_seeded(pkg):
    W = pkg.workloads
    v1 = W.room(60, 50, 40, 63, n_boxes=6, nmat=3, seed=9, box_min=3, box_max=12)
    v2 = W.room(60, 50, 40, 63, n_boxes=6, nmat=3, seed=9, box_min=3, box_max=12)
    assert np.array_equal(v1, v2)
    assert not W._unphysical(v1 != -1).any()
    m = pkg.Model.from_voxels(v1, np.ones((3, 2), np.float32), np.ones((3, 2), np.float32))
    assert m.classify().sum() > 0


def test_config_builders(pkg):
    W = pkg.workloads
    c1 = W.config_c1()
    assert c1.dims == (160, 120, 100) and c1.pml_faces == W.FACE_ZP and c1.pml_width == 12
    assert len(c1.receivers) == 8 and c1.a.shape == (3, 2)
    lam = c1.c * c1.dt / c1.dx
    assert abs(lam - 0.99 / np.sqrt(3)) < 1e-12
    c3 = W.config_c3(dims=(64, 48, 40))
    assert len(c3.batch_sources) == 16 and len(c3.receivers) == 16
    for srcs in c3.batch_sources:
        (x, y, z), sig = srcs[0]
        assert c3.vox[z, y, x] == -1 and sig[0] == 1.0
    noise = W.band_noise(20000, 24000.0, seed=1)
    assert abs(np.sqrt(np.mean(noise.astype(np.float64) ** 2)) - 1.0) < 1e-3
    spec = np.abs(np.fft.rfft(noise))
    f = np.fft.rfftfreq(len(noise), 1 / 24000.0)
    assert spec[(f > 4000)].mean() < 0.02 * spec[(f > 100) & (f < 1900)].mean()


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    m = bench.max_over_ranks(1.5 + rank)
    out[rank] = m
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert dict(out) == {0: 2.5, 1: 2.5}


def test_replica_rate():
    sys.path.insert(0, ROOT)
    import bench
    # two replicas of 1e6 cells, 100 steps, slowest rank 10 ms -> 2e10 cells/s
    assert bench.replica_rate(1e6, 100, 2, 10.0) == pytest.approx(20000.0)


def test_pack_rooms_places_rooms_without_overlap(pkg):
    W = pkg.workloads
    rooms = [W.room(nx, ny, nz, 63 & ~W.FACE_ZP, n_boxes=0, nmat=2, seed=k)
             for k, (nx, ny, nz) in enumerate([(20, 16, 12), (14, 22, 9), (30, 10, 15), (12, 12, 12)])]
    packed, offsets = W.pack_rooms(rooms, filler=1)
    gz, gy, gx = packed.shape
    assert gz == max(r.shape[0] for r in rooms)
    boxes = []
    for r, (ox, oy, oz) in zip(rooms, offsets):
        nz, ny, nx = r.shape
        assert oz + nz == gz  # top-aligned: every open z+ face on the grid's z+ face
        assert np.array_equal(packed[oz:oz + nz, oy:oy + ny, ox:ox + nx], r)
        boxes.append((ox, ox + nx, oy, oy + ny))
    for i in range(len(boxes)):
        for j in range(i + 1, len(boxes)):
            a, b = boxes[i], boxes[j]
            assert a[1] <= b[0] or b[1] <= a[0] or a[3] <= b[2] or b[3] <= a[2]
    # every air cell of the packed grid belongs to one room
    assert (packed == -1).sum() == sum((r == -1).sum() for r in rooms)
