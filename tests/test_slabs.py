"""z-slab decomposition (anc-field_b200/slabs.py) without a GPU: the plane
split, the pairing of the halo transfers between ranks, and whole exchanges
over torch.distributed on two and three gloo ranks (and in one process)
driving a numpy stand-in of the engine whose steps have the engine's
dependency structure across planes: a decomposed run must equal the
undivided one exactly."""
import ctypes
import os
import socket
import types

import numpy as np
import pytest


def test_split_planes_covers_the_interior_once(pkg):
    S = pkg.slabs
    for nz in (3, 4, 10, 33, 320):
        for parts in (1, 2, 3, 5):
            if nz - 2 < parts:
                with pytest.raises(ValueError):
                    S.split_planes(nz, parts)
                continue
            r = S.split_planes(nz, parts)
            assert r[0][0] == 1 and r[-1][1] == nz - 1
            assert all(r[k][1] == r[k + 1][0] for k in range(parts - 1))
            sizes = [b - a for a, b in r]
            assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("world", [2, 3, 4])
@pytest.mark.parametrize("faces,psi_on", [(2 | 32, False), (63, True), (0, False)])
def test_halo_transfers_pair_up(pkg, world, faces, psi_on):
    """Every send has the matching receive on its peer, in the same order
    per (sender, receiver) pair; the data goes from the sender's own end
    plane into the receiver's halo on the facing side."""
    S = pkg.slabs
    for which in ("A", "B"):
        plans = [S.halo_plan(r, world, faces, psi_on, which) for r in range(world)]
        for src in range(world):
            for dst in range(world):
                sent = [(side, f) for op, peer, side, f in plans[src] if op == "send" and peer == dst]
                recv = [(side, f) for op, peer, side, f in plans[dst] if op == "recv" and peer == src]
                assert [f for _, f in sent] == [f for _, f in recv]
                assert all(s == 1 - r for (s, _), (r, _) in zip(sent, recv))
                if abs(src - dst) != 1:
                    assert not sent
        down, up = S.exchange_fields(faces, psi_on, which)
        assert S.PRESSURE in down
        if which == "A":
            assert up == [] and (S.PSI in down) == psi_on
        else:
            assert up == [S.PRESSURE]


class FakeSim:
    """numpy stand-in for one part: pressure u, auxiliary fields v[0..2] and
    psi over local planes 0..nl-1 (planes 0 and nl-1 halos). Phase 1 reads
    u at z-1, z, z+1 and the auxiliary fields at z+1; phase 2 reads the new
    u and the new psi at z and z+1 -- the reads of the engine's interior/PML
    pressure and PML auxiliary updates."""

    def __init__(self, u0, n):
        self.nl = u0.shape[0]
        self.n = n
        self.un = u0.copy()
        self.vn = [np.zeros_like(u0) for _ in range(3)]
        self.psin = np.zeros_like(u0)

    def info(self):
        return types.SimpleNamespace(nx=self.n, ny=1, batch=1)

    def prepare(self, steps):
        pass

    def step_phase(self, phase):
        own = slice(1, self.nl - 1)
        if phase == 1:
            u, ps = self.un.copy(), self.psin.copy()
            self.v = [v.copy() for v in self.vn]
            un = u.copy()
            un[own] = u[own] + 0.25 * (u[:-2] - 2 * u[own] + u[2:]) + 0.01 * self.v[0][2:] - \
                0.02 * self.v[1][2:] + 0.03 * self.v[2][2:]
            psin = ps.copy()
            psin[own] = 0.1 * un[own] + 0.5 * ps[own]
            self.un, self.psin = un, psin
        else:
            for k in range(3):
                vn = self.v[k].copy()
                vn[own] = (0.5 - 0.1 * k) * self.v[k][own] + (self.un[2:] - self.un[own]) + 0.2 * self.psin[2:]
                self.vn[k] = vn

    def halo(self, side, direction, field, ptr, cap):
        arr = self.un if field == 0 else (self.psin if field == 4 else self.vn[field - 1])
        buf = np.ctypeslib.as_array((ctypes.c_float * cap).from_address(ptr))
        z = (1 if side == 0 else self.nl - 2) if direction == 0 else (0 if side == 0 else self.nl - 1)
        if direction == 0:
            buf[:self.n] = arr[z]
        else:
            arr[z] = buf[:self.n]


def _reference(u0, steps):
    sim = FakeSim(u0, u0.shape[1])
    for _ in range(steps):
        sim.step_phase(1)
        sim.step_phase(2)
    return sim


NZ, N, STEPS = 23, 7, 9
FACES, PSI_ON = 63, True  # PML slabs on every axis: x and y slabs cross every interface


def _u0():
    rng = np.random.default_rng(4)
    u = rng.standard_normal((NZ, N)).astype(np.float32)
    u[0] = u[-1] = 0.0
    return u


def _parts(pkg, world, u0):
    return [(a, b, FakeSim(u0[a - 1:b + 1].copy(), N)) for a, b in pkg.slabs.split_planes(NZ, world)]


def _assemble(parts):
    u = np.zeros((NZ, N), np.float32)
    v = np.zeros((3, NZ, N), np.float32)
    for a, b, sim in parts:
        u[a:b] = sim.un[1:-1]
        for k in range(3):
            v[k, a:b] = sim.vn[k][1:-1]
    return u, v


@pytest.mark.parametrize("world", [1, 2, 3, 5])
def test_local_exchange_equals_undivided_run(pkg, world):
    u0 = _u0()
    parts = _parts(pkg, world, u0)
    pkg.slabs.run_local([pkg.slabs.Part(s, a, b, []) for a, b, s in parts], STEPS, FACES, PSI_ON,
                        torch_device="cpu")
    ref = _reference(u0, STEPS)
    u, v = _assemble(parts)
    assert np.array_equal(u[1:-1], ref.un[1:-1])
    for k in range(3):
        assert np.array_equal(v[k, 1:-1], ref.vn[k][1:-1])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_worker(rank, world, port, out_dir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import conftest
    pkg = conftest._load_pkg()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        a, b, sim = _parts(pkg, world, _u0())[rank]
        pkg.slabs.run_rank(pkg.slabs.Part(sim, a, b, []), STEPS, FACES, PSI_ON, rank, world, device="cpu")
        np.save(os.path.join(out_dir, "r%d.npy" % rank), np.stack([sim.un[1:-1]] + [v[1:-1] for v in sim.vn]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_rank_exchange_on_gloo_equals_undivided_run(pkg, tmp_path, world):
    import torch.multiprocessing as mp
    mp.spawn(_rank_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    ref = _reference(_u0(), STEPS)
    for r, (a, b) in enumerate(pkg.slabs.split_planes(NZ, world)):
        got = np.load(tmp_path / ("r%d.npy" % r))
        assert np.array_equal(got[0], ref.un[a:b])
        for k in range(3):
            assert np.array_equal(got[1 + k], ref.vn[k][a:b])
