"""Batch sharding across ranks (anc-field_b200/sharding.py): the split of
members over ranks and the order-preserving gather of the receiver blocks,
on two gloo ranks on CPU."""
import os
import socket

import numpy as np
import pytest


def test_shard_range_covers_every_item_once(pkg):
    S = pkg.sharding
    for n in (0, 1, 5, 16, 17, 255):
        for world in (1, 2, 3, 4, 8):
            seen = []
            sizes = []
            for r in range(world):
                lo, hi = S.shard_range(n, world, r)
                seen.extend(range(lo, hi))
                sizes.append(hi - lo)
            assert seen == list(range(n))
            assert max(sizes) - min(sizes) <= 1
            assert sizes[0] == max(sizes)
    with pytest.raises(ValueError):
        S.shard_range(4, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_worker(rank, world, port, n_items, out_dir):
    import sys
    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import conftest
    pkg = conftest._load_pkg()
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world)
    try:
        full = np.arange(n_items * 3 * 5, dtype=np.float32).reshape(n_items, 3, 5)
        lo, hi = pkg.sharding.shard_range(n_items, world, rank)
        got = pkg.sharding.gather_rows(full[lo:hi], n_items, world, rank)
        np.save(os.path.join(out_dir, "r%d.npy" % rank), got)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_items", [5, 16, 1])
def test_gather_rows_on_two_gloo_ranks(tmp_path, n_items):
    import torch.multiprocessing as mp
    world = 2
    mp.spawn(_gather_worker, args=(world, _free_port(), n_items, str(tmp_path)), nprocs=world, join=True)
    full = np.arange(n_items * 3 * 5, dtype=np.float32).reshape(n_items, 3, 5)
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / ("r%d.npy" % r)), full)
