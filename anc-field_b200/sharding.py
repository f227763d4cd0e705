"""Batch sharding across GPUs: sources (batch members) or rooms split over
the ranks of a torch.distributed job, one simulation per rank, and the
receiver arrays gathered in member order. There is no exchange during the
run; the only collective is the final gather (all_gather of equal-sized,
padded blocks, NCCL on GPUs, gloo on CPU).

The path does not couple members: member m of a sharded run equals member m
of one batched run bit for bit (every member's arithmetic is its own).
"""
import numpy as np


def shard_range(n_items, world, rank):
    """[lo, hi) of the items of `rank`: contiguous, sizes differ by at most
    one, the first n_items % world ranks take the larger share."""
    if world < 1 or not (0 <= rank < world) or n_items < 0:
        raise ValueError("bad shard arguments")
    base, extra = divmod(n_items, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def gather_rows(local, n_items, world, rank, device="cpu"):
    """The per-rank blocks local[0:hi-lo] (same trailing shape on every
    rank) joined in rank order on every rank, as a numpy array of n_items
    rows. One collective: all_gather of blocks padded to the largest shard."""
    import torch
    import torch.distributed as dist
    local = np.ascontiguousarray(local)
    lo, hi = shard_range(n_items, world, rank)
    if local.shape[0] != hi - lo:
        raise ValueError("local block has %d rows, shard %d" % (local.shape[0], hi - lo))
    if world == 1 or not (dist.is_available() and dist.is_initialized()):
        return local.copy()
    cap = shard_range(n_items, world, 0)[1]  # rank 0 holds the largest shard
    tail = local.shape[1:]
    buf = torch.zeros((cap,) + tail, dtype=torch.from_numpy(local[:0]).dtype, device=device)
    if hi > lo:
        buf[:hi - lo] = torch.from_numpy(local).to(device)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf)
    out = []
    for r in range(world):
        a, b = shard_range(n_items, world, r)
        out.append(parts[r][:b - a].cpu().numpy())
    return np.concatenate(out, axis=0)


def run_batch_sharded(pkg, make_sim, members, steps, world=1, rank=0, device="cpu"):
    """members: one list of ((i, j, k), signal) sources per batch member.
    make_sim(batch) returns a Simulation with the model, PML and receivers
    set and `batch` members; this rank adds the sources of its shard (member
    m of the shard as batch index m), runs `steps` steps and returns
    (receivers [n_members, n_receivers, steps] on every rank, the rank's own
    run seconds from CUDA events)."""
    lo, hi = shard_range(len(members), world, rank)
    n = hi - lo
    sim = make_sim(max(n, 1))
    for m in range(n):
        for cell, sig in members[lo + m]:
            sim.AddSourceCell(cell, sig, batch=m)
    sim.prepare(steps)
    sim.Run(steps)
    run_s = sim.info().last_run_ms / 1e3
    local = np.stack([sim.mics(batch=m) for m in range(n)]) if n else np.zeros((0,) + sim.mics(batch=0).shape,
                                                                               np.float32)
    sim.close()
    return gather_rows(local.astype(np.float32), len(members), world, rank, device), run_s
