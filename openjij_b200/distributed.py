"""Replica sharding over GPUs (one process per GPU, torch.distributed).

The annealing path has no exchange step: reads are independent, and every
random number is a pure function of (seed, global sweep, global replica,
site).  A run of R replicas over W ranks therefore gives each rank a
contiguous replica range whose first index is passed to the C ABI as
``replica_offset`` (a multiple of 32, the bit-packed kernel's group size), and
the union of the shards is bit-identical to the one-GPU run.  The only
collective is the final gather of spins and energies, on the host side of
the run.
"""
from __future__ import annotations

import numpy as np

ALIGN = 32


def shard_range(num_replicas: int, world_size: int, rank: int, align: int = ALIGN):
    """(start, count) of ``rank``'s replicas: blocks of ``align`` replicas dealt
    out as evenly as possible, lower ranks first; start is a multiple of align."""
    if world_size < 1 or not 0 <= rank < world_size:
        raise ValueError("rank must be in [0, world_size)")
    if num_replicas < 0:
        raise ValueError("num_replicas must be >= 0")
    blocks = (num_replicas + align - 1) // align
    per, extra = divmod(blocks, world_size)
    first = rank * per + min(rank, extra)
    nblk = per + (1 if rank < extra else 0)
    start = min(first * align, num_replicas)
    stop = min((first + nblk) * align, num_replicas)
    return start, stop - start


def gather_replicas(local: np.ndarray, num_replicas: int, group=None) -> np.ndarray:
    """All-gathers the ranks' replica shards (leading axis) into the full
    [num_replicas, ...] array on every rank, in replica order."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    shape_tail = tuple(local.shape[1:])
    width = max(shard_range(num_replicas, world, r)[1] for r in range(world))
    buf = np.zeros((width,) + shape_tail, dtype=local.dtype)
    buf[: local.shape[0]] = local
    t = torch.from_numpy(buf)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t, group=group)
    out = np.empty((num_replicas,) + shape_tail, dtype=local.dtype)
    for r, p in enumerate(parts):
        start, count = shard_range(num_replicas, world, r)
        out[start:start + count] = p.numpy()[:count]
    return out


def sa_run_sharded(graph, spins_full: np.ndarray, betas, mcs, seed: int, group=None, **kwargs):
    """Runs this rank's shard of ``spins_full`` [R][n] through ``oj_sa_run``
    (``openjij_b200._native.sa_run``) with its replica offset, then gathers the
    spins and FP64 energies of all ranks.  Returns (spins [R][n], energies [R])."""
    import torch.distributed as dist

    from openjij_b200 import _native as N

    R = spins_full.shape[0]
    start, count = shard_range(R, dist.get_world_size(group), dist.get_rank(group))
    local = np.ascontiguousarray(spins_full[start:start + count])
    energies = np.zeros(count)
    if count:
        N.sa_run(graph, local, betas, mcs, seed=seed, energies=energies, replica_offset=start, **kwargs)
    return gather_replicas(local, R, group), gather_replicas(energies, R, group)
