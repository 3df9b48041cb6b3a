"""Replica sharding on CPU with two gloo ranks: the shard ranges, the gather,
and the property the GPU shards rely on — a shard replayed at its replica
offset equals that slice of the unsharded run (the kernels' replay stands in
for the GPU here)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from openjij_b200.distributed import shard_range


def test_shard_ranges_cover_and_align():
    for R in (0, 1, 31, 32, 33, 100, 1024, 1025):
        for W in (1, 2, 3, 8):
            got = [shard_range(R, W, r) for r in range(W)]
            pos = 0
            for start, count in got:
                assert start == pos and count >= 0
                assert start % 32 == 0 or count == 0
                pos += count
            assert pos == R
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out_path):
    import torch.distributed as dist

    from openjij_b200 import instances as I
    from openjij_b200.distributed import gather_replicas, shard_range
    from oracle import oracle as O

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        g = O.AugCSR(I.lattice_pm_j(6, seed=4)[0])
        R = 80
        s0 = np.random.default_rng(5).choice(np.array([-1, 1], np.int8), size=(R, g.n))
        betas, mcs = I.geometric_betas(0.1, 3.0, 15)
        per = np.repeat(betas, mcs).astype(np.float32)
        start, count = shard_range(R, world, rank)
        local = O.replay_sa(g, s0[start:start + count], per, 9, rep0=start)
        full = gather_replicas(local, R)
        if rank == 0:
            np.save(out_path, full)
    finally:
        dist.destroy_process_group()


def test_two_rank_shards_reproduce_whole_run(tmp_path):
    from openjij_b200 import instances as I
    from oracle import oracle as O

    out = str(tmp_path / "full.npy")
    mp.start_processes(_worker, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    g = O.AugCSR(I.lattice_pm_j(6, seed=4)[0])
    s0 = np.random.default_rng(5).choice(np.array([-1, 1], np.int8), size=(80, g.n))
    betas, mcs = I.geometric_betas(0.1, 3.0, 15)
    whole = O.replay_sa(g, s0, np.repeat(betas, mcs).astype(np.float32), 9)
    np.testing.assert_array_equal(np.load(out), whole)
