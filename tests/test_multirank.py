"""Multi-rank host logic on CPU: two gloo ranks split a batch of LiDAR
frames with partition_frames, each runs the voxel stage of its own frames
(CPU oracle), and the gathered per-frame results equal one process's; the
timing reduction returns the slowest rank's time."""
import os
import socket

import numpy as np
import pytest

from rvpoint_b200 import datasets as D
from rvpoint_b200.sharding import partition_frames, rank_batch


def test_partition_balances_and_covers():
    rng = np.random.default_rng(1)
    sizes = rng.integers(20_000, 131_072, 37)
    for world in (1, 2, 3, 8):
        parts = partition_frames(sizes, world)
        assert sorted(f for p in parts for f in p) == list(range(37))
        loads = [int(sizes[p].sum()) if p else 0 for p in parts]
        assert max(loads) - min(loads) <= int(sizes.max())
    assert partition_frames([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        partition_frames([1], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, batch, q):
    import torch.distributed as dist
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from oracle.oracle import Restatement
        from rvpoint_b200.sharding import max_over_ranks
        R = Restatement()
        sizes = np.diff(batch.offsets)
        mine = partition_frames(sizes, world)[rank]
        sub = rank_batch(batch, mine)
        res = {}
        for j, f in enumerate(mine):
            v, _ = R.voxel_grid(sub.frame(j), 0.1)
            res[f] = v
        gathered = [None] * world
        dist.all_gather_object(gathered, res)
        slowest = max_over_ranks(10.0 + rank)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            q.put((merged, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_frames_like_one_process(restatement):
    import torch.multiprocessing as mp
    batch = D.lidar_batch(n_frames=6, seed=31, min_pts=3000, max_pts=9000)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, batch, q)) for r in range(2)]
    for p in procs:
        p.start()
    merged, slowest = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(6))
    for f in range(6):
        v, _ = restatement.voxel_grid(batch.frame(f), 0.1)
        assert np.array_equal(merged[f].view(np.int32), v.view(np.int32))
    assert slowest == 11.0
