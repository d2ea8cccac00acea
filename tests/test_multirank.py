"""Multi-rank host logic on CPU: gloo ranks (2 and 3) split a batch of LiDAR
frames with partition_frames, each runs the whole chain (voxel -> SOR ->
normals -> RANSAC, CPU oracle) on its own frames, and the gathered
per-frame results equal one process's; the timing reduction returns the
slowest rank's time."""
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


def _chain(R, frame):
    """voxel 0.1 -> SOR k=16 -> normals k=16 -> RANSAC 1000 / 0.05 (oracle)."""
    from oracle.oracle import libc_rand_stream
    v, _ = R.voxel_grid(frame, 0.1)
    s, _, _ = R.sor_exact(D.Cloud.from_xyz(v), 16, 1.0)
    sc = D.Cloud.from_xyz(s)
    n = R.normals_knn(sc, 16)
    best, model, _, _, _ = R.ransac_plane(sc, 0.05, 1000, libc_rand_stream(3000))
    return v, s, n, best, model


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
            res[f] = _chain(R, sub.frame(j))
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


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_split_frames_like_one_process(restatement, world):
    import torch.multiprocessing as mp
    batch = D.lidar_batch(n_frames=7, seed=31, min_pts=3000, max_pts=9000)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, batch, q)) for r in range(world)]
    for p in procs:
        p.start()
    merged, slowest = q.get(timeout=180)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(7))
    for f in range(7):
        want = _chain(restatement, batch.frame(f))
        got = merged[f]
        for a, b in zip(got[:3], want[:3]):
            assert np.array_equal(np.asarray(a).view(np.int32), np.asarray(b).view(np.int32))
        assert got[3] == want[3]
        assert np.array_equal(got[4].view(np.int32), want[4].view(np.int32))
    assert slowest == 10.0 + world - 1
