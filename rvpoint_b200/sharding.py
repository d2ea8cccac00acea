"""Frame sharding across ranks (one process per GPU).

Frames are independent units of the pipeline, so N GPUs split a batch of
frames with no data-path collective: each rank runs its own frames and the
only collectives are the timing reduction (max over ranks) and, when a
caller wants them in one place, gathering per-frame results.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence

import numpy as np


def partition_frames(frame_sizes: Sequence[int], world: int) -> List[List[int]]:
    """Greedy largest-first assignment of frames to ranks by point count
    (each frame to the currently lightest rank; ties to the lower rank).
    Returns, per rank, its frame indices in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(frame_sizes)), key=lambda f: (-int(frame_sizes[f]), f))
    heap = [(0, r) for r in range(world)]
    parts: List[List[int]] = [[] for _ in range(world)]
    for f in order:
        load, r = heapq.heappop(heap)
        parts[r].append(f)
        heapq.heappush(heap, (load + int(frame_sizes[f]), r))
    return [sorted(p) for p in parts]


def rank_batch(batch, frames: Sequence[int]):
    """The sub-batch of `frames` (a datasets.Batch), frames back to back."""
    from .datasets import Batch
    offs = np.asarray(batch.offsets, np.int64)
    xs, ys, zs, new = [], [], [], [0]
    for f in frames:
        a, b = int(offs[f]), int(offs[f + 1])
        xs.append(batch.x[a:b])
        ys.append(batch.y[a:b])
        zs.append(batch.z[a:b])
        new.append(new[-1] + (b - a))
    cat = lambda p: np.concatenate(p) if p else np.zeros(0, np.float32)  # noqa: E731
    return Batch(cat(xs), cat(ys), cat(zs), np.asarray(new, np.int64))


def max_over_ranks(value: float, device=None) -> float:
    """The maximum of `value` over all ranks (the step time of a job is its
    slowest rank's); the value itself when torch.distributed is not set up."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
