"""Autotuner for the batched pipeline.

Chooses the neighbour-grid cell size, the kNN block shape, the queries
per warp, the first-pass radius factor and the number of grid levels run
one query per lane by timing candidate settings on the caller's own
device-resident batch (CUDA events on the pipeline's stream, best of a few runs each). The
choice is cached per workload signature so later runs reuse it.
"""
from __future__ import annotations

import json
import os
from typing import Dict, Iterable, Optional, Tuple

_CACHE: Dict[str, dict] = {}


def signature(n_points: int, n_frames: int, cfg) -> str:
    bucket = 1 << max(0, int(n_points).bit_length() - 3)  # ~12% size buckets
    return (f"n{n_points // bucket * bucket}_f{n_frames}_leaf{cfg.leaf_size:.4g}_"
            f"sk{cfg.sor_k}_nk{cfg.normal_k}")


def _time_run(pipe, args, reps: int) -> float:
    import torch
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        torch.cuda.synchronize()
        s.record()
        pipe.run_device(*args)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    return best


def tune(pipe, x, y, z, offsets, n_frames: int, n_points: int,
         cells: Optional[Iterable[float]] = None,
         blocks: Iterable[int] = (64, 128, 256),
         qpws: Iterable[int] = (0, 3), rfacs: Iterable[float] = (0.7, 0.85, 1.0),
         lane_levels: Iterable[int] = (3, 2),
         reps: int = 2,
         cache_file: Optional[str] = None, verbose: bool = False) -> Tuple[dict, list]:
    """Returns (best setting, all trials) and applies the best to `pipe`.

    Two stages: every combination of cell size, kNN kernel mode
    (queries_per_warp: 0 one query per lane at every grid level, 3 a
    cooperative pass over dense cells, then one query per thread with its
    own adaptive window), first-pass radius factor and per-lane grid levels
    (mode 0 only) at the default block shape; then the block shape of the
    warp-per-query kernel at the best of those."""
    sig = signature(n_points, n_frames, pipe.cfg)
    if cache_file and os.path.exists(cache_file) and not _CACHE:
        try:
            _CACHE.update(json.load(open(cache_file)))
        except Exception:
            pass
    if sig in _CACHE:
        b = _CACHE[sig]
        _apply(pipe, b)
        return b, []
    leaf = pipe.cfg.leaf_size
    cells = (list(cells) if cells is not None
             else [leaf * m for m in (3.0, 5.0, 8.0, 10.0, 12.0, 15.0)])
    args = (x, y, z, offsets, n_frames, n_points)
    trials = []

    def trial(setting):
        _apply(pipe, setting)
        pipe.run_device(*args)  # warm
        t = _time_run(pipe, args, reps)
        r = dict(setting, ms=t)
        trials.append(r)
        if verbose:
            print(f"[autotune] {r}", flush=True)
        return r

    lane_levels = list(lane_levels)
    for c in cells:
        for q in qpws:
            for rf in rfacs:
                # the cooperative mode runs no per-lane chain: one level count
                for ll in (lane_levels[:1] if q == 3 else lane_levels):
                    trial({"cell": c, "block": 0, "qpw": q, "rfac": rf, "lane_levels": ll})
    best = min(trials, key=lambda r: r["ms"])
    for b in blocks:
        trial(dict({k: v for k, v in best.items() if k != "ms"}, block=b))
    best = dict(min(trials, key=lambda r: r["ms"]))
    best["trials"] = len(trials)
    _apply(pipe, best)
    _CACHE[sig] = best
    if cache_file:
        try:
            json.dump(_CACHE, open(cache_file, "w"), indent=1)
        except Exception:
            pass
    return best, trials


def _apply(pipe, s: dict) -> None:
    pipe.set_tuning(s["cell"], s["block"], s["qpw"])
    pipe.set_search_radius_factor(s["rfac"])
    pipe.set_lane_levels(s.get("lane_levels", 0))
