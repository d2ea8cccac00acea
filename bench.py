#!/usr/bin/env python
"""Batched point-cloud pipeline benchmark (one JSON line on rank 0).

Workload: 256 synthetic spinning-LiDAR frames (64 beams x 2048 azimuths cast
against a ground plane and 40 boxes, sigma = 2 cm, 5% drop, each thinned to
a log-uniform size in [20k, 131k] points), the chain
voxel(0.1 m) -> SOR(k=16, std_mul=1) -> normals(k=16) -> RANSAC(1000
hypotheses, 0.05 m) per frame. A step is one pass of the chain over the
whole batch. `value` is input points per second with the batch resident in
HBM; `e2e` is the same through the host-buffer C entry point for steps in
a row (rvp_pipeline_run_host_batches: each step's inputs go up and its
results come down, overlapped with the neighbouring steps' work) with the
host<->device copies inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--cell C [--rfac R]] [--no-tune] [--cpu-frames F]

Rank 0 also runs the learned-vs-plain RANSAC leg (``learned_ransac`` in the
line): 512 plane scenes of 50,000 points; plain GPU RANSAC (10,000
hypotheses, the reference's stream and stopping rule) against the learned
proposal (features + MLP + weighted RANSAC) to 99% of plain's best count.

Rank 0 also times the calls around the path (``next_rows``): PCD input,
PointerOctree SOR and normals and Euclidean clustering on the reference
pipeline driver's settings, through the public API with host arrays, beside
the reference's own CPU code on the same input (one thread).

N > 1: launched by torch.distributed.run, one rank per GPU; every rank owns
its own 256 frames (weak scaling, no data-path collective); time = max over
ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import multiprocessing as mp
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "pipeline Mpts/s on 1 B200; learned-vs-plain RANSAC time at equal inlier count"
UNIT = "Mpts/s"
WORKLOAD = "lidar_batch_256_frames_voxel0.1_sor16_normals16_ransac1000"
LEAF, SOR_K, SOR_ALPHA, NORMAL_K, R_THRESH, R_ITERS = 0.1, 16, 1.0, 16, 0.05, 1000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=256)
    ap.add_argument("--no-tune", action="store_true")
    ap.add_argument("--cell", type=float, default=0.0,
                    help="fixed grid cell (m) instead of the autotuner's choice")
    ap.add_argument("--rfac", type=float, default=1.0,
                    help="level-0 first-pass radius factor with --cell")
    ap.add_argument("--lane-levels", type=int, default=2,
                    help="grid levels of the one-query-per-lane kNN with --cell")
    ap.add_argument("--qpw", type=int, default=3,
                    help="kNN kernel mode with --cell (0 per-lane, 3 cooperative level 0)")
    ap.add_argument("--block", type=int, default=0,
                    help="warp-per-query kernel block size with --cell (0: 256)")
    ap.add_argument("--cpu-frames", type=int, default=5,
                    help="frames of the CPU baseline (and of the parity check)")
    ap.add_argument("--no-singles", action="store_true",
                    help="skip the single-cloud workloads (room chain, LiDAR radius, 2M normals)")
    ap.add_argument("--no-next-rows", action="store_true",
                    help="skip the PCD / octree / clustering timings")
    ap.add_argument("--learned-scenes", type=int, default=512,
                    help="plane scenes of the learned-vs-plain RANSAC leg (0: skip)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# CPU side (the reference's scalar path; test infrastructure under oracle/)
# ---------------------------------------------------------------------------
def _cpu_frame(args):
    """voxel -> sor_rvv -> normal_estimation_sc -> ransac_plane_rvv on one
    frame with the reference's own code (or the restatement if absent), one
    thread. Returns the time, the input size, the kind, and the outputs (for
    the comparison with the GPU's results of the same frame)."""
    x, y, z = args
    sys.path.insert(0, ROOT)
    import numpy as np
    from oracle import oracle as O
    from rvpoint_b200.datasets import Cloud
    os.environ["RVO_THREADS"] = "1"
    c = Cloud(np.ascontiguousarray(x), np.ascontiguousarray(y), np.ascontiguousarray(z))
    t0 = time.perf_counter()
    if O.reference_available():
        R = O.Reference()
        v = R.voxel_grid(c, LEAF)
        vc = Cloud.from_xyz(v)
        s = R.sor_rvv(vc, SOR_K, SOR_ALPHA)
        sc = Cloud.from_xyz(s)
        nrm = R.normals_sc(sc, NORMAL_K)
        best, model = R.ransac_plane(sc, R_THRESH, R_ITERS)
        kind = "reference"
    else:
        R = O.Restatement()
        v, _ = R.voxel_grid(c, LEAF)
        vc = Cloud.from_xyz(v)
        s, _, _ = R.sor_exact(vc, SOR_K, SOR_ALPHA)
        sc = Cloud.from_xyz(s)
        nrm = R.normals_knn(sc, NORMAL_K)
        best, model, _, _, _ = R.ransac_plane(sc, R_THRESH, R_ITERS,
                                              O.libc_rand_stream(3 * R_ITERS))
        kind = "port"
    dt = time.perf_counter() - t0
    return dt, int(x.shape[0]), kind, {"voxel": v, "sor": s, "normals": nrm, "best": int(best),
                                       "model": np.asarray(model, np.float32)}


def _cpu_room_chain(_=None):
    """The 100,000-point room chain with the reference's own code, one thread:
    voxel 0.01 -> sor_rvv k=30 -> normal_estimation_rvv(SpatialHash, r=0.03)
    -> ransac_plane_rvv 1000 / 0.01. Returns per-stage seconds."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from rvpoint_b200 import datasets as D
    os.environ["RVO_THREADS"] = "1"
    if not O.reference_available():
        return None
    R = O.Reference()
    c = D.room_cloud(n=100_000)
    t = {}
    t0 = time.perf_counter()
    v = R.voxel_grid(c, 0.01)
    t["voxel"] = time.perf_counter() - t0
    vc = D.Cloud.from_xyz(v)
    t0 = time.perf_counter()
    s = R.sor_rvv(vc, 30, 1.0)
    t["sor"] = time.perf_counter() - t0
    sc = D.Cloud.from_xyz(s)
    t0 = time.perf_counter()
    R.normals_hash(sc, 0.03, 0.03)
    t["normals"] = time.perf_counter() - t0
    t0 = time.perf_counter()
    best, _ = R.ransac_plane(sc, 0.01, 1000)
    t["ransac"] = time.perf_counter() - t0
    return {"seconds": t, "voxels": int(v.shape[0]), "kept": int(s.shape[0]), "ransac": best}


def _cpu_lidar_radius(_=None):
    """All-point radiusSearch r = 0.5 and the radius-bounded kNN (max_nn = 16)
    on the whole 64 x 2048-ray frame with the reference's SpatialHash (cell
    0.5), one thread."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as O
    from rvpoint_b200 import datasets as D
    if not O.reference_available():
        return None
    R = O.Reference()
    f = D.lidar_frame()
    t0 = time.perf_counter()
    o, _, _ = R.radius_search(f, 0.5, 0.5)
    t_r = time.perf_counter() - t0
    t0 = time.perf_counter()
    R.radius_search(f, 0.5, 0.5, max_nn=16)
    t_k = time.perf_counter() - t0
    return {"radius_s": t_r, "knn16_s": t_k, "points": f.n, "pairs": int(o[-1])}


def single_cloud_legs(ctx) -> dict:
    """The single-cloud workloads through the public API with host arrays in
    and out (wall clock, mean of 3 calls after one warm-up): the 100k room
    chain, all-point radius search r = 0.5 and kNN 16 on one whole LiDAR
    frame, and precision-mode normals (k = 32) of the 2,000,000-point
    translated room with their error against float64 on 100,000 sampled
    points."""
    import numpy as np
    from rvpoint_b200 import api
    from rvpoint_b200 import datasets as D

    def wall(fn, reps=3):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            r = fn()
        return (time.perf_counter() - t0) / reps * 1e3, r

    out = {}
    c = D.room_cloud(n=100_000)

    def room_chain():
        v = api.voxel_grid_downsamp_rvv_v2(c, 0.01, ctx=ctx)
        vc = D.Cloud.from_xyz(v)
        s = api.sor_rvv(vc, 30, 1.0, ctx=ctx)
        sc = D.Cloud.from_xyz(s)
        h = api.SpatialHash(ctx)
        h.setInputCloud(sc, 0.03)
        h.build()
        api.normal_estimation_rvv(sc, h, 10, 0.03)  # on the hash's context
        h.close()
        best, _ = api.ransac_plane_rvv(sc, 0.01, 1000, ctx=ctx)
        return len(v), len(s), best
    ms, (nv, ns, best) = wall(room_chain)
    out["room_chain_100k"] = {"workload": "room 100k: voxel 0.01 -> sor_rvv k=30 -> "
                                          "SpatialHash normals r=0.03 -> RANSAC 1000 / 0.01",
                              "gpu_ms": ms, "gpu_mpts_s": c.n / ms / 1e3, "voxels": nv,
                              "kept": ns, "ransac": best}
    f = D.lidar_frame()
    h = api.SpatialHash(ctx)
    h.setInputCloud(f, 0.5)
    h.build()
    ms_r, (offs, _, _) = wall(lambda: h.radiusSearchBatch(f.x, f.y, f.z, 0.5))
    ms_k, _ = wall(lambda: h.radiusSearchBatch(f.x, f.y, f.z, 0.5, max_nn=16))
    ms_kk, _ = wall(lambda: h.knn(f.x, f.y, f.z, 16))
    h.close()
    out["lidar_frame_radius"] = {"workload": "one 64 x 2048-ray frame, every point: "
                                             "radiusSearch r=0.5 (cell 0.5), max_nn=16, kNN 16",
                                 "points": f.n, "pairs_r05": int(offs[-1]),
                                 "radius_gpu_ms": ms_r, "radius_gpu_mqueries_s": f.n / ms_r / 1e3,
                                 "max_nn16_gpu_ms": ms_k, "knn16_gpu_ms": ms_kk}
    p = D.precision_room()
    ms, (nrm, cond, used) = wall(lambda: api.normal_estimation_precise(p, 32, ctx=ctx), reps=2)
    out["precision_normals_2m"] = {"workload": "2M-point room shifted by (1e4, 1e4, 0), k=32, "
                                               "precision mode", "gpu_ms": ms,
                                   "gpu_mpts_s": p.n / ms / 1e3,
                                   "fp64_eigen_fraction": float(np.mean(used > 0))}
    try:
        from scipy.spatial import cKDTree
        rng = np.random.default_rng(5)
        q = rng.choice(p.n, size=100_000, replace=False)
        P = np.stack([p.x, p.y, p.z], 1).astype(np.float64)
        _, nbr = cKDTree(P).query(P[q], k=33, workers=-1)
        X = P[nbr]
        Xc = X - X.mean(1, keepdims=True)
        w, V = np.linalg.eigh(np.einsum("nki,nkj->nij", Xc, Xc))
        ref = V[:, :, 0]
        g = nrm[q].astype(np.float64)
        cosang = np.abs((g * ref).sum(1)) / np.maximum(np.linalg.norm(g, axis=1), 1e-300)
        ang = np.arccos(np.clip(cosang, 0, 1))
        gap = w[:, 1] / np.maximum(w[:, 0], 1e-300)
        ok = gap > 1.0 + 1e-9
        out["precision_normals_2m"].update(
            {"angle_err_rad_vs_fp64": {"sampled_points": int(ok.sum()),
                                       "max": float(ang[ok].max()),
                                       "p99": float(np.percentile(ang[ok], 99))}})
    except Exception as e:  # pragma: no cover
        out["precision_normals_2m"]["angle_err_rad_vs_fp64"] = {"unavailable": str(e)}
    return out


def sample_frames(sizes, count: int):
    """Frames at evenly spaced quantiles of the batch's size distribution
    (the CPU cost is quadratic in the frame size, so a sample of the first
    frames would weight the mix by chance)."""
    import numpy as np
    order = np.argsort(sizes, kind="stable")
    qs = [(i + 0.5) / count for i in range(count)]
    return [int(order[min(len(order) - 1, int(q * len(order)))]) for q in qs]


def cpu_baseline(batch, n_frames_sample: int, gpu_results=None, singles: bool = True):
    """The reference's chain on a sample of frames spread over the batch's
    size range, each frame on one thread (the reference library is
    single-threaded); the frames run in separate processes at the same time
    to save wall clock, each timed on its own. The reference's outputs of
    those frames are compared with the GPU's results of the same frames
    (``parity``). With `singles`, the single-cloud workloads (the 100k room
    chain, the LiDAR frame's radius search) run beside them, one process
    each. Returns (cpu_baseline, single-cloud CPU times)."""
    import numpy as np
    from oracle import oracle as O
    O.build() if not os.path.exists(O.RESTATEMENT_SO) else None
    sizes = np.diff(batch.offsets)
    pick = sample_frames(sizes, n_frames_sample)
    jobs = [(batch.frame(f).x, batch.frame(f).y, batch.frame(f).z) for f in pick]
    with mp.get_context("spawn").Pool(len(jobs) + (2 if singles else 0)) as pool:
        room = pool.apply_async(_cpu_room_chain) if singles else None
        lidar = pool.apply_async(_cpu_lidar_radius) if singles else None
        res = pool.map(_cpu_frame, jobs)
        cpu_single = {"room_chain_100k": room.get(), "lidar_frame_radius": lidar.get()} \
            if singles else None
    t_tot = sum(r[0] for r in res)
    pts = sum(r[1] for r in res)
    kind = res[0][2]
    out = {"value": pts / t_tot / 1e6, "unit": UNIT, "cores": 1, "kind": kind,
           "sample": (f"{len(pick)} of {batch.n_frames} frames at evenly spaced size "
                      f"quantiles ({pts} input points; frame sizes "
                      f"{[int(sizes[f]) for f in pick]}), full chain, each frame on one "
                      f"thread; {t_tot:.1f} s of CPU time summed over the frames"),
           "frames": pick}
    if gpu_results is not None:
        out["parity"] = compare_frames(gpu_results, pick, [r[3] for r in res])
    return out, cpu_single


def compare_frames(g, frames, ref) -> dict:
    """The GPU's per-frame results against the reference's outputs of the
    same frames: voxel centroids, SOR output and the RANSAC count / model bit
    for bit; normals within 1e-4 rad of the reference's FP32 normals."""
    import numpy as np
    bits = lambda a: np.ascontiguousarray(a, np.float32).view(np.int32)  # noqa: E731
    vox = sor = ran = True
    close = []
    for f, r in zip(frames, ref):
        a, b = g["voxel_offsets"][f], g["voxel_offsets"][f + 1]
        vox &= np.array_equal(bits(g["voxel"][a:b]), bits(r["voxel"]))
        a, b = g["sor_offsets"][f], g["sor_offsets"][f + 1]
        same_sor = np.array_equal(bits(g["sor"][a:b]), bits(r["sor"]))
        sor &= same_sor
        ran &= int(g["ransac_count"][f]) == r["best"] and np.array_equal(
            bits(g["ransac_model"][f]), bits(r["model"]))
        if same_sor:
            u, v = g["normals"][a:b], r["normals"]
            cosang = np.abs((u * v).sum(1)) / np.maximum(
                np.linalg.norm(u, axis=1) * np.linalg.norm(v, axis=1), 1e-30)
            close.append(float((np.arccos(np.clip(cosang, 0, 1)) < 1e-4).mean()))
    return {"frames_checked": len(frames), "voxel_bit_exact": bool(vox),
            "sor_bit_exact": bool(sor), "ransac_bit_exact": bool(ran),
            "normals_within_1e-4_rad_min_fraction": min(close) if close else None}


def reference_arm(a, rank: int) -> None:
    if rank != 0:
        return
    from rvpoint_b200 import datasets as D
    from oracle import oracle as O
    if not os.path.exists(O.RESTATEMENT_SO):
        O.build()
    batch = D.lidar_batch(n_frames=a.frames)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    workers = max(1, cores)
    ctx = mp.get_context("spawn")
    times, pts_step, sizes_seen = [], [], []
    kind = "port"
    # a step is one frame per process; frames take seconds each on one core
    # (the reference's exact SOR is quadratic in the frame size), so the run
    # is bounded to at most 1 + 3 steps, whatever --steps / --warmup ask
    warm, steps = min(a.warmup, 1), min(a.steps, 3)
    # frames in a seeded random order, so that every step's sample has the
    # batch's size mix rather than the first frames'
    import numpy as np
    perm = np.random.default_rng(0).permutation(batch.n_frames)
    with ctx.Pool(workers) as pool:
        nxt = 0
        for step in range(warm + steps):
            # one frame per worker per step, frames in order
            sel = [int(perm[(nxt + j) % batch.n_frames])
                   for j in range(min(workers, batch.n_frames))]
            nxt = (nxt + len(sel)) % batch.n_frames
            jobs = [(batch.frame(f).x, batch.frame(f).y, batch.frame(f).z) for f in sel]
            t0 = time.perf_counter()
            res = pool.map(_cpu_frame, jobs)
            dt = time.perf_counter() - t0
            sizes_seen.extend(r[1] for r in res)
            kind = res[0][2]
            if step >= warm:
                times.append(dt)
                pts_step.append(sum(r[1] for r in res))
    value = sum(pts_step) / sum(times) / 1e6
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": a.gpus, "steps": steps, "warmup": warm,
            "requested": {"steps": a.steps, "warmup": a.warmup},
            "ms_per_step": 1e3 * statistics.mean(times), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames_per_step": min(workers, batch.n_frames),
                       "leaf": LEAF, "sor_k": SOR_K, "normal_k": NORMAL_K,
                       "ransac_iters": R_ITERS, "ransac_thresh": R_THRESH},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": workers, "kind": kind,
                             "sample": f"{min(workers, batch.n_frames)} frames per step in a "
                                       f"seeded random order, one frame per process, "
                                       f"{workers} processes; frame sizes {sizes_seen}"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class Clocks:
    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [v.strip() for v in vis.split(",") if v.strip()]
        gid = ids[gpu_index] if gpu_index < len(ids) else str(gpu_index)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gid}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = [r.split(",") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            r = [v.strip() for v in r]
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
            except Exception:
                continue
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
# kernels timed live for the roofline (CUDA events around each launch): the
# SOR kNN kernel of each grid level and RANSAC
LEVEL_STAGES = ("sor_knn_l0", "sor_knn_l1", "sor_knn_l2", "sor_knn_coop")


def kernel_name(stage: str, coop: bool) -> str:
    if stage == "ransac":
        return "k_ransac"
    if stage == "sor_knn_coop":
        return "k_knn_coop<17,SOR_LIST> (cells of c)"
    if coop and stage == "sor_knn_l0":
        return "k_knn_adapt<17,SOR_LIST> (per-thread windows)"
    cells = {"sor_knn_l0": "c", "sor_knn_l1": "4c", "sor_knn_l2": "16c"}[stage]
    return f"k_knn_wt<17,SOR_LIST> (cells of {cells})"


def kernel_units(stage: str, coop: bool, counts, n_vox: int):
    """Queries one launch of a SOR kNN kernel processes: in cooperative mode
    the cooperative pass's and the adaptive kernel's (counts); without it
    the per-lane kernel on cells of c takes every query (on the coarser
    cells only the ones left open, a count the line does not carry)."""
    if coop:
        return {"sor_knn_coop": counts[0], "sor_knn_l0": counts[1]}.get(stage)
    if stage == "sor_knn_l0":
        return n_vox
    return None


def kernel_bytes(stage: str, units: int, n_sor: int, n_frames: int) -> float:
    """Algorithmic bytes of one launch: 12 B per query + 8 B per neighbour
    (k+1 = 17 neighbours) for a kNN kernel; RANSAC reads each kept point once
    and writes a count per hypothesis."""
    if stage == "ransac":
        return 12.0 * n_sor + 4.0 * R_ITERS * n_frames
    return (12.0 + 8.0 * (SOR_K + 1)) * units


def _write_pcd_binary(path: str, x, y, z) -> None:
    """A PCD file of fields x y z, DATA binary (io/simple_pcd_loader.h)."""
    import numpy as np
    n = int(x.shape[0])
    head = ("# .PCD v.7 - Point Cloud Data file format\nVERSION .7\nFIELDS x y z\n"
            "SIZE 4 4 4\nTYPE F F F\nCOUNT 1 1 1\n"
            f"WIDTH {n}\nHEIGHT 1\nVIEWPOINT 0 0 0 1 0 0 0\nPOINTS {n}\nDATA binary\n")
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(np.ascontiguousarray(np.stack([x, y, z], 1), np.float32).tobytes())


def next_rows_leg(ctx, batch) -> dict:
    """The calls around the hot path on the reference pipeline driver's
    settings (pipeline_export.cpp:37-67): loadPCD of the batch (binary),
    then on a 100k-point room cloud thinned by voxel 0.01: PointerOctree
    build + sor_pointer_octree (k 20, std 1, radius 0.25), PointerOctree
    normals (radius 0.03), Euclidean clustering (tolerance 0.15, 50 to
    100,000 points; the reference's quadratic search on a 20,000-point
    subset, the GPU on the same subset and on the whole cloud). GPU times are
    wall clock around the public API call with host arrays in and out; the
    CPU times are the reference's own code (oracle/_ref), one thread."""
    import numpy as np
    from oracle import oracle as O
    from rvpoint_b200 import api
    from rvpoint_b200 import datasets as D
    if not O.reference_available():
        return {"unavailable": "reference library not built"}
    R = O.Reference()
    out = {}

    def wall(fn, reps=3):
        fn()
        t0 = time.perf_counter()
        for _ in range(reps):
            r = fn()
        return (time.perf_counter() - t0) / reps * 1e3, r

    with tempfile.TemporaryDirectory() as td:
        path = os.path.join(td, "batch.pcd")
        _write_pcd_binary(path, batch.x, batch.y, batch.z)
        n = int(batch.x.shape[0])
        g_ms, _ = wall(lambda: api.load_pcd(path, device=True, ctx=ctx))
        c_ms, _ = wall(lambda: R.load_pcd(path, n), reps=1)
        out["pcd_load_binary"] = {"points": n, "bytes": os.path.getsize(path),
                                  "gpu_ms": g_ms, "cpu_ms": c_ms,
                                  "gpu_mpts_s": n / g_ms / 1e3, "cpu_mpts_s": n / c_ms / 1e3,
                                  "note": "file in page cache; GPU: into device arrays"}
    v = api.voxel_grid_downsamp_rvv_v2(D.room_cloud(n=100_000), 0.01, ctx=ctx)
    c = D.Cloud.from_xyz(v)
    nv = c.n

    def gpu_sor():
        t = api.PointerOctree(ctx)
        t.setInputCloud(c)
        t.build()
        r = api.sor_pointer_octree(c, t, 20, 1.0, 0.25)
        t.close()
        return r
    g_ms, g_out = wall(gpu_sor)
    c_ms, c_out = wall(lambda: R.sor_octree(1, c, 20, 1.0, 0.25), reps=1)
    same = bool(np.array_equal(np.ascontiguousarray(g_out).view(np.int32),
                               np.ascontiguousarray(c_out).view(np.int32)))
    out["sor_pointer_octree"] = {"points": nv, "gpu_ms": g_ms, "cpu_ms": c_ms,
                                 "speedup": c_ms / g_ms, "kept": int(g_out.shape[0]),
                                 "bit_exact": same}

    def gpu_normals():
        t = api.PointerOctree(ctx)
        t.setInputCloud(c)
        t.build()
        r = api.normal_estimation_tree(c, t, 10, 0.03)
        t.close()
        return r
    g_ms, _ = wall(gpu_normals)
    c_ms, _ = wall(lambda: R.normals_octree(1, c, 0.03), reps=1)
    out["normals_pointer_octree"] = {"points": nv, "gpu_ms": g_ms, "cpu_ms": c_ms,
                                     "speedup": c_ms / g_ms}
    sub = c.subset(np.arange(min(nv, 20_000)))
    g_ms, g_cl = wall(lambda: api.euclidean_clusters(sub, 0.15, 50, 100_000, ctx=ctx))
    c_ms, c_cl = wall(lambda: R.euclidean_clusters(sub, 0.15, 50, 100_000), reps=1)
    same = len(g_cl) == len(c_cl) and all(np.array_equal(a, b) for a, b in zip(g_cl, c_cl))
    gf_ms, _ = wall(lambda: api.euclidean_clusters(c, 0.15, 50, 100_000, ctx=ctx))
    out["euclidean_clustering"] = {"points": int(sub.n), "gpu_ms": g_ms, "cpu_ms": c_ms,
                                   "speedup": c_ms / g_ms, "clusters": len(g_cl),
                                   "same_clusters": same, "gpu_ms_full_cloud": gf_ms,
                                   "full_cloud_points": nv}
    return out


def learned_leg(ctx, n_scenes: int, n_train: int, reps: int = 3) -> dict:
    """Learned-vs-plain RANSAC on n_scenes synthetic plane scenes of 50,000
    points (1-6 planes, 30-70% outliers, 5 mm noise), timed with CUDA events,
    inputs resident. The network is trained first on n_train held-out scenes,
    on the GPU.

    Equal inlier count, one stopping rule for every arm: each scene's target
    is 99% of the best count plain RANSAC reaches with up to 10,000
    hypotheses (the reference's rand() stream and adaptive stop, p = 0.99),
    and every arm stops a scene at the first hypothesis whose exact count
    over all 50,000 points reaches it:
      plain_to_count     uniform draws from the reference's stream;
      learned_to_count   features + MLP + preemptive weighted proposal;
      preemptive_uniform_to_count
                         the same preemptive rounds over the same candidates
                         with equal weights (what the preemption alone buys).
    Without a target (the learned arm's own budget): one preemptive round,
    its best hypotheses counted exactly; the fraction of scenes within 1% of
    plain's 10,000-hypothesis best."""
    import torch
    from rvpoint_b200 import datasets as D
    from rvpoint_b200 import learned as LR
    T = 0.02
    tr = D.plane_batch(n_train, seed=D.SEED_BASE + 4000)
    ev = D.plane_batch(n_scenes, seed=D.SEED_BASE + 4)
    bt, be = LR.DeviceBatch.from_host(tr), LR.DeviceBatch.from_host(ev)
    del tr, ev
    scorer = LR.PlaneScorer(max(bt.n, be.n), max(n_train, n_scenes), ctx=ctx)
    info = LR.train(scorer, bt, LR.TrainConfig())

    def timed(fn):
        for _ in range(3):
            out = fn()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            out = fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps, out

    t_plain, (_, best, it_plain) = timed(lambda: LR.ransac_frames(be, 10_000, T, ctx=ctx))
    tg = torch.ceil(best.double() * 0.99).to(torch.int32)
    t_ptg, (_, bp, it_ptg) = timed(lambda: LR.ransac_frames(be, 10_000, T, targets=tg, ctx=ctx))
    lr = LR.LearnedRansac(scorer)
    cand, coffs = lr.prepare(be)
    # the feature kNN among each scene's candidates (two blocks per scene,
    # each with the scene's grid in shared memory): its cell size sets only
    # the speed
    knn_modes = {}
    for cell in (1.0, 1.5, 2.0, 2.5):
        knn_modes[f"cell{cell}"] = timed(
            lambda: LR.proposal_features(scorer, be, cand, coffs, cell, lr.scope))[0]
    best_mode = min(knn_modes, key=knn_modes.get)
    lr.cell = float(best_mode[4:])
    t_l, (_, bl, it_l) = timed(lambda: lr.run(be, cand, coffs, 10_000, T, targets=tg))
    t_f, feat = timed(lambda: LR.proposal_features(scorer, be, cand, coffs, lr.cell, lr.scope))
    t_m, logits = timed(lambda: scorer.forward(feat))
    t_w, _ = timed(lambda: lr.ransac(be, cand, coffs, logits, 10_000, T, targets=tg))
    flat = torch.zeros_like(logits)
    t_u, (_, bu, it_u) = timed(lambda: lr.ransac(be, cand, coffs, flat, 10_000, T, targets=tg))
    # the learned arm on its own budget: one preemptive round, no target
    one = LR.LearnedRansac(scorer, draws=lr.draws)

    def one_round():
        f_ = LR.proposal_features(scorer, be, cand, coffs, one.cell, one.scope)
        lg = scorer.forward(f_)
        return LR.ransac_preemptive(be, cand, coffs, lg, T, draws=one.draws, max_rounds=1,
                                    seed=one.seed, logit_power=one.logit_power, ctx=ctx)
    t_1, (_, b1, _) = timed(one_round)
    q = lambda t, p: float(t.double().quantile(p).item())  # noqa: E731
    within = lambda b: float((b.double() >= 0.99 * best.double()).float().mean().item())  # noqa: E731
    out = {"scenes": n_scenes, "points_per_scene": 50_000, "thresh": T,
           "train_scenes": n_train, "train_seconds": info["seconds"],
           "train_loss_first_last": [info["losses"][0][1], info["losses"][-1][1]],
           "candidates_per_scene": lr.cand_per_frame, "feature_scope": lr.scope,
           "proposal": (f"preemptive: {lr.draws} draws per round ranked on the candidates, "
                        "best 32 counted exactly" if lr.preemptive else "weighted draws, "
                        "each counted exactly"),
           "stopping_rule": "every arm stops a scene at 99% of plain RANSAC's "
                            "10,000-hypothesis best count",
           "plain_10k_ms": t_plain,
           "plain_10k_hypotheses_mean": float(it_plain.double().mean().item()),
           "plain_to_count_ms": t_ptg,
           "plain_hypotheses_to_count": {"mean": float(it_ptg.double().mean().item()),
                                         "median": q(it_ptg, 0.5), "p90": q(it_ptg, 0.9)},
           "learned_to_count_ms": t_l,
           "learned_parts_ms": {"features": t_f, "mlp": t_m, "weighted_ransac": t_w},
           "feature_knn_ms_by_mode": knn_modes, "feature_knn_mode": best_mode,
           "learned_hypotheses_drawn_to_count": {"mean": float(it_l.double().mean().item()),
                                                 "median": q(it_l, 0.5), "p90": q(it_l, 0.9)},
           "learned_reached_fraction": float((bl >= tg).float().mean().item()),
           "preemptive_uniform_to_count_ms": t_u,
           "preemptive_uniform_hypotheses_drawn_to_count": {
               "mean": float(it_u.double().mean().item()), "median": q(it_u, 0.5),
               "p90": q(it_u, 0.9)},
           "preemptive_uniform_reached_fraction": float((bu >= tg).float().mean().item()),
           "time_ratio_plain_to_count_over_learned": t_ptg / t_l,
           "time_ratio_preemptive_uniform_over_learned": t_u / t_l,
           "time_ratio_plain10k_over_learned": t_plain / t_l,
           "learned_one_round_no_target": {
               "ms": t_1, "draws_per_scene": one.draws,
               "scenes_within_1pct_of_plain_10k": within(b1),
               "mean_count_over_plain_10k": float((b1.double() / best.double()).mean().item())}}
    scorer.close()
    return out


def main():
    a = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        reference_arm(a, rank)
        return
    import numpy as np
    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from rvpoint_b200 import api, autotune
    from rvpoint_b200.sharding import max_over_ranks
    from rvpoint_b200 import datasets as D

    batch = D.lidar_batch(n_frames=a.frames, seed=D.SEED_BASE + 2 + 7919 * rank)
    n, nf = batch.n, batch.n_frames
    dev = torch.device("cuda", local)
    x = torch.from_numpy(batch.x).to(dev)
    y = torch.from_numpy(batch.y).to(dev)
    z = torch.from_numpy(batch.z).to(dev)
    offs = torch.from_numpy(batch.offsets).to(dev)
    ctx = api.Context(local)
    pipe = api.Pipeline(max_points=n, max_frames=nf, leaf_size=LEAF, sor_k=SOR_K,
                        sor_alpha=SOR_ALPHA, normal_k=NORMAL_K, ransac_thresh=R_THRESH,
                        ransac_iters=R_ITERS, ctx=ctx)
    args = (x, y, z, offs, nf, n)
    best = None
    pipe.run_device(*args)
    pipe.fit_tables()  # bucket table sized to this workload (stays in L2)
    if a.cell > 0:
        pipe.set_tuning(a.cell, a.block, a.qpw)
        pipe.set_search_radius_factor(a.rfac)
        pipe.set_lane_levels(a.lane_levels)
        best = {"cell": a.cell, "block": a.block, "qpw": a.qpw, "rfac": a.rfac,
                "lane_levels": a.lane_levels, "fixed": True}
    elif not a.no_tune:
        best, _ = autotune.tune(pipe, *args)
    for _ in range(max(a.warmup, 1)):
        pipe.run_device(*args)
    torch.cuda.synchronize()
    launches0 = ctx.launches
    pipe.run_device(*args)
    torch.cuda.synchronize()
    launches_per_step = ctx.launches - launches0

    # ---- timed region: inputs resident in HBM (180 MB of input > 126 MB L2)
    pipe.set_timing(a.steps)
    clocks = Clocks(local) if rank == 0 else None
    time.sleep(0.3 if clocks else 0)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(a.steps):
        pipe.run_device(*args)
    ev1.record()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = ev0.elapsed_time(ev1)
    clk = clocks.stop() if clocks else None
    pipe.check()
    stages = pipe.stage_times(levels=True)

    # ---- the same steps replayed from one CUDA graph (no per-stage events)
    pipe.set_timing(0)
    graph_kernels = pipe.capture(*args)
    for _ in range(2):
        pipe.replay()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    g0 = torch.cuda.Event(enable_timing=True)
    g1 = torch.cuda.Event(enable_timing=True)
    g0.record()
    for _ in range(a.steps):
        pipe.replay()
    g1.record()
    torch.cuda.synchronize()
    pipe.check()
    g_ms = max_over_ranks(g0.elapsed_time(g1), dev)
    graph = {"ms_per_step": g_ms / a.steps, "kernels_per_step": graph_kernels,
             "value": (n * world) / (g_ms / a.steps / 1e3) / 1e6}
    ms_max = max_over_ranks(ms, dev)
    ms_step = ms_max / a.steps
    value = (n * world) / (ms_step / 1e3) / 1e6

    # result sizes (for the algorithmic bytes)
    import ctypes
    from rvpoint_b200 import _lib as L
    vo_h, so_h = pipe.frame_offsets()
    n_vox, n_sor = int(vo_h[-1]), int(so_h[-1])

    # ---- e2e: host buffers through the C entry point, copies inside
    e2e = None
    h2d = d2h = 0
    if rank == 0 or world > 1:
        pin = lambda arr: torch.from_numpy(arr).pin_memory()  # noqa: E731
        hx, hy, hz = pin(batch.x), pin(batch.y), pin(batch.z)
        ho = pin(batch.offsets)
        out_vox = torch.empty((n, 3), dtype=torch.float32).pin_memory()
        out_sor = torch.empty((n, 3), dtype=torch.float32).pin_memory()
        out_vo = torch.empty(nf + 1, dtype=torch.int64).pin_memory()
        out_so = torch.empty(nf + 1, dtype=torch.int64).pin_memory()
        out_n = [torch.empty(n, dtype=torch.float32).pin_memory() for _ in range(3)]
        out_m = torch.empty((nf, 4), dtype=torch.float32).pin_memory()
        out_c = torch.empty(nf, dtype=torch.int32).pin_memory()
        pipe.set_timing(0)
        ctx.set_stream(torch.cuda.current_stream(dev).cuda_stream)
        P = lambda t_: ctypes.c_void_p(t_.data_ptr())  # noqa: E731

        def run_host():
            L.check(pipe.L.rvp_pipeline_run_host(pipe.h, P(hx), P(hy), P(hz), P(ho), nf,
                                                 P(out_vox), P(out_vo), P(out_sor), P(out_so),
                                                 P(out_n[0]), P(out_n[1]), P(out_n[2]),
                                                 P(out_m), P(out_c)), ctx.h)
        run_host()
        e_steps = max(2, a.steps)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(e_steps):
            run_host()
        e1.record()
        torch.cuda.synchronize()
        single_ms = e0.elapsed_time(e1) / e_steps

        # the same steps through rvp_pipeline_run_host_batches: step i + 1's
        # inputs go up and step i's results come down while a step runs
        # (every step still copies its inputs up and its results down)
        def arr(t_):
            return (ctypes.c_void_p * e_steps)(*([t_.data_ptr()] * e_steps))
        nfa = (ctypes.c_int * e_steps)(*([nf] * e_steps))

        def run_batches():
            L.check(pipe.L.rvp_pipeline_run_host_batches(
                pipe.h, e_steps, arr(hx), arr(hy), arr(hz), arr(ho), nfa, arr(out_vox),
                arr(out_vo), arr(out_sor), arr(out_so), arr(out_n[0]), arr(out_n[1]),
                arr(out_n[2]), arr(out_m), arr(out_c)), ctx.h)
        run_batches()
        torch.cuda.synchronize()
        e0.record()
        run_batches()
        e1.record()
        torch.cuda.synchronize()
        e_ms = e0.elapsed_time(e1) / e_steps
        h2d = 12 * n + 8 * (nf + 1)
        d2h = 8 * (nf + 1) * 2 + 12 * n_vox + 12 * n_sor + 12 * n_sor + 16 * nf + 4 * nf
        e_max = max_over_ranks(e_ms, dev)
        e2e = {"value": (n * world) / (e_max / 1e3) / 1e6, "unit": UNIT,
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e_max, "steps": e_steps,
               "api": "rvp_pipeline_run_host_batches (steps in a row, copies overlapped)",
               "single_call_ms_per_step": max_over_ranks(single_ms, dev)}

    if world > 1:
        dist.barrier()
    if rank != 0:
        dist.destroy_process_group()
        return

    # ---- roofline of the longest kernel timed live (per-level SOR kNN
    # kernels and RANSAC)
    coop = int(pipe.cfg.queries_per_warp) == 3
    counts = pipe.knn_counts() if coop else None
    routed = counts[0] if coop else None
    cand = {}
    for k in LEVEL_STAGES + ("ransac",):
        if stages.get(k, 0.0) <= 0.0:
            continue
        u = None if k == "ransac" else kernel_units(k, coop, counts, n_vox)
        if k == "ransac" or u:
            cand[k] = u
    dom = max(cand, key=lambda k: stages[k])
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
        peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    alg = kernel_bytes(dom, cand[dom], n_sor, nf)
    achieved = alg / (stages[dom] / 1e3) / 1e9
    dom_name = kernel_name(dom, coop)
    traffic = None
    tf = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tf):
        try:
            tr = json.load(open(tf)).get(dom)
            # captured on a smaller case: scaled by the queries processed
            # (traffic grows in proportion to them)
            if tr and tr.get("kernel") == dom_name and cand[dom]:
                traffic = tr["bytes"] * cand[dom] / tr["units"]
        except Exception:
            traffic = None
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "kernel": dom_name,
            "stage": dom, "peak_source": peak_src, "queries": cand[dom],
            "algorithmic_bytes_per_launch": alg, "launch_ms": stages[dom],
            "cooperative_queries": routed, "adaptive_queries": counts[1] if coop else None}

    cpu = singles = None
    if world == 1:
        pipe.run_device(*args)  # the timed batch once more, then its results to the host
        torch.cuda.synchronize()
        singles = single_cloud_legs(ctx) if not a.no_singles else None
        cpu, cpu_single = cpu_baseline(batch, a.cpu_frames, pipe.results(),
                                       singles=singles is not None)
        if singles is not None and cpu_single:
            rc = cpu_single.get("room_chain_100k")
            if rc:
                t = sum(rc["seconds"].values())
                singles["room_chain_100k"].update(
                    {"cpu_ms": t * 1e3, "cpu_mpts_s": 0.1 / t, "cpu_stage_s": rc["seconds"],
                     "cpu_cores": 1, "cpu_same_sizes": rc["voxels"] == singles[
                         "room_chain_100k"]["voxels"] and rc["kept"] == singles[
                         "room_chain_100k"]["kept"] and rc["ransac"] == singles[
                         "room_chain_100k"]["ransac"]})
            lr = cpu_single.get("lidar_frame_radius")
            if lr:
                singles["lidar_frame_radius"].update(
                    {"radius_cpu_ms": lr["radius_s"] * 1e3, "max_nn16_cpu_ms": lr["knn16_s"] * 1e3,
                     "cpu_cores": 1, "cpu_pairs_r05": lr["pairs"]})
    learned = learned_leg(ctx, a.learned_scenes, 64) if a.learned_scenes > 0 else None
    nxt = next_rows_leg(ctx, batch) if world == 1 and not a.no_next_rows else None
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "frames_per_gpu": nf, "points_per_gpu": n,
                       "voxel_points": n_vox, "sor_points": n_sor, "leaf": LEAF,
                       "sor_k": SOR_K, "normal_k": NORMAL_K, "ransac_iters": R_ITERS,
                       "ransac_thresh": R_THRESH, "parallelism": f"frames x{world}",
                       "l2": "inputs larger than L2 (no flush)",
                       "tuning": best},
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches_per_step * a.steps, "clocks": clk,
            "stages_ms": {k: v for k, v in stages.items() if k != "runs"},
            "graph": graph, "learned_ransac": learned, "next_rows": nxt,
            "single_cloud": singles}
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
