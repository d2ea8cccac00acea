"""GPU parity: every entry point through the C ABI against the CPU oracle
(the plain-C restatement of the reference's scalar path, itself pinned to the
reference in test_oracle.py), on seeded inputs the oracle finishes in seconds.

Bit-exact: neighbour lists (index, d2), voxel centroids and keys, SOR mean
distances / keep masks / outputs, RANSAC per-hypothesis counts, best count and
model. Tolerance: normals (CUDA's atan2f/cosf/sinf differ from glibc by ulps).
"""
import numpy as np
import pytest

from rvpoint_b200 import datasets as D

pytestmark = pytest.mark.gpu


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


def room(n, seed=7):
    return D.room_cloud(n=n, seed=seed)


def lidar_sub(n, seed=11):
    f = D.lidar_frame(seed=seed)
    rng = np.random.default_rng(seed)
    sel = np.sort(rng.choice(f.n, size=min(n, f.n), replace=False))
    return f.subset(sel)


# ---------------------------------------------------------------------------
# SpatialHash
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("cloud_fn,cell,radius", [
    (lambda: room(20000), 0.03, 0.03),
    (lambda: room(20000), 0.05, 0.03),
    (lambda: room(20000), 0.02, 0.05),
    (lambda: lidar_sub(30000), 0.5, 0.5),
    (lambda: lidar_sub(30000), 1.0, 0.5),
])
def test_radius_search_bit_exact(gpu_ctx, restatement, cloud_fn, cell, radius):
    from rvpoint_b200.api import SpatialHash
    c = cloud_fn()
    h = SpatialHash()
    h.setInputCloud(c, cell)
    h.build()
    assert not h.hasCollisions()
    offs, idx, d2 = h.radiusSearchBatch(c.x, c.y, c.z, radius)
    o2, i2, e2 = restatement.radius_search(c, cell, radius)
    assert np.array_equal(offs, o2)
    assert np.array_equal(idx, i2)
    assert np.array_equal(bits(d2), bits(e2))


@pytest.mark.parametrize("max_nn", [1, 16, 33, 100])
def test_radius_search_max_nn(gpu_ctx, restatement, max_nn):
    from rvpoint_b200.api import SpatialHash
    c = lidar_sub(20000)
    h = SpatialHash()
    h.setInputCloud(c, 0.5)
    h.build()
    offs, idx, d2 = h.radiusSearchBatch(c.x, c.y, c.z, 0.5, max_nn=max_nn)
    o2, i2, e2 = restatement.radius_search(c, 0.5, 0.5, max_nn=max_nn)
    assert np.array_equal(offs, o2)
    assert np.array_equal(idx, i2)
    assert np.array_equal(bits(d2), bits(e2))


def test_radius_search_foreign_queries_and_single(gpu_ctx, restatement):
    from rvpoint_b200.api import SpatialHash
    c = room(10000)
    rng = np.random.default_rng(3)
    q = D.Cloud.from_xyz(rng.uniform(-1.0, 5.0, size=(3000, 3)))  # many outside the bbox
    h = SpatialHash()
    h.setInputCloud(c, 0.04)
    h.build()
    offs, idx, d2 = h.radiusSearchBatch(q.x, q.y, q.z, 0.1)
    o2, i2, e2 = restatement.radius_search(c, 0.04, 0.1, queries=q)
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)
    assert np.array_equal(bits(d2), bits(e2))
    ind, dd = [], []
    n = h.radiusSearch((q.x[5], q.y[5], q.z[5]), 0.1, ind, dd)
    assert n == o2[6] - o2[5] and ind == list(i2[o2[5]:o2[6]])


def test_radius_search_dense_cluster_big_segments(gpu_ctx, restatement):
    """Lists longer than the per-warp staging buffer take the block sort."""
    from rvpoint_b200.api import SpatialHash
    rng = np.random.default_rng(5)
    p = np.concatenate([rng.normal(0, 0.05, size=(6000, 3)), rng.uniform(-2, 2, size=(2000, 3))])
    c = D.Cloud.from_xyz(p)
    h = SpatialHash()
    h.setInputCloud(c, 0.5)
    h.build()
    offs, idx, d2 = h.radiusSearchBatch(c.x, c.y, c.z, 0.3)
    o2, i2, e2 = restatement.radius_search(c, 0.5, 0.3)
    assert (np.diff(o2) > 1024).any()
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)
    assert np.array_equal(bits(d2), bits(e2))


def test_radius_search_duplicates_and_boundary(gpu_ctx, restatement):
    """Duplicate points, points exactly at the radius, cells at the bbox edge."""
    from rvpoint_b200.api import SpatialHash
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(5), indexing="ij"), -1)
    p = (g.reshape(-1, 3) * 0.25).astype(np.float32)
    p = np.concatenate([p, p[::7]])  # duplicates
    c = D.Cloud.from_xyz(p)
    for cell, r in [(0.25, 0.25), (0.5, 0.25), (0.1, 0.5), (0.25, 0.0)]:
        h = SpatialHash()
        h.setInputCloud(c, cell)
        h.build()
        offs, idx, d2 = h.radiusSearchBatch(c.x, c.y, c.z, r)
        o2, i2, e2 = restatement.radius_search(c, cell, r)
        assert np.array_equal(offs, o2) and np.array_equal(idx, i2), (cell, r)


def test_radius_search_collision_primes(gpu_ctx, restatement):
    """With primes that make cells collide, the reference's own window and
    duplicate hits are reproduced."""
    from rvpoint_b200.api import SpatialHash
    c = room(4000)
    h = SpatialHash()
    h.setHashPrimes(3, 5)
    h.setInputCloud(c, 0.1)
    h.build()
    assert h.hasCollisions()
    offs, idx, d2 = h.radiusSearchBatch(c.x, c.y, c.z, 0.1)
    o2, i2, e2 = restatement.radius_search(c, 0.1, 0.1, p1=3, p2=5)
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)


def test_empty_inputs(gpu_ctx):
    from rvpoint_b200 import api
    e = D.Cloud.from_xyz(np.zeros((0, 3), np.float32))
    h = api.SpatialHash()
    h.setInputCloud(e, 0.1)
    h.build()
    offs, idx, d2 = h.radiusSearchBatch(np.zeros(3, np.float32), np.zeros(3, np.float32),
                                        np.zeros(3, np.float32), 0.5)
    assert list(offs) == [0, 0, 0, 0] and len(idx) == 0
    assert len(api.voxel_grid_downsamp_rvv_v2(e, 0.1)) == 0
    assert len(api.sor_rvv(e, 10, 1.0)) == 0
    assert api.ransac_plane_rvv(D.Cloud.from_xyz(np.ones((2, 3))), 0.1, 100)[0] == 0


# ---------------------------------------------------------------------------
# kNN
# ---------------------------------------------------------------------------
def brute_knn(c, q, k):
    P = c.aos().astype(np.float32)
    Q = q.aos().astype(np.float32)
    out_i = np.zeros((Q.shape[0], k), np.int32)
    out_d = np.zeros((Q.shape[0], k), np.float32)
    for s in range(0, Q.shape[0], 512):
        qq = Q[s:s + 512]
        dx = (P[None, :, 0] - qq[:, None, 0]).astype(np.float32)
        dy = (P[None, :, 1] - qq[:, None, 1]).astype(np.float32)
        dz = (P[None, :, 2] - qq[:, None, 2]).astype(np.float32)
        d2 = ((dx * dx + dy * dy).astype(np.float32) + dz * dz).astype(np.float32)
        key = (d2.view(np.uint32).astype(np.uint64) << np.uint64(32)) | np.arange(P.shape[0], dtype=np.uint64)[None, :]
        part = np.argpartition(key, k - 1, axis=1)[:, :k]
        kk = np.take_along_axis(key, part, 1)
        o = np.argsort(kk, axis=1)
        sel = np.take_along_axis(part, o, 1)
        out_i[s:s + 512] = sel
        out_d[s:s + 512] = np.take_along_axis(d2, sel, 1)
    return out_i, out_d


@pytest.mark.parametrize("k", [8, 17, 31, 33, 64])
def test_knn_exact_unbounded(gpu_ctx, k):
    from rvpoint_b200.api import SpatialHash
    c = D.room_cloud(n=6000, seed=21)
    h = SpatialHash()
    h.setInputCloud(c, 0.05)
    h.build()
    idx, d2, cnt = h.knn(c.x, c.y, c.z, k)
    bi, bd = brute_knn(c, c, k)
    assert (cnt == k).all()
    assert np.array_equal(idx, bi)
    assert np.array_equal(bits(d2), bits(bd))


# ---------------------------------------------------------------------------
# voxel grid
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("n,leaf", [(20000, 0.01), (20000, 0.05), (50000, 0.1)])
def test_voxel_bit_exact(gpu_ctx, restatement, n, leaf):
    from rvpoint_b200 import api
    c = room(n)
    out, keys = api.voxel_grid_downsamp_rvv_v2(c, leaf, return_keys=True)
    o2, k2 = restatement.voxel_grid(c, leaf)
    assert out.shape == o2.shape
    assert np.array_equal(bits(out), bits(o2))
    assert np.array_equal(keys, k2)


def test_voxel_negative_coordinates(gpu_ctx, restatement):
    from rvpoint_b200 import api
    c = lidar_sub(40000)
    out = api.voxel_grid_downsamp_rvv_v2(c, 0.1)
    o2, _ = restatement.voxel_grid(c, 0.1)
    assert np.array_equal(bits(out), bits(o2))


# ---------------------------------------------------------------------------
# SOR
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("k,alpha", [(30, 1.0), (16, 1.0), (10, 0.5)])
def test_sor_exact_bit_exact(gpu_ctx, restatement, k, alpha):
    from rvpoint_b200 import api
    c = room(6000, seed=31)
    out, md, keep = api.sor_rvv(c, k, alpha, return_stats=True)
    o2, md2, keep2 = restatement.sor_exact(c, k, alpha)
    assert np.array_equal(bits(md), bits(md2))
    assert np.array_equal(keep.astype(bool), keep2)
    assert np.array_equal(bits(out), bits(o2))


def test_sor_spatial_hash_bit_exact(gpu_ctx, restatement):
    from rvpoint_b200 import api
    c = room(8000, seed=41)
    h = api.SpatialHash()
    h.setInputCloud(c, 0.1)
    h.build()
    out, md, keep = api.sor_spatial_hash(c, h, 16, 1.0, 0.1, return_stats=True)
    o2, md2, keep2 = restatement.sor_radius(c, 0.1, 16, 1.0, 0.1)
    assert np.array_equal(bits(md), bits(md2))
    assert np.array_equal(bits(out), bits(o2))


# ---------------------------------------------------------------------------
# normals (FP32 tolerance against the FP64 oracle)
# ---------------------------------------------------------------------------
def _angle_err(a, b):
    a = a / np.maximum(np.linalg.norm(a, axis=1, keepdims=True), 1e-30)
    b = b / np.maximum(np.linalg.norm(b, axis=1, keepdims=True), 1e-30)
    return np.arccos(np.clip(np.abs((a * b).sum(1)), 0, 1))


def test_normals_radius(gpu_ctx, restatement):
    from rvpoint_b200 import api
    v, _ = restatement.voxel_grid(room(30000, seed=51), 0.01)
    c = D.Cloud.from_xyz(v)
    h = api.SpatialHash()
    h.setInputCloud(c, 0.03)
    h.build()
    nx, ny, nz = api.normal_estimation_rvv(c, h, 10, 0.03)
    g = np.stack([nx, ny, nz], 1)
    f32 = restatement.normals_radius(c, 0.03, 0.03)
    f64 = restatement.normals_radius(c, 0.03, 0.03, f64=True)
    zero = np.all(f32 == 0, axis=1)
    assert np.array_equal(np.all(g == 0, axis=1), zero)  # same "< 3 neighbours" set
    e_gpu = _angle_err(g[~zero], f64[~zero])
    e_cpu = _angle_err(f32[~zero], f64[~zero])
    tol = 1e-3  # rad, FP32 tolerance against FP64
    # GPU FP32 is as close to FP64 as the reference's own FP32 path
    assert (e_gpu > tol).mean() <= (e_cpu > tol).mean() + 0.002
    assert np.quantile(e_gpu, 0.99) < 1e-2
    # and follows the reference's FP32 arithmetic closely
    assert (_angle_err(g[~zero], f32[~zero]) < 1e-4).mean() > 0.99


def test_normals_knn(gpu_ctx, restatement):
    from rvpoint_b200 import api
    v, _ = restatement.voxel_grid(room(8000, seed=61), 0.02)
    c = D.Cloud.from_xyz(v)
    nx, ny, nz = api.normal_estimation_sc(c, 16)
    g = np.stack([nx, ny, nz], 1)
    f32 = restatement.normals_knn(c, 16)
    f64 = restatement.normals_knn(c, 16, f64=True)
    e_gpu = _angle_err(g, f64)
    e_cpu = _angle_err(f32, f64)
    assert (e_gpu > 1e-3).mean() <= (e_cpu > 1e-3).mean() + 0.002
    assert (_angle_err(g, f32) < 1e-4).mean() > 0.99
    # sign convention: flipped towards the viewpoint like the reference
    same_sign = np.sign((g * f32).sum(1))
    assert (same_sign > 0).mean() > 0.99


# ---------------------------------------------------------------------------
# RANSAC
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("thresh,iters", [(0.01, 1000), (0.05, 300), (0.002, 2000)])
def test_ransac_bit_exact(gpu_ctx, restatement, thresh, iters):
    from oracle.oracle import libc_rand_stream
    from rvpoint_b200 import api
    c = room(30000, seed=71)
    rs = libc_rand_stream(3 * iters)
    best, model, counts, it = api.ransac_plane_rvv(c, thresh, iters, rand_stream=rs,
                                                   return_counts=True)
    b2, m2, c2, _, it2 = restatement.ransac_plane(c, thresh, iters, rs)
    assert best == b2 and it == it2
    assert np.array_equal(bits(model), bits(m2))
    assert np.array_equal(counts, c2)  # every hypothesis, bit-exact


def test_ransac_libc_stream_and_state(gpu_ctx, restatement):
    """Without an explicit stream the library draws srand(0)/rand() from libc
    and leaves the generator where the reference leaves it."""
    import ctypes
    from oracle.oracle import libc_rand_stream
    from rvpoint_b200 import api
    c = room(20000, seed=81)
    best, model = api.ransac_plane_rvv(c, 0.01, 1000)
    rs = libc_rand_stream(3000)
    b2, m2, _, _, it2 = restatement.ransac_plane(c, 0.01, 1000, rs)
    assert best == b2 and np.array_equal(bits(model), bits(m2))
    libc = ctypes.CDLL("libc.so.6")
    api.ransac_plane_rvv(c, 0.01, 1000)
    nxt = libc.rand()
    assert nxt == rs[3 * it2]


def test_extract_plane(gpu_ctx, restatement):
    from rvpoint_b200 import api
    c = room(20000, seed=91)
    m = np.array([0.0, 0.0, 1.0, -0.001], np.float32)
    a, b = api.extract_plane_inliers_outliers_rvv(c, m, 0.01)
    a2, b2 = restatement.extract_plane(c, m, 0.01)
    assert np.array_equal(a, a2) and np.array_equal(b, b2)


# ---------------------------------------------------------------------------
# batched frames
# ---------------------------------------------------------------------------
def test_pipeline_frames_match_per_frame_oracle(gpu_ctx, restatement):
    from oracle.oracle import libc_rand_stream
    from rvpoint_b200 import api
    batch = D.lidar_batch(n_frames=4, seed=5, min_pts=3000, max_pts=9000)
    p = api.Pipeline(max_points=batch.n, max_frames=batch.n_frames, leaf_size=0.1, sor_k=16,
                     sor_alpha=1.0, normal_k=16, ransac_thresh=0.05, ransac_iters=1000)
    r = p.run_host(batch)
    rs = libc_rand_stream(3000)
    for f in range(batch.n_frames):
        fr = batch.frame(f)
        v, _ = restatement.voxel_grid(fr, 0.1)
        a, b = r["voxel_offsets"][f], r["voxel_offsets"][f + 1]
        assert np.array_equal(bits(r["voxel"][a:b]), bits(v)), f
        vc = D.Cloud.from_xyz(v)
        s, md, keep = restatement.sor_exact(vc, 16, 1.0)
        a, b = r["sor_offsets"][f], r["sor_offsets"][f + 1]
        assert np.array_equal(bits(r["sor"][a:b]), bits(s)), f
        sc = D.Cloud.from_xyz(s)
        n32 = restatement.normals_knn(sc, 16)
        n64 = restatement.normals_knn(sc, 16, f64=True)
        e = _angle_err(r["normals"][a:b], n64)
        e_cpu = _angle_err(n32, n64)
        assert (e > 1e-3).mean() <= (e_cpu > 1e-3).mean() + 0.005, f
        best, model, _, _, _ = restatement.ransac_plane(sc, 0.05, 1000, rs)
        assert r["ransac_count"][f] == best, f
        assert np.array_equal(bits(r["ransac_model"][f]), bits(model)), f


def test_pipeline_tile_and_warp_paths_agree(gpu_ctx):
    """The per-lane kNN kernels, the warp-per-query kernel and the cooperative
    level-0 pass give identical SOR output and normals on a full-size frame
    batch."""
    from rvpoint_b200 import api
    batch = D.lidar_batch(n_frames=3, seed=9)
    outs = []
    for qpw in (0, 1, 3):
        p = api.Pipeline(max_points=batch.n, max_frames=batch.n_frames, cell_size=0.3,
                         queries_per_warp=qpw)
        outs.append(p.run_host(batch))
    a = outs[0]
    for b in outs[1:]:
        assert np.array_equal(a["sor_offsets"], b["sor_offsets"])
        assert np.array_equal(bits(a["sor"]), bits(b["sor"]))
        assert np.array_equal(bits(a["normals"]), bits(b["normals"]))
        assert np.array_equal(a["ransac_count"], b["ransac_count"])


def test_pipeline_search_radius_factor_does_not_change_results(gpu_ctx):
    from rvpoint_b200 import api
    batch = D.lidar_batch(n_frames=3, seed=17)
    outs = []
    for rf in (0.0, 0.6, 1.5):
        p = api.Pipeline(max_points=batch.n, max_frames=batch.n_frames, cell_size=0.5)
        p.set_search_radius_factor(rf)
        outs.append(p.run_host(batch))
    for o in outs[1:]:
        assert np.array_equal(bits(o["sor"]), bits(outs[0]["sor"]))
        assert np.array_equal(bits(o["normals"]), bits(outs[0]["normals"]))


@pytest.mark.parametrize("cell", [0.15, 0.3, 0.8])
def test_pipeline_cell_size_does_not_change_results(gpu_ctx, restatement, cell):
    from rvpoint_b200 import api
    batch = D.lidar_batch(n_frames=2, seed=13, min_pts=4000, max_pts=12000)
    p = api.Pipeline(max_points=batch.n, max_frames=batch.n_frames, cell_size=cell)
    r = p.run_host(batch)
    for f in range(batch.n_frames):
        v, _ = restatement.voxel_grid(batch.frame(f), 0.1)
        s, _, _ = restatement.sor_exact(D.Cloud.from_xyz(v), 16, 1.0)
        a, b = r["sor_offsets"][f], r["sor_offsets"][f + 1]
        assert np.array_equal(bits(r["sor"][a:b]), bits(s))


def test_pipeline_graph_replay_matches_direct_runs(gpu_ctx):
    """One run captured as a CUDA graph and replayed gives the direct run's
    results bit for bit, also after new frames are copied into the captured
    input buffers."""
    import torch
    from rvpoint_b200 import api
    b1 = D.lidar_batch(n_frames=3, seed=21, min_pts=20000, max_pts=60000)
    b2 = D.lidar_batch(n_frames=3, seed=22, min_pts=20000, max_pts=60000)
    cap_n = max(b1.n, b2.n)
    dev = torch.device("cuda", 0)
    bufs = [torch.zeros(cap_n, dtype=torch.float32, device=dev) for _ in range(3)]
    offs = torch.zeros(4, dtype=torch.int64, device=dev)

    def load(b):
        for t, a in zip(bufs, (b.x, b.y, b.z)):
            t[:b.n].copy_(torch.from_numpy(a))
        offs.copy_(torch.from_numpy(b.offsets))

    direct = api.Pipeline(max_points=cap_n, max_frames=3)
    ref = [direct.run_host(b) for b in (b1, b2)]

    g = api.Pipeline(max_points=cap_n, max_frames=3)
    load(b1)
    g.run_device(*bufs, offs, 3, b1.n)  # sizes every buffer before the capture
    kernels = g.capture(*bufs, offs, 3, b1.n)
    assert kernels > 20
    for b, r in zip((b1, b1), (ref[0], ref[0])):
        load(b)
        g.replay()
        out = g.results()
        for key in ("voxel", "sor", "normals", "ransac_model"):
            assert np.array_equal(bits(out[key]), bits(r[key])), key
        assert np.array_equal(out["ransac_count"], r["ransac_count"])
    # the graph keeps n_points: a second batch of another size needs a new capture
    load(b2)
    g.capture(*bufs, offs, 3, b2.n)
    g.replay()
    out = g.results()
    for key in ("voxel", "sor", "normals"):
        assert np.array_equal(bits(out[key]), bits(ref[1][key])), key


def test_pipeline_level_kernel_times(gpu_ctx):
    """Per-level kNN kernel timing: positive at level 0, and each stage's
    level kernels fit inside the stage."""
    import torch
    from rvpoint_b200 import api
    b = D.lidar_batch(n_frames=4, seed=23)
    dev = torch.device("cuda", 0)
    x, y, z = (torch.from_numpy(a).to(dev) for a in (b.x, b.y, b.z))
    offs = torch.from_numpy(b.offsets).to(dev)
    p = api.Pipeline(max_points=b.n, max_frames=4)
    p.run_device(x, y, z, offs, 4, b.n)
    p.set_timing(2)
    for _ in range(2):
        p.run_device(x, y, z, offs, 4, b.n)
    t = p.stage_times(levels=True)
    assert t["runs"] == 2
    assert t["sor_knn_l0"] > 0 and t["normals_knn_l0"] > 0
    timed = ("knn_l0", "knn_l1", "knn_l2", "knn_coop")
    assert sum(t[f"sor_{k}"] for k in timed) <= t["sor_knn"] * 1.001
    assert (sum(t[f"normals_{k}"] for k in timed)
            <= t["normals_knn"] * 1.001)


@pytest.mark.gpu
def test_pipeline_lane_levels_do_not_change_results(gpu_ctx):
    """Handing queries to the warp-per-query kernel after 1, 2 or 3 grid
    levels changes the work, not the results."""
    from rvpoint_b200 import api
    batch = D.lidar_batch(n_frames=3, seed=29)
    outs = []
    for ll in (0, 1, 2):
        p = api.Pipeline(max_points=batch.n, max_frames=batch.n_frames, cell_size=0.5)
        p.set_lane_levels(ll)
        outs.append(p.run_host(batch))
    for o in outs[1:]:
        assert np.array_equal(bits(o["sor"]), bits(outs[0]["sor"]))
        assert np.array_equal(bits(o["normals"]), bits(outs[0]["normals"]))
        assert np.array_equal(o["ransac_count"], outs[0]["ransac_count"])


@pytest.mark.gpu
@pytest.mark.parametrize("src,tol,mn,mx", [("room", 0.02, 3, 100000), ("lidar", 0.5, 1, 200)])
def test_euclidean_clusters_match_golden(gpu_ctx, src, tol, mn, mx):
    """EuclideanClustering::extract: the same clusters, in the same order,
    with the same sorted indices as the reference (golden fixtures)."""
    import os
    from rvpoint_b200 import api
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden.npz"))
    a = g[src]
    c = D.Cloud(np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1]),
                np.ascontiguousarray(a[:, 2]))
    cl = api.euclidean_clusters(c, tol, mn, mx, ctx=gpu_ctx)
    offs = np.cumsum([0] + [len(k) for k in cl]).astype(np.int64)
    assert np.array_equal(offs, g[f"ec_{src}_offsets"])
    assert np.array_equal(np.concatenate(cl).astype(np.int32), g[f"ec_{src}_idx"])


@pytest.mark.gpu
def test_euclidean_clusters_match_oracle_larger(gpu_ctx, restatement):
    from rvpoint_b200 import api
    fr = D.lidar_frame(seed=777)
    c = fr.subset(np.arange(0, fr.n, 5))
    for tol, mn, mx in ((0.3, 1, 2**31 - 1), (0.6, 5, 5000), (0.05, 1, 3)):
        got = api.euclidean_clusters(c, tol, mn, mx, ctx=gpu_ctx)
        ref = restatement.euclidean_clusters(c, tol, mn, mx)
        assert len(got) == len(ref)
        for u, v in zip(got, ref):
            assert np.array_equal(u, v)
    # device arrays in place; empty cloud
    import torch
    xs = [torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (c.x, c.y, c.z)]
    got = api.euclidean_clusters(tuple(xs), 0.3, ctx=gpu_ctx)
    ref = restatement.euclidean_clusters(c, 0.3)
    assert len(got) == len(ref) and all(np.array_equal(u, v) for u, v in zip(got, ref))
    e = np.zeros(0, np.float32)
    assert api.euclidean_clusters((e, e, e), 0.3, ctx=gpu_ctx) == []


@pytest.mark.gpu
def test_pipeline_host_batches_equal_single_runs(gpu_ctx):
    """rvp_pipeline_run_host_batches (inputs double-buffered, results coming
    down while the next batch runs) returns, batch by batch, what
    rvp_pipeline_run_host returns for each batch alone: batches of different
    sizes in a row, one repeated."""
    from rvpoint_b200 import api
    bs = [D.lidar_batch(n_frames=4, seed=s, min_pts=20000, max_pts=80000) for s in (31, 32, 33)]
    seq = [bs[0], bs[1], bs[0], bs[2]]
    cap_n = max(b.n for b in bs)
    p = api.Pipeline(max_points=cap_n, max_frames=4)
    ref = {id(b): p.run_host(b) for b in bs}
    outs = p.run_host_batches(seq)
    assert len(outs) == len(seq)
    for b, out in zip(seq, outs):
        r = ref[id(b)]
        for key in ("voxel", "sor", "normals", "ransac_model"):
            assert np.array_equal(bits(out[key]), bits(r[key])), key
        for key in ("voxel_offsets", "sor_offsets", "ransac_count"):
            assert np.array_equal(out[key], r[key]), key
    p.close()
