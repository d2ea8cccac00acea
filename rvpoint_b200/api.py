"""Python host API mirroring the reference's operator interface (namespace
rvpoint of Mumu-kun/rvpoint) on top of the C ABI.

Names, argument meaning and degenerate-input behaviour follow the reference:

* ``SpatialHash``  -- search/spatial_hashing.h:12-53 (setInputCloud, build,
  radiusSearch, setHashPrimes) plus batched queries;
* ``voxel_grid_downsamp_{sc,rvv,rvv_v2}`` -- filters/voxel_grid.h:14-34;
* ``sor_{sc,rvv,spatial_hash}`` -- filters/statistical_outlier_removal.h:18-36;
* ``normal_estimation_{sc,rvv}`` -- features/normal_estimation.h:15-34;
* ``ransac_plane_{sc,rvv}``, ``extract_plane_*`` -- segmentation/ransac_plane.h.

Where the reference fills a caller-allocated ``PointXYZ* out`` and returns a
count, these functions return the filled rows (``len`` is the count). Inputs
are numpy arrays (host) or CUDA torch tensors (device, used in place on the
current torch stream). Every call reaches the CUDA kernels; there is no CPU
path.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import MEM_DEVICE, MEM_HOST, check

try:  # torch is optional plumbing (device memory / streams)
    import torch
except Exception:  # pragma: no cover
    torch = None


def _is_dev(a) -> bool:
    return torch is not None and isinstance(a, torch.Tensor) and a.is_cuda


def _f32(a):
    if _is_dev(a):
        assert a.dtype == torch.float32 and a.is_contiguous(), "float32 contiguous tensor expected"
        return a
    return np.ascontiguousarray(a, dtype=np.float32)


def _ptr(a):
    if a is None:
        return None
    if _is_dev(a):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


def _xyz(cloud):
    """Accept a datasets.Cloud, a (x, y, z) triple or an (n, 3) array."""
    if hasattr(cloud, "x") and hasattr(cloud, "y") and hasattr(cloud, "z"):
        return _f32(cloud.x), _f32(cloud.y), _f32(cloud.z)
    if isinstance(cloud, (tuple, list)) and len(cloud) == 3:
        return _f32(cloud[0]), _f32(cloud[1]), _f32(cloud[2])
    a = cloud
    if _is_dev(a):
        return a[:, 0].contiguous(), a[:, 1].contiguous(), a[:, 2].contiguous()
    a = np.asarray(a, dtype=np.float32)
    return (np.ascontiguousarray(a[:, 0]), np.ascontiguousarray(a[:, 1]),
            np.ascontiguousarray(a[:, 2]))


def _empty(shape, dtype, like_dev: bool, device=None):
    if like_dev:
        tdt = {np.float32: torch.float32, np.int32: torch.int32, np.int64: torch.int64,
               np.uint8: torch.uint8}[dtype]
        return torch.empty(shape, dtype=tdt, device=device)
    return np.empty(shape, dtype=dtype)


class Context:
    """One CUDA device + stream + scratch arena (rvp_context)."""

    def __init__(self, device: int = 0):
        self.L = _lib.load()
        h = C.c_void_p()
        check(self.L.rvp_context_create(device, C.byref(h)))
        self.h = h
        self.device = device

    def set_stream(self, stream_handle: int) -> None:
        check(self.L.rvp_context_set_stream(self.h, C.c_void_p(stream_handle)), self.h)

    def use_torch_stream(self) -> None:
        if torch is not None and torch.cuda.is_available():
            self.set_stream(torch.cuda.current_stream(self.device).cuda_stream)

    def synchronize(self) -> None:
        check(self.L.rvp_context_synchronize(self.h), self.h)

    @property
    def launches(self) -> int:
        return int(self.L.rvp_context_launch_count(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self.L.rvp_context_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


def _mem_of(*arrays) -> int:
    devs = [_is_dev(a) for a in arrays if a is not None]
    if devs and all(devs):
        return MEM_DEVICE
    if any(devs):
        raise ValueError("mixing host and device arrays in one call")
    return MEM_HOST


def _prep(ctx: Context, mem: int) -> None:
    if mem == MEM_DEVICE:
        ctx.use_torch_stream()
    else:
        ctx.set_stream(0)


# ---------------------------------------------------------------------------
# SpatialHash
# ---------------------------------------------------------------------------
class SpatialHash:
    """search/spatial_hashing.h:12-53 on the GPU."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.rvp_hash_create(self.ctx.h, C.byref(h)), self.ctx.h)
        self.h = h
        self.n = 0

    def setHashPrimes(self, p1: int, p2: int) -> None:
        check(self.L.rvp_hash_set_primes(self.h, p1, p2), self.ctx.h)

    def setInputCloud(self, cloud, cell_size: float) -> None:
        x, y, z = _xyz(cloud)
        mem = _mem_of(x, y, z)
        _prep(self.ctx, mem)
        n = int(x.shape[0])
        check(self.L.rvp_hash_set_input_cloud(self.h, _ptr(x), _ptr(y), _ptr(z), n,
                                              float(cell_size), mem), self.ctx.h)
        self.n = n

    def build(self) -> None:
        _prep(self.ctx, MEM_HOST)
        check(self.L.rvp_hash_build(self.h), self.ctx.h)

    def hasCollisions(self) -> bool:
        v = C.c_int(0)
        check(self.L.rvp_hash_has_collisions(self.h, C.byref(v)), self.ctx.h)
        return bool(v.value)

    def radiusSearch(self, query: Sequence[float], radius: float, indices: Optional[list] = None,
                     dists: Optional[list] = None, max_nn: int = 0) -> int:
        """Single query, reference signature: clears and fills indices/dists
        (sorted by (d2, index)), returns the count."""
        q = np.asarray(query, dtype=np.float32).reshape(3)
        offs, idx, d2 = self.radiusSearchBatch(q[0:1], q[1:2], q[2:3], radius, max_nn)
        if indices is not None:
            indices.clear()
            indices.extend(int(v) for v in idx)
        if dists is not None:
            dists.clear()
            dists.extend(float(v) for v in d2)
        return int(offs[-1])

    def radiusSearchBatch(self, qx, qy, qz, radius: float, max_nn: int = 0,
                          capacity: Optional[int] = None):
        """All queries at once. Returns (offsets[nq+1], indices, dists) CSR."""
        qx, qy, qz = _f32(qx), _f32(qy), _f32(qz)
        mem = _mem_of(qx, qy, qz)
        _prep(self.ctx, mem)
        nq = int(qx.shape[0])
        dev = mem == MEM_DEVICE
        device = qx.device if dev else None
        offs = _empty((nq + 1,), np.int64, dev, device)
        cap = capacity if capacity is not None else (nq * max_nn if max_nn > 0 else 0)
        total = C.c_size_t(0)
        while True:
            idx = _empty((max(cap, 1),), np.int32, dev, device)
            d2 = _empty((max(cap, 1),), np.float32, dev, device)
            st = self.L.rvp_hash_radius_search(self.h, _ptr(qx), _ptr(qy), _ptr(qz), nq,
                                               float(radius), int(max_nn), mem, _ptr(offs),
                                               _ptr(idx), _ptr(d2), cap, C.byref(total))
            if st == _lib.RVP_ERR_CAPACITY:
                cap = int(total.value)
                continue
            check(st, self.ctx.h)
            t = int(total.value)
            return offs, idx[:t], d2[:t]

    def knn(self, qx, qy, qz, k: int, radius: float = 0.0):
        """Exact k nearest (ties by index); radius > 0 bounds the search like
        radiusSearch(q, radius, ..., max_nn=k). Returns (idx[nq,k], d2[nq,k],
        counts[nq]); rows past counts hold -1 / inf."""
        qx, qy, qz = _f32(qx), _f32(qy), _f32(qz)
        mem = _mem_of(qx, qy, qz)
        _prep(self.ctx, mem)
        nq = int(qx.shape[0])
        dev = mem == MEM_DEVICE
        device = qx.device if dev else None
        idx = _empty((nq, k), np.int32, dev, device)
        d2 = _empty((nq, k), np.float32, dev, device)
        cnt = _empty((nq,), np.int32, dev, device)
        check(self.L.rvp_hash_knn(self.h, _ptr(qx), _ptr(qy), _ptr(qz), nq, int(k), float(radius),
                                  mem, _ptr(idx), _ptr(d2), _ptr(cnt)), self.ctx.h)
        return idx, d2, cnt

    def close(self):
        if getattr(self, "h", None):
            self.L.rvp_hash_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# voxel grid
# ---------------------------------------------------------------------------
def voxel_grid_downsamp_rvv_v2(cloud, leaf_size: float, ctx: Optional[Context] = None,
                               return_keys: bool = False):
    """filters/voxel_grid.h:33 -> (V, 3) centroids in (ix, iy, iz) order."""
    ctx = ctx or default_context()
    x, y, z = _xyz(cloud)
    mem = _mem_of(x, y, z)
    _prep(ctx, mem)
    n = int(x.shape[0])
    dev = mem == MEM_DEVICE
    device = x.device if dev else None
    out = _empty((max(n, 1), 3), np.float32, dev, device)
    keys = _empty((max(n, 1), 3), np.int32, dev, device) if return_keys else None
    cnt = C.c_size_t(0)
    check(ctx.L.rvp_voxel_grid(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, float(leaf_size), mem,
                               _ptr(out), _ptr(keys), C.byref(cnt)), ctx.h)
    v = int(cnt.value)
    if return_keys:
        return out[:v], keys[:v]
    return out[:v]


def voxel_grid_downsamp_rvv(cloud, leaf_size: float, ctx=None):
    """filters/voxel_grid.h:21 (same result as _v2 on this path)."""
    return voxel_grid_downsamp_rvv_v2(cloud, leaf_size, ctx)


def voxel_grid_downsamp_sc(points_aos, leaf_size: float, ctx=None):
    """filters/voxel_grid.h:14 (AoS input)."""
    return voxel_grid_downsamp_rvv_v2(points_aos, leaf_size, ctx)


# ---------------------------------------------------------------------------
# SOR
# ---------------------------------------------------------------------------
def sor_rvv(cloud, k: int, alpha: float, ctx: Optional[Context] = None, return_stats=False):
    """filters/statistical_outlier_removal.h:24 -> kept points (input order)."""
    ctx = ctx or default_context()
    x, y, z = _xyz(cloud)
    mem = _mem_of(x, y, z)
    _prep(ctx, mem)
    n = int(x.shape[0])
    dev = mem == MEM_DEVICE
    device = x.device if dev else None
    out = _empty((max(n, 1), 3), np.float32, dev, device)
    md = _empty((max(n, 1),), np.float32, dev, device)
    keep = _empty((max(n, 1),), np.uint8, dev, device)
    cnt = C.c_size_t(0)
    check(ctx.L.rvp_sor(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, int(k), float(alpha), mem,
                        _ptr(out), C.byref(cnt), _ptr(md), _ptr(keep)), ctx.h)
    v = int(cnt.value)
    if return_stats:
        return out[:v], md[:n], keep[:n]
    return out[:v]


def sor_sc(points_aos, k: int, alpha: float, ctx=None):
    """filters/statistical_outlier_removal.h:18 (AoS input)."""
    return sor_rvv(points_aos, k, alpha, ctx)


def sor_spatial_hash(cloud, hash_: SpatialHash, k: int, alpha: float,
                     search_radius: float = 0.5, return_stats=False):
    """filters/statistical_outlier_removal.h:35, over the hash's cloud."""
    ctx = hash_.ctx
    _prep(ctx, MEM_HOST)
    n = hash_.n
    out = np.empty((max(n, 1), 3), np.float32)
    md = np.empty(max(n, 1), np.float32)
    keep = np.empty(max(n, 1), np.uint8)
    cnt = C.c_size_t(0)
    check(ctx.L.rvp_sor_spatial_hash(hash_.h, int(k), float(alpha), float(search_radius),
                                     MEM_HOST, _ptr(out), C.byref(cnt), _ptr(md), _ptr(keep)),
          ctx.h)
    v = int(cnt.value)
    if return_stats:
        return out[:v], md[:n], keep[:n]
    return out[:v]


# ---------------------------------------------------------------------------
# Octree / PointerOctree
# ---------------------------------------------------------------------------
class Octree:
    """search/octree.h:20-48 on the GPU: radiusSearch returns every point
    with d2 <= radius^2 in the tree's depth-first leaf order (max_nn is
    ignored, as in the reference)."""

    KIND = 0

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.L = self.ctx.L
        h = C.c_void_p()
        check(self.L.rvp_octree_create(self.ctx.h, self.KIND, C.byref(h)), self.ctx.h)
        self.h = h
        self.n = 0
        self._params = [64, 8, 1e-4]

    def _set_params(self):
        check(self.L.rvp_octree_set_params(self.h, int(self._params[0]), int(self._params[1]),
                                           float(self._params[2])), self.ctx.h)

    def setMaxPointsPerLeaf(self, n: int) -> None:
        self._params[0] = n
        self._set_params()

    def setMaxDepth(self, d: int) -> None:
        self._params[1] = d
        self._set_params()

    def setBuildEpsilon(self, eps: float) -> None:
        self._params[2] = eps
        self._set_params()

    def setInputCloud(self, cloud) -> None:
        x, y, z = _xyz(cloud)
        mem = _mem_of(x, y, z)
        _prep(self.ctx, mem)
        n = int(x.shape[0])
        check(self.L.rvp_octree_set_input_cloud(self.h, _ptr(x), _ptr(y), _ptr(z), n, mem),
              self.ctx.h)
        self.n = n

    def build(self) -> None:
        _prep(self.ctx, MEM_HOST)
        check(self.L.rvp_octree_build(self.h), self.ctx.h)

    def order(self) -> np.ndarray:
        """The points in the tree's leaf order."""
        _prep(self.ctx, MEM_HOST)
        o = np.empty(max(self.n, 1), np.int32)
        check(self.L.rvp_octree_order(self.h, MEM_HOST, _ptr(o)), self.ctx.h)
        return o[:self.n]

    def radiusSearch(self, query: Sequence[float], radius: float, indices: Optional[list] = None,
                     dists: Optional[list] = None, max_nn: int = 0) -> int:
        q = np.asarray(query, dtype=np.float32).reshape(3)
        offs, idx, d2 = self.radiusSearchBatch(q[0:1], q[1:2], q[2:3], radius)
        if indices is not None:
            indices.clear()
            indices.extend(int(v) for v in idx)
        if dists is not None:
            dists.clear()
            dists.extend(float(v) for v in d2)
        return int(offs[-1])

    def radiusSearchBatch(self, qx, qy, qz, radius: float, capacity: Optional[int] = None):
        """All queries at once. Returns (offsets[nq+1], indices, dists) CSR."""
        qx, qy, qz = _f32(qx), _f32(qy), _f32(qz)
        mem = _mem_of(qx, qy, qz)
        _prep(self.ctx, mem)
        nq = int(qx.shape[0])
        dev = mem == MEM_DEVICE
        device = qx.device if dev else None
        offs = _empty((nq + 1,), np.int64, dev, device)
        cap = capacity if capacity is not None else 0
        total = C.c_size_t(0)
        while True:
            idx = _empty((max(cap, 1),), np.int32, dev, device)
            d2 = _empty((max(cap, 1),), np.float32, dev, device)
            st = self.L.rvp_octree_radius_search(self.h, _ptr(qx), _ptr(qy), _ptr(qz), nq,
                                                 float(radius), mem, _ptr(offs), _ptr(idx),
                                                 _ptr(d2), cap, C.byref(total))
            if st == _lib.RVP_ERR_CAPACITY:
                cap = int(total.value)
                continue
            check(st, self.ctx.h)
            t = int(total.value)
            return offs, idx[:t], d2[:t]

    def close(self):
        if getattr(self, "h", None):
            self.L.rvp_octree_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass


class PointerOctree(Octree):
    """search/pointer_octree.h:26-62 (root box [min - eps, max + eps])."""

    KIND = 1

    def radiusSearchScalar(self, query, radius, indices=None, dists=None) -> int:
        """pointer_octree.cpp:242-282: the same list as radiusSearch."""
        return self.radiusSearch(query, radius, indices, dists)


def _sor_tree(tree, k, alpha, search_radius, return_stats):
    ctx = tree.ctx
    _prep(ctx, MEM_HOST)
    n = tree.n
    out = np.empty((max(n, 1), 3), np.float32)
    md = np.empty(max(n, 1), np.float32)
    keep = np.empty(max(n, 1), np.uint8)
    cnt = C.c_size_t(0)
    check(ctx.L.rvp_sor_octree(tree.h, int(k), float(alpha), float(search_radius), MEM_HOST,
                               _ptr(out), C.byref(cnt), _ptr(md), _ptr(keep)), ctx.h)
    v = int(cnt.value)
    if return_stats:
        return out[:v], md[:n], keep[:n]
    return out[:v]


def sor_octree(cloud, tree: Octree, k: int, alpha: float, search_radius: float = 0.5,
               return_stats=False):
    """filters/statistical_outlier_removal.h:29 over the tree's cloud."""
    return _sor_tree(tree, k, alpha, search_radius, return_stats)


def sor_pointer_octree(cloud, tree: PointerOctree, k: int, alpha: float,
                       search_radius: float = 0.5, return_stats=False):
    """filters/statistical_outlier_removal.h:41 over the tree's cloud (the
    reference's nth_element step included)."""
    return _sor_tree(tree, k, alpha, search_radius, return_stats)


def normal_estimation_tree(cloud, tree: Octree, k: int, radius: float, vp_x: float = 0.0,
                           vp_y: float = 0.0, vp_z: float = 0.0, eigen_iters: int = 4):
    """features/normal_estimation.h:23/39 (Octree / PointerOctree overloads)
    over the tree's cloud. Returns (nx, ny, nz)."""
    ctx = tree.ctx
    _prep(ctx, MEM_HOST)
    n = tree.n
    nx, ny, nz = (np.empty(max(n, 1), np.float32) for _ in range(3))
    check(ctx.L.rvp_normals_octree(tree.h, float(radius), vp_x, vp_y, vp_z, int(eigen_iters),
                                   MEM_HOST, _ptr(nx), _ptr(ny), _ptr(nz)), ctx.h)
    return nx[:n], ny[:n], nz[:n]


def normal_estimation_self(cloud, k: int, radius: float, vp_x: float = 0.0, vp_y: float = 0.0,
                           vp_z: float = 0.0, eigen_iters: int = 4, ctx=None):
    """features/normal_estimation.h:47 (builds a PointerOctree itself)."""
    t = PointerOctree(ctx)
    try:
        t.setInputCloud(cloud)
        t.build()
        return normal_estimation_tree(cloud, t, k, radius, vp_x, vp_y, vp_z, eigen_iters)
    finally:
        t.close()


# ---------------------------------------------------------------------------
# normals
# ---------------------------------------------------------------------------
def normal_estimation_rvv(cloud, hash_: SpatialHash, k: int, radius: float, vp_x: float = 0.0,
                          vp_y: float = 0.0, vp_z: float = 0.0, eigen_iters: int = 4):
    """features/normal_estimation.h:31 (SpatialHash overload; k is unused by
    the reference too). Returns (nx, ny, nz) over the hash's cloud."""
    ctx = hash_.ctx
    _prep(ctx, MEM_HOST)
    n = hash_.n
    nx = np.empty(max(n, 1), np.float32)
    ny = np.empty(max(n, 1), np.float32)
    nz = np.empty(max(n, 1), np.float32)
    check(ctx.L.rvp_normals_radius(hash_.h, float(radius), vp_x, vp_y, vp_z, int(eigen_iters),
                                   MEM_HOST, _ptr(nx), _ptr(ny), _ptr(nz)), ctx.h)
    return nx[:n], ny[:n], nz[:n]


def normal_estimation_sc(points, k: int, radius: float = 0.0, vp_x: float = 0.0,
                         vp_y: float = 0.0, vp_z: float = 0.0, eigen_iters: int = 4, ctx=None):
    """features/normal_estimation.h:15: k+1 nearest including self."""
    ctx = ctx or default_context()
    x, y, z = _xyz(points)
    mem = _mem_of(x, y, z)
    _prep(ctx, mem)
    n = int(x.shape[0])
    dev = mem == MEM_DEVICE
    device = x.device if dev else None
    nx = _empty((max(n, 1),), np.float32, dev, device)
    ny = _empty((max(n, 1),), np.float32, dev, device)
    nz = _empty((max(n, 1),), np.float32, dev, device)
    check(ctx.L.rvp_normals_knn(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, int(k), vp_x, vp_y, vp_z,
                                int(eigen_iters), mem, _ptr(nx), _ptr(ny), _ptr(nz)), ctx.h)
    return nx[:n], ny[:n], nz[:n]


def normal_estimation_precise(points, k: int, vp=(0.0, 0.0, 0.0), cond_fp64: float = 1e6,
                              ctx=None):
    """Precision mode: shifted, compensated FP32 covariance of the k+1
    nearest; FP64 eigen-solve only where cond > cond_fp64. Returns
    (normals[n,3], cond[n], used_fp64[n])."""
    ctx = ctx or default_context()
    x, y, z = _xyz(points)
    mem = _mem_of(x, y, z)
    _prep(ctx, mem)
    n = int(x.shape[0])
    dev = mem == MEM_DEVICE
    device = x.device if dev else None
    nx = _empty((max(n, 1),), np.float32, dev, device)
    ny = _empty((max(n, 1),), np.float32, dev, device)
    nz = _empty((max(n, 1),), np.float32, dev, device)
    cond = _empty((max(n, 1),), np.float32, dev, device)
    used = _empty((max(n, 1),), np.uint8, dev, device)
    check(ctx.L.rvp_normals_knn_precise(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, int(k), vp[0], vp[1],
                                        vp[2], float(cond_fp64), mem, _ptr(nx), _ptr(ny),
                                        _ptr(nz), _ptr(cond), _ptr(used)), ctx.h)
    if dev:
        return torch.stack([nx[:n], ny[:n], nz[:n]], 1), cond[:n], used[:n]
    return np.stack([nx[:n], ny[:n], nz[:n]], 1), cond[:n], used[:n]


# ---------------------------------------------------------------------------
# RANSAC
# ---------------------------------------------------------------------------
def ransac_plane_rvv(cloud, dist_thresh: float, max_iters: int, collinear_thresh: float = 1e-6,
                     probability: float = 0.99, rand_stream=None, return_counts: bool = False,
                     ctx: Optional[Context] = None):
    """segmentation/ransac_plane.h:19 -> (best_count, model[4]).

    rand_stream: the 3*max_iters raw rand() values the reference draws after
    srand(0); None lets the library draw them from libc (and leave libc's
    generator where the reference leaves it). return_counts adds the
    per-hypothesis inlier counts (-1 repeated index, -2 collinear) and the
    number of iterations the reference executes."""
    ctx = ctx or default_context()
    x, y, z = _xyz(cloud)
    mem = _mem_of(x, y, z)
    _prep(ctx, mem)
    n = int(x.shape[0])
    model = np.zeros(4, np.float32)
    best = C.c_int(0)
    iters = C.c_int(0)
    rs = None
    if rand_stream is not None:
        rs = np.ascontiguousarray(np.asarray(rand_stream)[: 3 * max_iters], dtype=np.int32)
        if mem == MEM_DEVICE:
            rs = torch.from_numpy(rs).to(x.device)
    counts = None
    if return_counts:
        counts = _empty((max(max_iters, 1),), np.int32, mem == MEM_DEVICE,
                        x.device if mem == MEM_DEVICE else None)
    check(ctx.L.rvp_ransac_plane(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, float(dist_thresh),
                                 int(max_iters), float(collinear_thresh), float(probability),
                                 _ptr(rs), mem, model.ctypes.data_as(C.c_void_p), C.byref(best),
                                 C.byref(iters), _ptr(counts)), ctx.h)
    if return_counts:
        return int(best.value), model, counts[:max_iters], int(iters.value)
    return int(best.value), model


def ransac_plane_sc(points_aos, dist_thresh, max_iters, collinear_thresh=1e-6, probability=0.99,
                    ctx=None):
    """segmentation/ransac_plane.h:11 (AoS input)."""
    return ransac_plane_rvv(points_aos, dist_thresh, max_iters, collinear_thresh, probability,
                            ctx=ctx)


def extract_plane_inliers_outliers_rvv(cloud, model, dist_thresh: float, ctx=None):
    """segmentation/ransac_plane.h:41 -> (inliers (m,3), outliers (n-m,3))."""
    ctx = ctx or default_context()
    x, y, z = _xyz(cloud)
    _prep(ctx, MEM_HOST)
    n = int(x.shape[0])
    m = np.ascontiguousarray(model, dtype=np.float32)
    ins = np.empty((max(n, 1), 3), np.float32)
    outs = np.empty((max(n, 1), 3), np.float32)
    ni, no = C.c_size_t(0), C.c_size_t(0)
    check(ctx.L.rvp_extract_plane(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, _ptr(m),
                                  float(dist_thresh), MEM_HOST, _ptr(ins), _ptr(outs),
                                  C.byref(ni), C.byref(no)), ctx.h)
    return ins[: ni.value], outs[: no.value]


def extract_plane_inliers_rvv(cloud, model, dist_thresh: float, ctx=None):
    """segmentation/ransac_plane.h:27."""
    return extract_plane_inliers_outliers_rvv(cloud, model, dist_thresh, ctx)[0]


def extract_plane_outliers_rvv(cloud, model, dist_thresh: float, ctx=None):
    """segmentation/ransac_plane.h:34."""
    return extract_plane_inliers_outliers_rvv(cloud, model, dist_thresh, ctx)[1]


# ---------------------------------------------------------------------------
# batched frames
# ---------------------------------------------------------------------------
def euclidean_clusters(cloud, tolerance: float, min_size: int = 1,
                       max_size: int = 2**31 - 1, ctx: Optional[Context] = None):
    """EuclideanClustering::extract (segmentation/euclidean_clustering.cpp
    :113-189): list of sorted index arrays, by lowest index."""
    ctx = ctx or default_context()
    x, y, z = _xyz(cloud)
    mem = _mem_of(x, y, z)
    _prep(ctx, mem)
    n = int(x.shape[0])
    dev = mem == MEM_DEVICE
    device = x.device if dev else None
    offs = _empty((n + 1,), np.int64, dev, device)
    idx = _empty((max(n, 1),), np.int32, dev, device)
    k = C.c_size_t(0)
    check(ctx.L.rvp_euclidean_clusters(ctx.h, _ptr(x), _ptr(y), _ptr(z), n, float(tolerance),
                                       int(min_size), int(max_size), mem, _ptr(offs), _ptr(idx),
                                       C.byref(k)), ctx.h)
    k = int(k.value)
    if dev:
        offs, idx = offs.cpu().numpy(), idx.cpu().numpy()
    return [idx[offs[i]:offs[i + 1]].copy() for i in range(k)]


def load_pcd(path: str, device: bool = False, ctx: Optional[Context] = None):
    """io/simple_pcd_loader.h loadPCD: (x, y, z) float32 arrays (CUDA tensors
    with device=True)."""
    ctx = ctx or default_context()
    n = C.c_size_t(0)
    st = ctx.L.rvp_pcd_load(ctx.h, path.encode(), MEM_HOST, None, None, None, 0, C.byref(n))
    if st not in (_lib.RVP_OK, _lib.RVP_ERR_CAPACITY):
        check(st, ctx.h)
    cap = int(n.value)
    mem = MEM_DEVICE if device else MEM_HOST
    _prep(ctx, mem)
    x, y, z = (_empty((max(cap, 1),), np.float32, device, torch.device("cuda", ctx.device)
                      if device else None) for _ in range(3))
    check(ctx.L.rvp_pcd_load(ctx.h, path.encode(), mem, _ptr(x), _ptr(y), _ptr(z), max(cap, 1),
                             C.byref(n)), ctx.h)
    k = int(n.value)
    return x[:k], y[:k], z[:k]


class EuclideanClustering:
    """segmentation/euclidean_clustering.h:17-70 (no neighbour searcher)."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx
        self.cloud = None
        self.tolerance = 0.05
        self.min_size = 1
        self.max_size = 2**31 - 1

    def setInputCloud(self, cloud):
        self.cloud = cloud

    def setClusterTolerance(self, tolerance: float):
        self.tolerance = float(tolerance)

    def setMinClusterSize(self, n: int):
        self.min_size = int(n)

    def setMaxClusterSize(self, n: int):
        self.max_size = int(n)

    def extract(self):
        if self.cloud is None:
            return []
        return euclidean_clusters(self.cloud, self.tolerance, self.min_size, self.max_size,
                                  ctx=self.ctx)


GRID_LEVELS = 5  # RVP_GRID_LEVELS: neighbour-grid cells of c, 2c, 4c, 8c, 16c
# kNN kernels timed per search stage: the per-lane kernels on cells of c, 4c
# and 16c, and the cooperative pass
TIMED_KNN = ("knn_l0", "knn_l1", "knn_l2", "knn_coop")


class Pipeline:
    """voxel -> SOR -> normals(k+1 NN) -> RANSAC over many frames at once."""

    def __init__(self, max_points: int, max_frames: int, leaf_size=0.1, sor_k=16, sor_alpha=1.0,
                 normal_k=16, eigen_iters=4, viewpoint=(0.0, 0.0, 0.0), ransac_thresh=0.05,
                 ransac_iters=1000, ransac_collinear=1e-6, ransac_prob=0.99, cell_size=0.0,
                 block_threads=0, queries_per_warp=0, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.L = self.ctx.L
        cfg = _lib.PipelineConfig(leaf_size, sor_k, sor_alpha, normal_k, eigen_iters,
                                  viewpoint[0], viewpoint[1], viewpoint[2], ransac_thresh,
                                  ransac_iters, ransac_collinear, ransac_prob, cell_size,
                                  block_threads, queries_per_warp)
        self.cfg = cfg
        h = C.c_void_p()
        check(self.L.rvp_pipeline_create(self.ctx.h, C.byref(cfg), int(max_points),
                                         int(max_frames), C.byref(h)), self.ctx.h)
        self.h = h
        self.max_points = max_points
        self.max_frames = max_frames
        self.last_frames = 0

    def run_device(self, x, y, z, offsets_dev, n_frames: int, n_points: int) -> None:
        """x, y, z, offsets: CUDA tensors; results stay on the device."""
        self.ctx.use_torch_stream()
        self.last_frames = int(n_frames)
        check(self.L.rvp_pipeline_run_device(self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(offsets_dev),
                                             int(n_frames), int(n_points)), self.ctx.h)

    def capture(self, x, y, z, offsets_dev, n_frames: int, n_points: int) -> int:
        """Record one run over these device tensors as a CUDA graph; returns
        the kernel launches one replay makes. Refill the same tensors and
        call replay() for each new batch."""
        self.ctx.use_torch_stream()
        self.last_frames = int(n_frames)
        k = C.c_uint64(0)
        check(self.L.rvp_pipeline_capture(self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(offsets_dev),
                                          int(n_frames), int(n_points), C.byref(k)), self.ctx.h)
        self._graph_inputs = (x, y, z, offsets_dev)  # the graph reads these buffers
        return int(k.value)

    def replay(self) -> None:
        self.ctx.use_torch_stream()
        check(self.L.rvp_pipeline_replay(self.h), self.ctx.h)

    STAGES = ("voxel", "grid_build", "sor_knn", "sor_filter", "normals_knn", "normals",
              "ransac")

    def set_tuning(self, cell_size: float, block_threads: int = 0,
                   queries_per_warp: int = 0) -> None:
        check(self.L.rvp_pipeline_set_tuning(self.h, float(cell_size), int(block_threads),
                                             int(queries_per_warp)), self.ctx.h)
        self.cfg.cell_size = cell_size
        self.cfg.block_threads = block_threads
        self.cfg.queries_per_warp = queries_per_warp

    def set_lane_levels(self, levels: int) -> None:
        """Chain levels (cells of c, 4c, 16c) of the one-query-per-lane kNN
        kernels, 1 to 3 (0: all)."""
        check(self.L.rvp_pipeline_set_lane_levels(self.h, int(levels)), self.ctx.h)
        self.lane_levels = int(levels)

    def set_search_radius_factor(self, rfac: float) -> None:
        check(self.L.rvp_pipeline_set_search_radius_factor(self.h, float(rfac)), self.ctx.h)

    def frame_offsets(self, n_frames: Optional[int] = None):
        """(voxel_offsets, sor_offsets) of the last run, as host int64 arrays."""
        nf = n_frames if n_frames is not None else self.last_frames
        vo = np.empty(nf + 1, np.int64)
        so = np.empty(nf + 1, np.int64)
        check(self.L.rvp_pipeline_frame_offsets(self.h, _ptr(vo), _ptr(so)), self.ctx.h)
        return vo, so

    def fit_tables(self) -> None:
        check(self.L.rvp_pipeline_fit_tables(self.h), self.ctx.h)

    def check(self) -> None:
        check(self.L.rvp_pipeline_check(self.h), self.ctx.h)

    # warp kernel: ring at level 0 / tight window / ring at level 1 / ring at
    # level 2 / whole frame; tile kernel: certified at level 0 / 1 / 2; plus
    # "tau_window": the per-thread tight window of a handed-on bound
    PATHS = ("warp_ring0", "warp_tight", "warp_ring1", "warp_ring2", "warp_whole_frame",
             "tile_l0", "tile_l1", "tile_l2")

    def knn_stats(self, enable: bool = True) -> dict:
        out = np.zeros(20, np.uint32)
        check(self.L.rvp_pipeline_knn_stats(self.h, int(enable), _ptr(out)), self.ctx.h)
        return {"sor": dict(zip(self.PATHS, map(int, out[:8])), tau_window=int(out[16])),
                "normals": dict(zip(self.PATHS, map(int, out[8:16])), tau_window=int(out[17]))}

    def knn_routed(self) -> int:
        """SOR kNN queries the last run's cooperative pass took (0 without it)."""
        return self.knn_counts()[0]

    def knn_counts(self) -> tuple:
        """SOR kNN queries of the last run's cooperative pass and of the
        adaptive per-thread kernel after it (zeros without the cooperative
        mode)."""
        out = np.zeros(2, np.uint64)
        check(self.L.rvp_pipeline_knn_routed(self.h, _ptr(out)), self.ctx.h)
        return int(out[0]), int(out[1])

    def set_timing(self, max_runs: int) -> None:
        check(self.L.rvp_pipeline_set_timing(self.h, int(max_runs)), self.ctx.h)

    GRID_LEVELS = GRID_LEVELS
    LEVEL_KERNELS = tuple(f"{st}_{k}" for st in ("sor", "normals") for k in TIMED_KNN)

    def stage_times(self, levels: bool = False) -> dict:
        """Mean ms per stage over the runs recorded since set_timing; with
        levels=True also the kNN kernel of each grid level."""
        n = len(self.STAGES) + (len(self.LEVEL_KERNELS) if levels else 0)
        ms = (C.c_float * n)()
        runs = C.c_int(0)
        check(self.L.rvp_pipeline_stage_times(self.h, ms, n, C.byref(runs)), self.ctx.h)
        names = self.STAGES + (self.LEVEL_KERNELS if levels else ())
        return {"runs": runs.value, **{s: float(ms[i]) for i, s in enumerate(names)}}

    def outputs(self) -> _lib.PipelineOutputs:
        o = _lib.PipelineOutputs()
        check(self.L.rvp_pipeline_outputs_get(self.h, C.byref(o)), self.ctx.h)
        return o

    def run_host(self, batch):
        """batch: datasets.Batch (host). Returns per-frame results as numpy."""
        self.ctx.set_stream(0)
        x, y, z = _f32(batch.x), _f32(batch.y), _f32(batch.z)
        offs = np.ascontiguousarray(batch.offsets, dtype=np.int64)
        nf = int(offs.shape[0] - 1)
        self.last_frames = nf
        n = int(offs[-1])
        vox = np.empty((max(n, 1), 3), np.float32)
        vo = np.empty(nf + 1, np.int64)
        sor = np.empty((max(n, 1), 3), np.float32)
        so = np.empty(nf + 1, np.int64)
        nx = np.empty(max(n, 1), np.float32)
        ny = np.empty(max(n, 1), np.float32)
        nz = np.empty(max(n, 1), np.float32)
        model = np.empty((nf, 4), np.float32)
        cnt = np.empty(nf, np.int32)
        check(self.L.rvp_pipeline_run_host(self.h, _ptr(x), _ptr(y), _ptr(z), _ptr(offs), nf,
                                           _ptr(vox), _ptr(vo), _ptr(sor), _ptr(so), _ptr(nx),
                                           _ptr(ny), _ptr(nz), _ptr(model), _ptr(cnt)),
              self.ctx.h)
        nv, ns = int(vo[-1]), int(so[-1])
        return dict(voxel=vox[:nv], voxel_offsets=vo, sor=sor[:ns], sor_offsets=so,
                    normals=np.stack([nx[:ns], ny[:ns], nz[:ns]], 1), ransac_model=model,
                    ransac_count=cnt)

    def run_host_batches(self, batches):
        """Several host batches in a row (rvp_pipeline_run_host_batches: the
        next batch goes up and the previous results come down while a batch
        runs). Returns one result dict per batch, as run_host."""
        self.ctx.set_stream(0)
        nb = len(batches)
        arrs = {k: [] for k in ("x", "y", "z", "o", "vox", "vo", "sor", "so", "nx", "ny", "nz",
                                "m", "c")}
        nfs = []
        for b in batches:
            x, y, z = _f32(b.x), _f32(b.y), _f32(b.z)
            offs = np.ascontiguousarray(b.offsets, dtype=np.int64)
            nf = int(offs.shape[0] - 1)
            n = int(offs[-1])
            nfs.append(nf)
            for k, v in (("x", x), ("y", y), ("z", z), ("o", offs),
                         ("vox", np.empty((max(n, 1), 3), np.float32)),
                         ("vo", np.empty(nf + 1, np.int64)),
                         ("sor", np.empty((max(n, 1), 3), np.float32)),
                         ("so", np.empty(nf + 1, np.int64)),
                         ("nx", np.empty(max(n, 1), np.float32)),
                         ("ny", np.empty(max(n, 1), np.float32)),
                         ("nz", np.empty(max(n, 1), np.float32)),
                         ("m", np.empty((nf, 4), np.float32)), ("c", np.empty(nf, np.int32))):
                arrs[k].append(v)
        ptrs = {k: (C.c_void_p * nb)(*[a.ctypes.data for a in v]) for k, v in arrs.items()}
        nfa = (C.c_int * nb)(*nfs)
        self.last_frames = nfs[-1] if nfs else 0
        check(self.L.rvp_pipeline_run_host_batches(
            self.h, nb, ptrs["x"], ptrs["y"], ptrs["z"], ptrs["o"], nfa, ptrs["vox"], ptrs["vo"],
            ptrs["sor"], ptrs["so"], ptrs["nx"], ptrs["ny"], ptrs["nz"], ptrs["m"], ptrs["c"]),
            self.ctx.h)
        out = []
        for i in range(nb):
            nv, ns = int(arrs["vo"][i][-1]), int(arrs["so"][i][-1])
            out.append(dict(voxel=arrs["vox"][i][:nv], voxel_offsets=arrs["vo"][i],
                            sor=arrs["sor"][i][:ns], sor_offsets=arrs["so"][i],
                            normals=np.stack([arrs["nx"][i][:ns], arrs["ny"][i][:ns],
                                              arrs["nz"][i][:ns]], 1),
                            ransac_model=arrs["m"][i], ransac_count=arrs["c"][i]))
        return out

    def results(self, max_points: int | None = None) -> dict:
        """Per-frame results of the last run, copied to numpy."""
        nf = int(self.last_frames)
        n = int(max_points if max_points is not None else self.max_points)
        vox = np.empty((max(n, 1), 3), np.float32)
        vo = np.empty(nf + 1, np.int64)
        sor = np.empty((max(n, 1), 3), np.float32)
        so = np.empty(nf + 1, np.int64)
        nx = np.empty(max(n, 1), np.float32)
        ny = np.empty(max(n, 1), np.float32)
        nz = np.empty(max(n, 1), np.float32)
        model = np.empty((nf, 4), np.float32)
        cnt = np.empty(nf, np.int32)
        check(self.L.rvp_pipeline_copy_outputs(self.h, _ptr(vox), _ptr(vo), _ptr(sor), _ptr(so),
                                               _ptr(nx), _ptr(ny), _ptr(nz), _ptr(model),
                                               _ptr(cnt)), self.ctx.h)
        nv, ns = int(vo[-1]), int(so[-1])
        return dict(voxel=vox[:nv], voxel_offsets=vo, sor=sor[:ns], sor_offsets=so,
                    normals=np.stack([nx[:ns], ny[:ns], nz[:ns]], 1), ransac_model=model,
                    ransac_count=cnt)

    def close(self):
        if getattr(self, "h", None):
            self.L.rvp_pipeline_destroy(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass
