"""ctypes front-end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Two libraries back it:

* ``restatement`` -- oracle/_build/librvp_oracle.so, the plain-C restatement
  of the reference's scalar path (oracle/rvp_oracle.c);
* ``reference``   -- oracle/_ref/librvpoint_ref.so, the reference's own
  sources compiled here by oracle/Makefile (present only where the reference
  checkout was available at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the library under rvpoint_b200/ never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "librvp_oracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "librvpoint_ref.so")

_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int)
_lp = C.POINTER(C.c_longlong)
_dp = C.POINTER(C.c_double)
_sz = C.c_size_t


# where the reference checkout is looked for when RVP_REFERENCE is not set
_REFERENCE_CHECKOUT = "/root/reference"


def reference_checkout():
    """The reference checkout to compile oracle/_ref from (None if absent)."""
    ref = os.environ.get("RVP_REFERENCE", _REFERENCE_CHECKOUT)
    return ref if os.path.exists(os.path.join(ref, "src", "core", "point_types.h")) else None


def build(quiet: bool = True) -> None:
    """Compile the restatement (and the reference, when its sources exist)."""
    cmd = ["make", "-C", HERE]
    ref = reference_checkout()
    if ref:
        cmd.append(f"REF={ref}")
    subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def _ptr(a, t):
    return a.ctypes.data_as(t) if a is not None else None


_libs: dict = {}


def _lib(path):
    if path not in _libs:
        if not os.path.exists(path):
            if path == RESTATEMENT_SO:
                build()
            else:
                raise FileNotFoundError(path)
        _libs[path] = C.CDLL(path)
    return _libs[path]


def _clusters(fn, c, tolerance, min_size, max_size):
    x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
    n = x.shape[0]
    offs = np.zeros(n + 1, np.int64)
    idx = np.zeros(max(n, 1), np.int32)
    k = fn(xp, yp, zp, n, tolerance, int(min_size), int(max_size), _ptr(offs, _lp),
           _ptr(idx, _ip))
    return [idx[offs[i]:offs[i + 1]].copy() for i in range(k)]


def reference_available() -> bool:
    return os.path.exists(REFERENCE_SO)


# --------------------------------------------------------------------------
# restatement (plain C)
# --------------------------------------------------------------------------
class Restatement:
    def __init__(self):
        L = self.L = _lib(RESTATEMENT_SO)
        L.rvo_hash_radius_search.restype = C.c_longlong
        L.rvo_hash_radius_search.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int64, C.c_int64,
                                             _fp, _fp, _fp, _sz, C.c_float, C.c_int, _lp, _ip,
                                             _fp, C.c_longlong]
        L.rvo_voxel_grid.restype = _sz
        L.rvo_voxel_grid.argtypes = [_fp, _fp, _fp, _sz, C.c_float, _fp, _ip]
        L.rvo_sor_exact.restype = _sz
        L.rvo_sor_exact.argtypes = [_fp, _fp, _fp, _sz, C.c_int, C.c_float, _fp, _fp,
                                    C.POINTER(C.c_ubyte)]
        L.rvo_sor_radius.restype = _sz
        L.rvo_sor_radius.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_float,
                                     C.c_float, _fp, _fp, C.POINTER(C.c_ubyte)]
        L.rvo_normals_radius.restype = None
        L.rvo_normals_radius.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_float, C.c_float,
                                         C.c_float, C.c_float, C.c_int, C.c_int, _fp, _fp, _fp]
        L.rvo_normals_knn.restype = None
        L.rvo_normals_knn.argtypes = [_fp, _fp, _fp, _sz, C.c_int, C.c_float, C.c_float,
                                      C.c_float, C.c_int, C.c_int, _fp, _fp, _fp]
        L.rvo_ransac_plane.restype = C.c_int
        L.rvo_ransac_plane.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_float,
                                       C.c_float, _ip, _fp, _ip, _fp, _ip]
        L.rvo_extract_plane.restype = None
        L.rvo_extract_plane.argtypes = [_fp, _fp, _fp, _sz, _fp, C.c_float, _fp, _fp,
                                        C.POINTER(_sz), C.POINTER(_sz)]
        L.rvo_euclidean_clusters.restype = C.c_long
        L.rvo_euclidean_clusters.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_int,
                                             _lp, _ip]
        L.rvo_octree_order.restype = None
        L.rvo_octree_order.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int,
                                       C.c_float, _ip]
        L.rvo_octree_radius_search.restype = C.c_longlong
        L.rvo_octree_radius_search.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int,
                                               C.c_float, _fp, _fp, _fp, _sz, C.c_float, _lp,
                                               _ip, _fp, C.c_longlong]
        L.rvo_nth_element.restype = C.c_int
        L.rvo_nth_element.argtypes = [_fp, _sz, _sz]
        L.rvo_sor_octree.restype = _sz
        L.rvo_sor_octree.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int, C.c_float,
                                     C.c_int, C.c_float, C.c_float, _fp, _fp,
                                     C.POINTER(C.c_ubyte)]
        L.rvo_normals_octree.restype = None
        L.rvo_normals_octree.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int,
                                         C.c_float, C.c_float, C.c_float, C.c_float,
                                         C.c_float, C.c_int, _fp, _fp, _fp]
        L.rvo_knn_lists.restype = None
        L.rvo_knn_lists.argtypes = [_fp, _fp, _fp, _sz, C.c_int, _ip, _fp]
        L.rvo_normals_knn_exact_f64.restype = None
        L.rvo_normals_knn_exact_f64.argtypes = [_fp, _fp, _fp, _sz, _ip, C.c_int, C.c_float,
                                                C.c_float, C.c_float, _dp, _dp, _dp, _dp]

    def radius_search(self, c, cell, radius, max_nn=0, queries=None, p1=73856093,
                      p2=19349663, cap=None):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        q = queries if queries is not None else c
        qx, qxp = _f(q.x); qy, qyp = _f(q.y); qz, qzp = _f(q.z)
        nq = qx.shape[0]
        offs = np.zeros(nq + 1, np.int64)
        cap = cap if cap is not None else max(1, nq * (max_nn if max_nn > 0 else 64))
        while True:
            idx = np.zeros(cap, np.int32); d2 = np.zeros(cap, np.float32)
            tot = self.L.rvo_hash_radius_search(xp, yp, zp, x.shape[0], cell, p1, p2, qxp, qyp,
                                                qzp, nq, radius, max_nn, _ptr(offs, _lp),
                                                _ptr(idx, _ip), _ptr(d2, _fp), cap)
            if tot >= 0:
                return offs, idx[:tot], d2[:tot]
            cap = int(offs[-1])

    def voxel_grid(self, c, leaf):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        out = np.zeros((max(n, 1), 3), np.float32); keys = np.zeros((max(n, 1), 3), np.int32)
        v = self.L.rvo_voxel_grid(xp, yp, zp, n, leaf, _ptr(out, _fp), _ptr(keys, _ip))
        return out[:v].copy(), keys[:v].copy()

    def sor_exact(self, c, k, alpha):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        out = np.zeros((max(n, 1), 3), np.float32); md = np.zeros(max(n, 1), np.float32)
        keep = np.zeros(max(n, 1), np.uint8)
        v = self.L.rvo_sor_exact(xp, yp, zp, n, k, alpha, _ptr(out, _fp), _ptr(md, _fp),
                                 keep.ctypes.data_as(C.POINTER(C.c_ubyte)))
        return out[:v].copy(), md[:n], keep[:n].astype(bool)

    def sor_radius(self, c, cell, k, alpha, search_radius):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        out = np.zeros((max(n, 1), 3), np.float32); md = np.zeros(max(n, 1), np.float32)
        keep = np.zeros(max(n, 1), np.uint8)
        v = self.L.rvo_sor_radius(xp, yp, zp, n, cell, k, alpha, search_radius, _ptr(out, _fp),
                                  _ptr(md, _fp), keep.ctypes.data_as(C.POINTER(C.c_ubyte)))
        return out[:v].copy(), md[:n], keep[:n].astype(bool)

    def normals_radius(self, c, cell, radius, vp=(0, 0, 0), iters=4, f64=False):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        nx = np.zeros(n, np.float32); ny = np.zeros(n, np.float32); nz = np.zeros(n, np.float32)
        self.L.rvo_normals_radius(xp, yp, zp, n, cell, radius, vp[0], vp[1], vp[2], iters,
                                  int(f64), _ptr(nx, _fp), _ptr(ny, _fp), _ptr(nz, _fp))
        return np.stack([nx, ny, nz], 1)

    def normals_knn(self, c, k, vp=(0, 0, 0), iters=4, f64=False):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        nx = np.zeros(n, np.float32); ny = np.zeros(n, np.float32); nz = np.zeros(n, np.float32)
        self.L.rvo_normals_knn(xp, yp, zp, n, k, vp[0], vp[1], vp[2], iters, int(f64),
                               _ptr(nx, _fp), _ptr(ny, _fp), _ptr(nz, _fp))
        return np.stack([nx, ny, nz], 1)

    def ransac_plane(self, c, thresh, max_iters, rand_stream, collinear=1e-6, prob=0.99):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        rs = np.ascontiguousarray(rand_stream[: 3 * max_iters], dtype=np.int32)
        model = np.zeros(4, np.float32); counts = np.zeros(max(max_iters, 1), np.int32)
        models = np.zeros((max(max_iters, 1), 4), np.float32); it = C.c_int(0)
        best = self.L.rvo_ransac_plane(xp, yp, zp, x.shape[0], thresh, max_iters, collinear,
                                       prob, _ptr(rs, _ip), _ptr(model, _fp), _ptr(counts, _ip),
                                       _ptr(models, _fp), C.byref(it))
        return best, model, counts[:max_iters], models[:max_iters], it.value

    def extract_plane(self, c, model, thresh):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        m = np.ascontiguousarray(model, np.float32)
        a = np.zeros((max(n, 1), 3), np.float32); b = np.zeros((max(n, 1), 3), np.float32)
        ni, no = _sz(0), _sz(0)
        self.L.rvo_extract_plane(xp, yp, zp, n, _ptr(m, _fp), thresh, _ptr(a, _fp),
                                 _ptr(b, _fp), C.byref(ni), C.byref(no))
        return a[: ni.value].copy(), b[: no.value].copy()

    def euclidean_clusters(self, c, tolerance, min_size=1, max_size=2**31 - 1):
        """List of sorted index arrays, in the reference's cluster order."""
        return _clusters(self.L.rvo_euclidean_clusters, c, tolerance, min_size, max_size)

    # Octree (kind 0) / PointerOctree (kind 1); tree = (cap, max_depth, eps)
    def octree_order(self, kind, c, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        order = np.zeros(max(x.shape[0], 1), np.int32)
        self.L.rvo_octree_order(kind, xp, yp, zp, x.shape[0], tree[0], tree[1], tree[2],
                                _ptr(order, _ip))
        return order[:x.shape[0]]

    def octree_radius(self, kind, c, radius, queries=None, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        q = queries if queries is not None else c
        qx, qxp = _f(q.x); qy, qyp = _f(q.y); qz, qzp = _f(q.z)
        nq = qx.shape[0]
        offs = np.zeros(nq + 1, np.int64)
        cap = 1 << 16
        while True:
            idx = np.zeros(cap, np.int32); d2 = np.zeros(cap, np.float32)
            t = self.L.rvo_octree_radius_search(kind, xp, yp, zp, x.shape[0], tree[0], tree[1],
                                                tree[2], qxp, qyp, qzp, nq, radius,
                                                _ptr(offs, _lp), _ptr(idx, _ip), _ptr(d2, _fp),
                                                cap)
            if t >= 0:
                return offs, idx[:t].copy(), d2[:t].copy()
            cap = int(offs[-1]) + 1

    def nth_element(self, a, nth):
        a = np.ascontiguousarray(a, np.float32).copy()
        heap = self.L.rvo_nth_element(_ptr(a, _fp), a.shape[0], nth)
        return a, bool(heap)

    def sor_octree(self, kind, c, k, alpha, search_radius, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        out = np.zeros((max(n, 1), 3), np.float32)
        md = np.zeros(max(n, 1), np.float32); keep = np.zeros(max(n, 1), np.uint8)
        m = self.L.rvo_sor_octree(kind, xp, yp, zp, n, tree[0], tree[1], tree[2], k, alpha,
                                  search_radius, _ptr(out, _fp), _ptr(md, _fp),
                                  _ptr(keep, C.POINTER(C.c_ubyte)))
        return out[:m].copy(), md[:n], keep[:n].astype(bool)

    def normals_octree(self, kind, c, radius, vp=(0, 0, 0), iters=4, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        nx, ny, nz = (np.zeros(max(n, 1), np.float32) for _ in range(3))
        self.L.rvo_normals_octree(kind, xp, yp, zp, n, tree[0], tree[1], tree[2], radius,
                                  vp[0], vp[1], vp[2], iters, _ptr(nx, _fp), _ptr(ny, _fp),
                                  _ptr(nz, _fp))
        return np.stack([nx[:n], ny[:n], nz[:n]], 1)

    def knn_lists(self, c, kk):
        """(n, kk) indices and squared distances of every point's kk nearest
        (self included), ordered by (d2, index); brute force over threads."""
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        idx = np.zeros((max(n, 1), kk), np.int32); d2 = np.zeros((max(n, 1), kk), np.float32)
        self.L.rvo_knn_lists(xp, yp, zp, n, kk, _ptr(idx, _ip), _ptr(d2, _fp))
        return idx[:n], d2[:n]

    def normals_exact_f64(self, c, nbr_idx, vp=(0, 0, 0)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        nbr = np.ascontiguousarray(nbr_idx, np.int32)
        n, kk = nbr.shape
        out = [np.zeros(n, np.float64) for _ in range(4)]
        self.L.rvo_normals_knn_exact_f64(xp, yp, zp, n, _ptr(nbr, _ip), kk, vp[0], vp[1], vp[2],
                                         *[_ptr(o, _dp) for o in out])
        return np.stack(out[:3], 1), out[3]


# --------------------------------------------------------------------------
# the reference's own code (built from its sources)
# --------------------------------------------------------------------------
class Reference:
    def __init__(self):
        L = self.L = _lib(REFERENCE_SO)
        L.ref_hash_radius_search.restype = C.c_longlong
        L.ref_hash_radius_search.argtypes = [_fp, _fp, _fp, _sz, C.c_float, _fp, _fp, _fp, _sz,
                                             C.c_float, C.c_int, _lp, _ip, _fp, C.c_longlong]
        L.ref_voxel_grid.restype = _sz
        L.ref_voxel_grid.argtypes = [_fp, _fp, _fp, _sz, C.c_float, _fp]
        L.ref_sor_rvv.restype = _sz
        L.ref_sor_rvv.argtypes = [_fp, _fp, _fp, _sz, C.c_int, C.c_float, _fp]
        L.ref_sor_spatial_hash.restype = _sz
        L.ref_sor_spatial_hash.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_float,
                                           C.c_float, _fp]
        L.ref_normals_hash.restype = None
        L.ref_normals_hash.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_float,
                                       C.c_float, C.c_float, C.c_float, C.c_int, _fp, _fp, _fp]
        L.ref_normals_sc.restype = None
        L.ref_normals_sc.argtypes = [_fp, _sz, C.c_int, C.c_float, C.c_float, C.c_float,
                                     C.c_float, C.c_int, _fp, _fp, _fp]
        L.ref_ransac_plane.restype = C.c_int
        L.ref_ransac_plane.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_float,
                                       C.c_float, _fp]
        L.ref_extract_plane.restype = None
        L.ref_extract_plane.argtypes = [_fp, _fp, _fp, _sz, _fp, C.c_float, _fp, _fp,
                                        C.POINTER(_sz), C.POINTER(_sz)]
        L.ref_count_plane_inliers.restype = _sz
        L.ref_count_plane_inliers.argtypes = [_fp, _fp, _fp, _sz, _fp, C.c_float, _fp]
        L.ref_load_pcd.restype = C.c_long
        L.ref_load_pcd.argtypes = [C.c_char_p, _fp, _sz]
        L.ref_save_pcd.restype = None
        L.ref_save_pcd.argtypes = [C.c_char_p, _fp, _sz, C.c_int]
        L.ref_save_pcd_rgb.restype = None
        L.ref_save_pcd_rgb.argtypes = [C.c_char_p, _fp, C.POINTER(C.c_ubyte), _sz, C.c_int]
        L.ref_octree_radius.restype = C.c_long
        L.ref_octree_radius.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int,
                                        C.c_float, _fp, _fp, _fp, _sz, C.c_float, _lp, _ip,
                                        _fp, _sz]
        L.ref_sor_octree.restype = _sz
        L.ref_sor_octree.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int, C.c_float,
                                     C.c_int, C.c_float, C.c_float, _fp]
        L.ref_normals_octree.restype = None
        L.ref_normals_octree.argtypes = [C.c_int, _fp, _fp, _fp, _sz, C.c_int, C.c_int,
                                         C.c_float, C.c_float, C.c_float, C.c_float,
                                         C.c_float, C.c_int, _fp, _fp, _fp]
        L.ref_pointer_octree_leaves.restype = C.c_long
        L.ref_pointer_octree_leaves.argtypes = [_fp, _fp, _fp, _sz, C.c_int, C.c_int,
                                                C.c_float, _ip, _lp]
        L.ref_nth_element.restype = None
        L.ref_nth_element.argtypes = [_fp, _sz, _sz]
        L.ref_euclidean_clusters.restype = C.c_long
        L.ref_euclidean_clusters.argtypes = [_fp, _fp, _fp, _sz, C.c_float, C.c_int, C.c_int,
                                             _lp, _ip]
        L.ref_rand_stream.restype = None
        L.ref_rand_stream.argtypes = [C.c_uint, C.c_int, _ip]

    def radius_search(self, c, cell, radius, max_nn=0, queries=None, cap=None):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        q = queries if queries is not None else c
        qx, qxp = _f(q.x); qy, qyp = _f(q.y); qz, qzp = _f(q.z)
        nq = qx.shape[0]
        offs = np.zeros(nq + 1, np.int64)
        cap = cap if cap is not None else max(1, nq * (max_nn if max_nn > 0 else 64))
        while True:
            idx = np.zeros(cap, np.int32); d2 = np.zeros(cap, np.float32)
            tot = self.L.ref_hash_radius_search(xp, yp, zp, x.shape[0], cell, qxp, qyp, qzp, nq,
                                                radius, max_nn, _ptr(offs, _lp), _ptr(idx, _ip),
                                                _ptr(d2, _fp), cap)
            if tot >= 0:
                return offs, idx[:tot], d2[:tot]
            cap = int(offs[-1])

    def voxel_grid(self, c, leaf):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        out = np.zeros((max(x.shape[0], 1), 3), np.float32)
        v = self.L.ref_voxel_grid(xp, yp, zp, x.shape[0], leaf, _ptr(out, _fp))
        return out[:v].copy()

    def sor_rvv(self, c, k, alpha):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        out = np.zeros((max(x.shape[0], 1), 3), np.float32)
        v = self.L.ref_sor_rvv(xp, yp, zp, x.shape[0], k, alpha, _ptr(out, _fp))
        return out[:v].copy()

    def sor_spatial_hash(self, c, cell, k, alpha, search_radius):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        out = np.zeros((max(x.shape[0], 1), 3), np.float32)
        v = self.L.ref_sor_spatial_hash(xp, yp, zp, x.shape[0], cell, k, alpha, search_radius,
                                        _ptr(out, _fp))
        return out[:v].copy()

    def normals_hash(self, c, cell, radius, k=10, vp=(0, 0, 0), iters=4):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        nx = np.zeros(n, np.float32); ny = np.zeros(n, np.float32); nz = np.zeros(n, np.float32)
        self.L.ref_normals_hash(xp, yp, zp, n, cell, k, radius, vp[0], vp[1], vp[2], iters,
                                _ptr(nx, _fp), _ptr(ny, _fp), _ptr(nz, _fp))
        return np.stack([nx, ny, nz], 1)

    def normals_sc(self, c, k, vp=(0, 0, 0), iters=4):
        aos = np.ascontiguousarray(np.stack([c.x, c.y, c.z], 1), np.float32)
        n = aos.shape[0]
        nx = np.zeros(n, np.float32); ny = np.zeros(n, np.float32); nz = np.zeros(n, np.float32)
        self.L.ref_normals_sc(_ptr(aos, _fp), n, k, 0.0, vp[0], vp[1], vp[2], iters,
                              _ptr(nx, _fp), _ptr(ny, _fp), _ptr(nz, _fp))
        return np.stack([nx, ny, nz], 1)

    def ransac_plane(self, c, thresh, max_iters, collinear=1e-6, prob=0.99):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        model = np.zeros(4, np.float32)
        best = self.L.ref_ransac_plane(xp, yp, zp, x.shape[0], thresh, max_iters, collinear,
                                       prob, _ptr(model, _fp))
        return best, model

    def save_pcd(self, path, xyz, binary, rgb=None):
        a = np.ascontiguousarray(xyz, np.float32)
        if rgb is None:
            self.L.ref_save_pcd(path.encode(), _ptr(a, _fp), a.shape[0], int(binary))
        else:
            c = np.ascontiguousarray(rgb, np.uint8)
            self.L.ref_save_pcd_rgb(path.encode(), _ptr(a, _fp), _ptr(c, C.POINTER(C.c_ubyte)),
                                    a.shape[0], int(binary))

    def load_pcd(self, path, cap):
        out = np.zeros((max(cap, 1), 3), np.float32)
        k = self.L.ref_load_pcd(path.encode(), _ptr(out, _fp), cap)
        return out[:max(k, 0)].copy() if k >= 0 else None

    # kind 0: Octree, 1: PointerOctree::radiusSearch, 2: radiusSearchScalar
    def octree_radius(self, kind, c, radius, queries=None, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        q = queries if queries is not None else c
        qx, qxp = _f(q.x); qy, qyp = _f(q.y); qz, qzp = _f(q.z)
        nq = qx.shape[0]
        offs = np.zeros(nq + 1, np.int64)
        cap = 1 << 16
        while True:
            idx = np.zeros(cap, np.int32); d2 = np.zeros(cap, np.float32)
            t = self.L.ref_octree_radius(kind, xp, yp, zp, x.shape[0], tree[0], tree[1],
                                         tree[2], qxp, qyp, qzp, nq, radius, _ptr(offs, _lp),
                                         _ptr(idx, _ip), _ptr(d2, _fp), cap)
            if t <= cap:
                return offs, idx[:t].copy(), d2[:t].copy()
            cap = t

    def sor_octree(self, kind, c, k, alpha, search_radius, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        out = np.zeros((max(x.shape[0], 1), 3), np.float32)
        m = self.L.ref_sor_octree(kind, xp, yp, zp, x.shape[0], tree[0], tree[1], tree[2], k,
                                  alpha, search_radius, _ptr(out, _fp))
        return out[:m].copy()

    # kind 0: Octree, 1: PointerOctree, 2: the self-building overload
    def normals_octree(self, kind, c, radius, vp=(0, 0, 0), iters=4, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        nx, ny, nz = (np.zeros(max(n, 1), np.float32) for _ in range(3))
        self.L.ref_normals_octree(kind, xp, yp, zp, n, tree[0], tree[1], tree[2], radius,
                                  vp[0], vp[1], vp[2], iters, _ptr(nx, _fp), _ptr(ny, _fp),
                                  _ptr(nz, _fp))
        return np.stack([nx[:n], ny[:n], nz[:n]], 1)

    def pointer_octree_leaves(self, c, tree=(64, 8, 1e-4)):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        order = np.zeros(max(n, 1), np.int32); offs = np.zeros(n + 2, np.int64)
        L = self.L.ref_pointer_octree_leaves(xp, yp, zp, n, tree[0], tree[1], tree[2],
                                             _ptr(order, _ip), _ptr(offs, _lp))
        return order[:n], offs[:L + 1]

    def nth_element(self, a, nth):
        a = np.ascontiguousarray(a, np.float32).copy()
        self.L.ref_nth_element(_ptr(a, _fp), a.shape[0], nth)
        return a

    def euclidean_clusters(self, c, tolerance, min_size=1, max_size=2**31 - 1):
        return _clusters(self.L.ref_euclidean_clusters, c, tolerance, min_size, max_size)

    def extract_plane(self, c, model, thresh):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        n = x.shape[0]
        m = np.ascontiguousarray(model, np.float32)
        a = np.zeros((max(n, 1), 3), np.float32); b = np.zeros((max(n, 1), 3), np.float32)
        ni, no = _sz(0), _sz(0)
        self.L.ref_extract_plane(xp, yp, zp, n, _ptr(m, _fp), thresh, _ptr(a, _fp), _ptr(b, _fp),
                                 C.byref(ni), C.byref(no))
        return a[: ni.value].copy(), b[: no.value].copy()

    def count_plane_inliers(self, c, model, thresh):
        x, xp = _f(c.x); y, yp = _f(c.y); z, zp = _f(c.z)
        m = np.ascontiguousarray(model, np.float32)
        scratch = np.zeros((max(x.shape[0], 1), 3), np.float32)
        return int(self.L.ref_count_plane_inliers(xp, yp, zp, x.shape[0], _ptr(m, _fp), thresh,
                                                  _ptr(scratch, _fp)))

    def rand_stream(self, count, seed=0):
        out = np.zeros(count, np.int32)
        self.L.ref_rand_stream(seed, count, _ptr(out, _ip))
        return out


def libc_rand_stream(count: int, seed: int = 0) -> np.ndarray:
    """Raw glibc rand() values after srand(seed) -- the hypothesis source of
    ransac_plane_sc (ransac_plane.cpp:60,69-71), taken from libc itself."""
    libc = C.CDLL("libc.so.6")
    libc.srand(C.c_uint(seed))
    libc.rand.restype = C.c_int
    return np.array([libc.rand() for _ in range(count)], dtype=np.int32)
