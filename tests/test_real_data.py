"""Real clouds: the PCD files that ship with the reference (bunny.pcd, ascii;
0000000000.pcd, a binary LiDAR scan; table_scene_lms400.pcd,
binary_compressed) through the steps of its integration tests
(tests/integration/test_spatial_hash_comparison.cpp:18-149: voxel 0.01,
then SpatialHash radius search r = 0.05 with cell 1.5 r), plus SOR.

The files are not part of this repository: they are read from
$RVP_DATA_DIR, else from the reference checkout's data/ folder, and the
tests skip where neither exists.

CPU: the restatement against the reference's own code on these clouds.
GPU: PCD load, voxel grid, radius search and SOR through the C ABI against
the restatement (and the load against the reference's loadPCD), bit for bit.
"""
import os

import numpy as np
import pytest

from rvpoint_b200 import datasets as D

# file, voxel leaf, radius, SOR k
CASES = [("bunny.pcd", 0.01, 0.05, 10),
         ("0000000000.pcd", 0.1, 0.5, 16),
         ("table_scene_lms400.pcd", 0.01, 0.05, 16)]


def data_dir():
    d = os.environ.get("RVP_DATA_DIR")
    if d and os.path.isdir(d):
        return d
    from oracle import oracle as O
    ref = O.reference_checkout()
    if ref and os.path.isdir(os.path.join(ref, "data")):
        return os.path.join(ref, "data")
    return None


def _path(name):
    d = data_dir()
    if d is None or not os.path.exists(os.path.join(d, name)):
        pytest.skip(f"{name} not available (set RVP_DATA_DIR)")
    return os.path.join(d, name)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def _load_ref(reference, path):
    pts = reference.load_pcd(path, 2_000_000)
    assert pts is not None and pts.shape[0] > 0
    return D.Cloud.from_xyz(pts)


@pytest.mark.parametrize("name,leaf,radius,k", CASES)
def test_restatement_matches_reference_on_real_clouds(reference, restatement, name, leaf, radius,
                                                      k):
    c = _load_ref(reference, _path(name))
    v = reference.voxel_grid(c, leaf)
    v2, _ = restatement.voxel_grid(c, leaf)
    assert np.array_equal(bits(v), bits(v2))
    vc = D.Cloud.from_xyz(v2)
    cell = 1.5 * radius
    o, i, d = reference.radius_search(vc, cell, radius)
    o2, i2, d2 = restatement.radius_search(vc, cell, radius)
    assert np.array_equal(o, o2) and np.array_equal(i, i2) and np.array_equal(bits(d), bits(d2))
    if vc.n <= 40_000:  # the reference's sor_rvv is quadratic on one thread
        s = reference.sor_rvv(vc, k, 1.0)
        s2, _, _ = restatement.sor_exact(vc, k, 1.0)
        assert np.array_equal(bits(s), bits(s2))


@pytest.mark.gpu
@pytest.mark.parametrize("name,leaf,radius,k", CASES)
def test_gpu_matches_oracle_on_real_clouds(gpu_ctx, reference, restatement, name, leaf, radius,
                                           k):
    from rvpoint_b200 import api
    path = _path(name)
    x, y, z = api.load_pcd(path)
    ref = reference.load_pcd(path, 2_000_000)
    assert np.array_equal(bits(np.stack([x, y, z], 1)), bits(ref))
    c = D.Cloud.from_xyz(ref)
    v = api.voxel_grid_downsamp_rvv_v2(c, leaf)
    v2, _ = restatement.voxel_grid(c, leaf)
    assert np.array_equal(bits(v), bits(v2))
    vc = D.Cloud.from_xyz(v2)
    h = api.SpatialHash()
    h.setInputCloud(vc, 1.5 * radius)
    h.build()
    offs, idx, d2 = h.radiusSearchBatch(vc.x, vc.y, vc.z, radius)
    o2, i2, e2 = restatement.radius_search(vc, 1.5 * radius, radius)
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)
    assert np.array_equal(bits(d2), bits(e2))
    s, md, keep = api.sor_rvv(vc, k, 1.0, return_stats=True)
    s2, md2, keep2 = restatement.sor_exact(vc, k, 1.0)
    assert np.array_equal(bits(md), bits(md2))
    assert np.array_equal(bits(s), bits(s2))
