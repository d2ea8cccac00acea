"""CPU: the oracle restatement pinned against the reference.

1. Against the committed golden fixtures (outputs of the reference's own
   scalar code, tests/golden/make_golden.py) -- always runs.
2. Against the reference library compiled from its sources (oracle/_ref),
   on fresh seeded inputs -- runs where oracle/_ref was built.
"""
import os

import numpy as np
import pytest

from rvpoint_b200 import datasets as D

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden.npz")


def bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.int32)


@pytest.fixture(scope="module")
def golden():
    return dict(np.load(GOLDEN))


def cloud(a):
    return D.Cloud.from_xyz(a)


@pytest.mark.parametrize("name,src,cell,r,mnn", [
    ("room_r03", "room", 0.03, 0.03, 0),
    ("room_r05_c02", "room", 0.02, 0.05, 0),
    ("lidar_r5", "lidar", 0.5, 0.5, 0),
    ("lidar_knn16", "lidar", 0.5, 0.5, 16),
])
def test_golden_radius_search(golden, restatement, name, src, cell, r, mnn):
    o, i, d = restatement.radius_search(cloud(golden[src]), cell, r, max_nn=mnn)
    assert np.array_equal(o, golden[f"rs_{name}_offsets"])
    assert np.array_equal(i, golden[f"rs_{name}_idx"])
    assert np.array_equal(bits(d), bits(golden[f"rs_{name}_d2"]))


@pytest.mark.parametrize("name,src,leaf", [("vox_room_01", "room", 0.01),
                                           ("vox_room_05", "room", 0.05),
                                           ("vox_lidar_1", "lidar", 0.1)])
def test_golden_voxel(golden, restatement, name, src, leaf):
    v, _ = restatement.voxel_grid(cloud(golden[src]), leaf)
    assert np.array_equal(bits(v), bits(golden[name]))


def test_golden_sor(golden, restatement):
    s, _, _ = restatement.sor_exact(cloud(golden["room"]), 30, 1.0)
    assert np.array_equal(bits(s), bits(golden["sor_room_k30"]))
    s, _, _ = restatement.sor_exact(cloud(golden["lidar"]), 16, 1.0)
    assert np.array_equal(bits(s), bits(golden["sor_lidar_k16"]))
    s, _, _ = restatement.sor_radius(cloud(golden["room"]), 0.1, 16, 1.0, 0.1)
    assert np.array_equal(bits(s), bits(golden["sorh_room_k16"]))


def test_golden_normals(golden, restatement):
    n = restatement.normals_radius(cloud(golden["room"]), 0.03, 0.03)
    assert np.array_equal(bits(n), bits(golden["nrm_room_r03"]))
    n = restatement.normals_knn(cloud(golden["room"]), 16)
    # the reference's partial_sort leaves equal distances in unspecified
    # order; with distinct distances the restatement is bit-identical
    same = np.all(bits(n) == bits(golden["nrm_room_knn16"]), axis=1)
    assert same.mean() > 0.999


def test_golden_ransac(golden, restatement):
    rs = golden["rand_stream_3000"]
    for name, t in [("room", 0.01), ("lidar", 0.05)]:
        best, model, counts, _, _ = restatement.ransac_plane(cloud(golden[name]), t, 1000, rs)
        assert best == int(golden[f"ransac_{name}_best"][0])
        assert np.array_equal(bits(model), bits(golden[f"ransac_{name}_model"]))


def test_libc_rand_stream_matches_reference_stream(golden):
    from oracle.oracle import libc_rand_stream
    assert np.array_equal(libc_rand_stream(3000), golden["rand_stream_3000"])


# ---------------------------------------------------------------------------
# against the compiled reference, fresh inputs
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("seed", [1, 2])
def test_reference_radius_and_knn(reference, restatement, seed):
    c = D.room_cloud(n=15000, seed=seed)
    for cell, r, mnn in [(0.03, 0.03, 0), (0.05, 0.05, 16), (0.1, 0.04, 0)]:
        a = reference.radius_search(c, cell, r, max_nn=mnn)
        b = restatement.radius_search(c, cell, r, max_nn=mnn)
        assert all(np.array_equal(x.view(np.int32) if x.dtype == np.float32 else x,
                                  y.view(np.int32) if y.dtype == np.float32 else y)
                   for x, y in zip(a, b))


def test_reference_collision_primes(reference, restatement):
    """setHashPrimes with colliding primes: duplicates and all."""
    import ctypes  # noqa: F401
    c = D.room_cloud(n=3000, seed=3)
    # reference API has no primes argument in the shim; compare the default
    # and the restatement's own collision path against brute force instead
    o, i, d = restatement.radius_search(c, 0.1, 0.1, p1=3, p2=5)
    o0, i0, d0 = restatement.radius_search(c, 0.1, 0.1)
    # collisions only ever add (duplicate or far-filtered) entries
    assert (np.diff(o) >= np.diff(o0)).all()


@pytest.mark.parametrize("seed", [3, 4])
def test_reference_voxel_sor_normals_ransac(reference, restatement, seed):
    c = D.room_cloud(n=12000, seed=seed)
    v1, _ = restatement.voxel_grid(c, 0.02)
    v2 = reference.voxel_grid(c, 0.02)
    assert np.array_equal(bits(v1), bits(v2))
    vc = cloud(v1)
    s1, _, _ = restatement.sor_exact(vc, 30, 1.0)
    s2 = reference.sor_rvv(vc, 30, 1.0)
    assert np.array_equal(bits(s1), bits(s2))
    n1 = restatement.normals_radius(vc, 0.05, 0.05)
    n2 = reference.normals_hash(vc, 0.05, 0.05)
    assert np.array_equal(bits(n1), bits(n2))
    rs = reference.rand_stream(3000)
    b1, m1, counts, models, _ = restatement.ransac_plane(vc, 0.01, 1000, rs)
    b2, m2 = reference.ransac_plane(vc, 0.01, 1000)
    assert b1 == b2 and np.array_equal(bits(m1), bits(m2))
    for h in range(0, 1000, 37):  # per-hypothesis counts via the reference's extraction
        if counts[h] >= 0:
            assert reference.count_plane_inliers(vc, models[h], 0.01) == counts[h]
    a1, o1 = restatement.extract_plane(vc, m1, 0.01)
    a2, o2 = reference.extract_plane(vc, m2, 0.01)
    assert np.array_equal(a1, a2) and np.array_equal(o1, o2)


def test_reference_lidar_frame(reference, restatement):
    f = D.lidar_frame(seed=77)
    rng = np.random.default_rng(0)
    f = f.subset(np.sort(rng.choice(f.n, 6000, replace=False)))
    a = reference.radius_search(f, 0.5, 0.5, max_nn=16)
    b = restatement.radius_search(f, 0.5, 0.5, max_nn=16)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    v1, _ = restatement.voxel_grid(f, 0.1)
    assert np.array_equal(bits(v1), bits(reference.voxel_grid(f, 0.1)))
    vc = cloud(v1)
    s1, _, _ = restatement.sor_exact(vc, 16, 1.0)
    assert np.array_equal(bits(s1), bits(reference.sor_rvv(vc, 16, 1.0)))


@pytest.mark.parametrize("name,src,tol,mn,mx", [("room", "room", 0.02, 3, 100000),
                                                ("lidar", "lidar", 0.5, 1, 200)])
def test_golden_euclidean_clusters(golden, restatement, name, src, tol, mn, mx):
    cl = restatement.euclidean_clusters(cloud(golden[src]), tol, mn, mx)
    offs = np.cumsum([0] + [len(k) for k in cl]).astype(np.int64)
    assert np.array_equal(offs, golden[f"ec_{name}_offsets"])
    idx = np.concatenate(cl).astype(np.int32) if cl else np.zeros(0, np.int32)
    assert np.array_equal(idx, golden[f"ec_{name}_idx"])


# ---- Octree / PointerOctree ------------------------------------------------
@pytest.mark.parametrize("kind", [0, 1])
def test_golden_octree(golden, restatement, kind):
    room = cloud(golden["room"])
    for tname, tree in (("d", (64, 8, 1e-4)), ("s", (8, 5, 1e-3))):
        assert np.array_equal(restatement.octree_order(kind, room, tree),
                              golden[f"oct{kind}_order_{tname}"])
    o, i, d = restatement.octree_radius(kind, room, 0.05)
    assert np.array_equal(o, golden[f"oct{kind}_r05_offsets"])
    assert np.array_equal(i, golden[f"oct{kind}_r05_idx"])
    assert np.array_equal(bits(d), bits(golden[f"oct{kind}_r05_d2"]))
    s, _, _ = restatement.sor_octree(kind, room, 20, 1.0, 0.1)
    assert np.array_equal(bits(s), bits(golden[f"oct{kind}_sor_k20"]))
    n = restatement.normals_octree(kind, room, 0.05)
    assert np.array_equal(bits(n), bits(golden[f"oct{kind}_nrm_r05"]))


def test_golden_nth_element(golden, restatement):
    heap = False
    for t in range(4):
        r, h = restatement.nth_element(golden[f"nth{t}_in"], int(golden[f"nth{t}_k"][0]))
        assert np.array_equal(bits(r), bits(golden[f"nth{t}_out"]))
        heap |= h
    assert heap  # the heap-selection branch is pinned too


def test_reference_nth_element(reference, restatement):
    """The restated introselect against the C++ library's nth_element on
    random, few-valued, sorted, reversed and organ-pipe arrays (the last ones
    reach the heap selection)."""
    rng = np.random.default_rng(0)
    heaps = 0
    for t in range(3000):
        n = int(rng.integers(1, 300))
        kind = t % 5
        if kind == 0:
            a = rng.random(n).astype(np.float32)
        elif kind == 1:
            a = rng.integers(0, 4, n).astype(np.float32)
        elif kind == 2:
            a = np.sort(rng.random(n)).astype(np.float32)
        elif kind == 3:
            a = np.sort(rng.random(n))[::-1].astype(np.float32)
        else:
            h = n // 2
            a = np.concatenate([np.arange(h), np.arange(n - h)[::-1]]).astype(np.float32)
        nth = int(rng.integers(0, n))
        s, hp = restatement.nth_element(a, nth)
        heaps += hp
        assert np.array_equal(bits(reference.nth_element(a, nth)), bits(s)), (t, n, nth)
    assert heaps > 0


@pytest.mark.parametrize("seed", [5, 6])
def test_reference_octrees(reference, restatement, seed):
    c = D.room_cloud(n=2500, seed=seed)
    q = D.Cloud.from_xyz(np.array([[0.5, 0.5, 0.5]], np.float32))
    for kind in (0, 1):
        for tree in ((64, 8, 1e-4), (8, 8, 1e-4), (16, 3, 1e-3), (1, 12, 1e-4), (-1, 8, 1e-4)):
            _, i, _ = reference.octree_radius(kind, c, 1e6, queries=q, tree=tree)
            assert np.array_equal(restatement.octree_order(kind, c, tree), i)
        for r in (0.05, 0.2):
            a = reference.octree_radius(kind, c, r)
            b = restatement.octree_radius(kind, c, r)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
            assert np.array_equal(bits(a[2]), bits(b[2]))
        for k, al, r in ((10, 1.0, 0.1), (5, 0.5, 0.05)):
            assert np.array_equal(bits(reference.sor_octree(kind, c, k, al, r)),
                                  bits(restatement.sor_octree(kind, c, k, al, r)[0]))
        assert np.array_equal(bits(reference.normals_octree(kind, c, 0.08)),
                              bits(restatement.normals_octree(kind, c, 0.08)))
    # radiusSearchScalar and the self-building normals overload
    a = reference.octree_radius(2, c, 0.1)
    b = restatement.octree_radius(1, c, 0.1)
    assert np.array_equal(a[1], b[1])
    assert np.array_equal(bits(reference.normals_octree(2, c, 0.08)),
                          bits(restatement.normals_octree(1, c, 0.08)))
    o, l = reference.pointer_octree_leaves(c)
    assert np.array_equal(o, restatement.octree_order(1, c))


def test_reference_octree_edge_cases(reference, restatement):
    """One point, all points equal (the depth limit holds them in one leaf),
    a flat plane (z splits put everything on one side) and a tiny epsilon."""
    rng = np.random.default_rng(12)
    clouds = [np.array([[1.0, 2.0, 3.0]], np.float32),
              np.tile(np.array([[0.5, 0.5, 0.5]], np.float32), (300, 1)),
              np.concatenate([rng.uniform(0, 2, (500, 2)), np.zeros((500, 1))], 1).astype(np.float32),
              rng.normal(size=(700, 3)).astype(np.float32)]
    q = D.Cloud.from_xyz(np.array([[0.0, 0.0, 0.0]], np.float32))
    for pts in clouds:
        c = D.Cloud.from_xyz(pts)
        for kind in (0, 1):
            for tree in ((64, 8, 1e-4), (2, 6, 1e-6), (1, 21, 0.0)):
                _, i, _ = reference.octree_radius(kind, c, 1e6, queries=q, tree=tree)
                assert np.array_equal(restatement.octree_order(kind, c, tree), i), (kind, tree)
            a = reference.octree_radius(kind, c, 0.3)
            b = restatement.octree_radius(kind, c, 0.3)
            assert np.array_equal(a[1], b[1]) and np.array_equal(bits(a[2]), bits(b[2]))
