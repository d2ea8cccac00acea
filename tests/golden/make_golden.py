"""Regenerate the golden fixtures from the reference's own code.

Runs the reference's scalar path (oracle/_ref/librvpoint_ref.so, compiled
from the reference sources by oracle/Makefile) on small seeded inputs and
stores inputs and outputs in tests/golden/golden.npz. The fixtures pin the
CPU restatement (oracle/rvp_oracle.c) and, through it, the GPU parity tests.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from rvpoint_b200 import datasets as D  # noqa: E402


def main():
    O.build()
    R = O.Reference()
    out = {}
    # inputs (seeded; stored so the fixtures do not depend on numpy's streams)
    room = D.room_cloud(n=4000, seed=1234)
    lid = D.lidar_frame(seed=4321)
    rng = np.random.default_rng(99)
    lid = lid.subset(np.sort(rng.choice(lid.n, 5000, replace=False)))
    out["room"] = room.aos()
    out["lidar"] = lid.aos()
    # SpatialHash radiusSearch (spatial_hashing.cpp:110-168)
    for name, c, cell, r, mnn in [("room_r03", room, 0.03, 0.03, 0),
                                  ("room_r05_c02", room, 0.02, 0.05, 0),
                                  ("lidar_r5", lid, 0.5, 0.5, 0),
                                  ("lidar_knn16", lid, 0.5, 0.5, 16)]:
        o, i, d = R.radius_search(c, cell, r, max_nn=mnn)
        out[f"rs_{name}_offsets"] = o
        out[f"rs_{name}_idx"] = i
        out[f"rs_{name}_d2"] = d
    # voxel grid (voxel_grid_downsamp_rvv_v2 -> _sc)
    out["vox_room_01"] = R.voxel_grid(room, 0.01)
    out["vox_room_05"] = R.voxel_grid(room, 0.05)
    out["vox_lidar_1"] = R.voxel_grid(lid, 0.1)
    # SOR (sor_rvv -> sor_sc; sor_spatial_hash)
    out["sor_room_k30"] = R.sor_rvv(room, 30, 1.0)
    out["sor_lidar_k16"] = R.sor_rvv(lid, 16, 1.0)
    out["sorh_room_k16"] = R.sor_spatial_hash(room, 0.1, 16, 1.0, 0.1)
    # normals (SpatialHash overload; brute-force _sc)
    out["nrm_room_r03"] = R.normals_hash(room, 0.03, 0.03)
    out["nrm_room_knn16"] = R.normals_sc(room, 16)
    # RANSAC (ransac_plane_rvv -> _sc) + per-hypothesis counts via the
    # reference's own inlier extraction of each hypothesis model
    for name, c, t, it in [("room", room, 0.01, 1000), ("lidar", lid, 0.05, 1000)]:
        best, model = R.ransac_plane(c, t, it)
        out[f"ransac_{name}_best"] = np.array([best], np.int32)
        out[f"ransac_{name}_model"] = model
    out["rand_stream_3000"] = R.rand_stream(3000)
    # Euclidean clustering (euclidean_clustering.cpp:113-189), CSR
    for name, c, tol, mn, mx in [("room", room, 0.02, 3, 100000), ("lidar", lid, 0.5, 1, 200)]:
        cl = R.euclidean_clusters(c, tol, mn, mx)
        out[f"ec_{name}_offsets"] = np.cumsum([0] + [len(k) for k in cl]).astype(np.int64)
        out[f"ec_{name}_idx"] = (np.concatenate(cl) if cl else np.zeros(0)).astype(np.int32)
    # Octree / PointerOctree: leaf order (radiusSearch over everything),
    # radius lists in tree order, sor_octree / sor_pointer_octree, normals
    big = D.Cloud.from_xyz(np.array([[0.0, 0.0, 0.0]], np.float32))
    for kind in (0, 1):
        for tname, tree in (("d", (64, 8, 1e-4)), ("s", (8, 5, 1e-3))):
            _, i, _ = R.octree_radius(kind, room, 1e6, queries=big, tree=tree)
            out[f"oct{kind}_order_{tname}"] = i
        o, i, d = R.octree_radius(kind, room, 0.05)
        out[f"oct{kind}_r05_offsets"] = o
        out[f"oct{kind}_r05_idx"] = i
        out[f"oct{kind}_r05_d2"] = d
        out[f"oct{kind}_sor_k20"] = R.sor_octree(kind, room, 20, 1.0, 0.1)
        out[f"oct{kind}_nrm_r05"] = R.normals_octree(kind, room, 0.05)
    # std::nth_element (sor_pointer_octree's step): inputs and results
    rng = np.random.default_rng(7)
    nth_in = [rng.random(257).astype(np.float32), rng.integers(0, 5, 100).astype(np.float32),
              np.concatenate([np.arange(150), np.arange(150)[::-1]]).astype(np.float32),
              # organ pipe of 85 with nth 35: the depth limit runs out (heap selection)
              np.concatenate([np.arange(42), np.arange(43)[::-1]]).astype(np.float32)]
    for t, a in enumerate(nth_in):
        nth = [100, 37, 120, 35][t]
        out[f"nth{t}_in"] = a
        out[f"nth{t}_k"] = np.array([nth], np.int64)
        out[f"nth{t}_out"] = R.nth_element(a, nth)
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()
