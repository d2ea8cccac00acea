"""The C++ drop-in (include/rvpoint/): reference names and signatures over
the C ABI, compiled the way a caller of the reference would compile it.

CPU: the test driver tests/dropin_main.cpp compiles against the headers and
links against librvpoint_b200.so. GPU: it runs the chain voxel -> SOR ->
SpatialHash -> radiusSearch / normals -> SOR over the hash -> RANSAC -> plane
split, and every output matches the CPU oracle: bit for bit, normals within
the tolerance of the other normal tests, libc's rand() state included.
"""
import os
import subprocess

import numpy as np
import pytest

from rvpoint_b200 import datasets as D

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "rvpoint_b200", "lib")


def _build(tmp_path):
    from rvpoint_b200 import build as B
    B.build()
    exe = str(tmp_path / "dropin_main")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include", "rvpoint"),
           os.path.join(ROOT, "tests", "dropin_main.cpp"), "-o", exe, "-L", LIBDIR,
           "-lrvpoint_b200", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_compiles_and_links(tmp_path):
    assert os.path.exists(_build(tmp_path))


def _arrays(buf, dtypes):
    res, p = [], 0
    for dt in dtypes:
        n = int(np.frombuffer(buf, np.uint64, 1, p)[0])
        p += 8
        a = np.frombuffer(buf, dt, n, p)
        p += n * np.dtype(dt).itemsize
        res.append(a.copy())
    assert p == len(buf)
    return res


def _angle(a, b):
    """Angle between lines (sign-free), in double: atan2(|a x b|, |a . b|)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), np.abs(np.sum(a * b, 1)))


@pytest.mark.gpu
def test_dropin_chain_matches_oracle(tmp_path, restatement):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle.oracle import libc_rand_stream
    exe = _build(tmp_path)
    c = D.room_cloud(n=20_000, seed=77)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.uint64(c.n).tobytes())
        for a in (c.x, c.y, c.z):
            f.write(np.ascontiguousarray(a, np.float32).tobytes())
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(outp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    f32, i32, i64 = np.float32, np.int32, np.int64
    (vox, vox_sc, sor, sor2, counts, idx, d2, nx, ny, nz, kx, ky, kz, filt, rb, model,
     best_sc, model_sc, pin, pout, coffs, cidx, degen) = _arrays(
        outp.read_bytes(), [f32, f32, f32, f32, i64, i32, f32, f32, f32, f32, f32, f32, f32,
                            f32, i32, f32, i32, f32, f32, f32, i64, i32, i64])
    bits = lambda a: np.ascontiguousarray(a, np.float32).view(np.int32)  # noqa: E731
    v, _ = restatement.voxel_grid(c, 0.05)
    assert np.array_equal(bits(vox), bits(v.ravel()))
    assert np.array_equal(bits(vox_sc), bits(v.ravel()))
    vc = D.Cloud.from_xyz(v)
    s, _, _ = restatement.sor_exact(vc, 10, 1.0)
    assert np.array_equal(bits(sor), bits(s.ravel()))
    assert np.array_equal(bits(sor2), bits(s.ravel()))
    sc = D.Cloud.from_xyz(s)
    # radius searches (every 97th point, odd ones cut at 8)
    p = 0
    for j, q in enumerate(range(0, sc.n, 97)):
        qc = D.Cloud.from_xyz(s[q:q + 1])
        _, ri, rd = restatement.radius_search(sc, 0.15, 0.15, max_nn=8 if q % 2 else 0,
                                              queries=qc)
        assert counts[j] == len(ri)
        assert np.array_equal(idx[p:p + counts[j]], ri)
        assert np.array_equal(bits(d2[p:p + counts[j]]), bits(rd))
        p += counts[j]
    assert p == len(idx)

    def close_as_cpu(gpu, c32, c64):
        # within 1e-3 rad of the FP64 oracle at least as often as the FP32 CPU
        e, e_cpu = _angle(gpu, c64), _angle(c32, c64)
        return (e > 1e-3).mean() <= (e_cpu > 1e-3).mean() + 0.005
    assert close_as_cpu(np.stack([nx, ny, nz], 1), restatement.normals_radius(sc, 0.15, 0.15),
                        restatement.normals_radius(sc, 0.15, 0.15, f64=True))
    sub = D.Cloud.from_xyz(s[:3000])
    assert close_as_cpu(np.stack([kx, ky, kz], 1), restatement.normals_knn(sub, 16),
                        restatement.normals_knn(sub, 16, f64=True))
    fr, _, _ = restatement.sor_radius(sc, 0.15, 10, 1.0, 0.15)
    assert np.array_equal(bits(filt), bits(fr.ravel()))
    rs = libc_rand_stream(3000)
    best, m, _, _, it = restatement.ransac_plane(sc, 0.01, 1000, rs)
    assert rb[0] == best and np.array_equal(bits(model), bits(m))
    assert rb[1] == libc_rand_stream(3 * it + 1)[-1]
    assert best_sc[0] == best and np.array_equal(bits(model_sc), bits(m))
    a, b = restatement.extract_plane(sc, m, 0.01)
    assert np.array_equal(bits(pin), bits(a.ravel()))
    assert np.array_equal(bits(pout), bits(b.ravel()))
    cl = restatement.euclidean_clusters(sc, 0.08, 2)
    assert np.array_equal(coffs, np.cumsum([0] + [len(k) for k in cl]))
    assert np.array_equal(cidx, np.concatenate(cl))
    assert list(degen) == [0, 0, 1]


def _build_octree_driver(tmp_path):
    from rvpoint_b200 import build as B
    B.build()
    exe = str(tmp_path / "dropin_octree")
    cmd = ["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include", "rvpoint"),
           os.path.join(ROOT, "tests", "dropin_octree.cpp"), "-o", exe, "-L", LIBDIR,
           "-lrvpoint_b200", "-Wl,-rpath," + LIBDIR]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_octree_compiles_and_links(tmp_path):
    assert os.path.exists(_build_octree_driver(tmp_path))


@pytest.mark.gpu
def test_dropin_octree_matches_oracle(tmp_path, restatement):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import api
    exe = _build_octree_driver(tmp_path)
    c = D.room_cloud(n=6000, seed=91)
    inp = tmp_path / "in.bin"
    with open(inp, "wb") as f:
        f.write(np.uint64(c.n).tobytes())
        for a in (c.x, c.y, c.z):
            f.write(np.ascontiguousarray(a, np.float32).tobytes())
    outp = tmp_path / "out.bin"
    r = subprocess.run([exe, str(inp), str(outp)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    f32, i32, i64 = np.float32, np.int32, np.int64
    (cnt, li, ld, s0, s1, ox, oy, oz, px, py, pz, sx, sy, sz, coffs, cidx, threw) = _arrays(
        outp.read_bytes(), [i64, i32, f32, f32, f32] + [f32] * 9 + [i64, i32, i64])
    bits = lambda a: np.ascontiguousarray(a, np.float32).view(np.int32)  # noqa: E731
    q = c.subset(np.arange(50))
    pos = 0
    for t, (kind, tree) in enumerate(((0, (16, 8, 1e-4)), (1, (64, 8, 1e-4)),
                                      (1, (64, 8, 1e-4)))):
        o, i, d = restatement.octree_radius(kind, c, 0.1, queries=q, tree=tree)
        assert np.array_equal(cnt[50 * t:50 * t + 50], np.diff(o))
        m = int(o[-1])
        assert np.array_equal(li[pos:pos + m], i)
        assert np.array_equal(bits(ld[pos:pos + m]), bits(d))
        pos += m
    r0, _, _ = restatement.sor_octree(0, c, 20, 1.0, 0.25, (16, 8, 1e-4))
    r1, _, _ = restatement.sor_octree(1, c, 20, 1.0, 0.25)
    assert np.array_equal(bits(s0), bits(r0.ravel()))
    assert np.array_equal(bits(s1), bits(r1.ravel()))
    # normals: the same GPU results as the Python API over the same trees
    for (nx_, ny_, nz_), (kind, tree) in (((ox, oy, oz), (0, (16, 8, 1e-4))),
                                          ((px, py, pz), (1, (64, 8, 1e-4))),
                                          ((sx, sy, sz), (1, (64, 8, 1e-4)))):
        t = (api.Octree if kind == 0 else api.PointerOctree)()
        t.setMaxPointsPerLeaf(tree[0])
        t.setInputCloud(c)
        t.build()
        g = np.stack(api.normal_estimation_tree(c, t, 10, 0.1), 1)
        assert np.array_equal(bits(np.stack([nx_, ny_, nz_], 1)), bits(g))
        f32n = restatement.normals_octree(kind, c, 0.1, tree=tree)
        assert (_angle(g, f32n) < 1e-4).mean() > 0.99
        t.close()
    cl = restatement.euclidean_clusters(c, 0.05, 3)
    assert np.array_equal(coffs, np.cumsum([0] + [len(k) for k in cl]))
    assert np.array_equal(cidx, np.concatenate(cl))
    assert int(threw[0]) == 1
