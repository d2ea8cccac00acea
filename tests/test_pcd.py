"""PCD input (io/simple_pcd_loader.h:143-291): ascii, binary and
binary_compressed files, with extra fields around x, y, z. The reference's
own loader (CPU) pins the files; rvp_pcd_load (GPU) must return the same
points bit for bit, on the device and into host arrays."""
import os

import numpy as np
import pytest

from pcd_files import write_pcd
from rvpoint_b200 import datasets as D

MODES = ["ascii", "binary", "binary_compressed"]


def _xyz():
    c = D.room_cloud(n=3000, seed=61)
    xyz = np.stack([c.x, c.y, c.z], 1).astype(np.float32)
    return np.concatenate([xyz, xyz[:500]])  # repeats for the LZF back-references


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("extra", [True, False])
def test_reference_reads_the_written_files(tmp_path, reference, mode, extra):
    xyz = _xyz()
    p = str(tmp_path / f"c_{mode}.pcd")
    write_pcd(p, xyz, mode, extra)
    got = reference.load_pcd(p, xyz.shape[0])
    assert got is not None and np.array_equal(got.view(np.int32), xyz.view(np.int32))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("device", [True, False])
def test_pcd_load_matches(tmp_path, gpu_ctx, mode, device):
    from rvpoint_b200 import api
    xyz = _xyz()
    p = str(tmp_path / f"c_{mode}.pcd")
    write_pcd(p, xyz, mode, True)
    x, y, z = api.load_pcd(p, device=device, ctx=gpu_ctx)
    if device:
        x, y, z = x.cpu().numpy(), y.cpu().numpy(), z.cpu().numpy()
    got = np.stack([x, y, z], 1)
    assert np.array_equal(got.view(np.int32), xyz.view(np.int32))


def _build_driver(tmp_path):
    import subprocess
    from rvpoint_b200 import build as B
    B.build()
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    lib = os.path.join(root, "rvpoint_b200", "lib")
    exe = str(tmp_path / "dropin_pcd")
    r = subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(root, "include", "rvpoint"),
                        os.path.join(root, "tests", "dropin_pcd.cpp"), "-o", exe, "-L", lib,
                        "-lrvpoint_b200", "-Wl,-rpath," + lib], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_dropin_save_matches_reference_bytes(tmp_path, reference):
    """savePCD / savePCDRGB write no GPU data: the files must be the
    reference's byte for byte, ascii (default stream formatting) and binary."""
    import subprocess
    exe = _build_driver(tmp_path)
    xyz = _xyz()[:700]
    rgb = np.random.default_rng(3).integers(0, 256, (xyz.shape[0], 3), dtype=np.uint8)
    inp = tmp_path / "in.bin"
    inp.write_bytes(np.uint64(xyz.shape[0]).tobytes() + xyz.tobytes() + rgb.tobytes())
    r = subprocess.run([exe, "save", str(inp), str(tmp_path / "ours")], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    for binary in (False, True):
        tag = "b" if binary else "a"
        reference.save_pcd(str(tmp_path / f"ref_{tag}.pcd"), xyz, binary)
        reference.save_pcd(str(tmp_path / f"ref_rgb_{tag}.pcd"), xyz, binary, rgb)
        for kind in ("", "rgb_"):
            ours = (tmp_path / f"ours_{kind}{tag}.pcd").read_bytes()
            ref = (tmp_path / f"ref_{kind}{tag}.pcd").read_bytes()
            assert ours == ref, (kind, tag)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", MODES)
def test_dropin_load_matches_reference(tmp_path, reference, mode):
    import subprocess
    exe = _build_driver(tmp_path)
    xyz = _xyz()
    p = str(tmp_path / f"c_{mode}.pcd")
    write_pcd(p, xyz, mode, True)
    out = tmp_path / "out.bin"
    r = subprocess.run([exe, "load", p, str(out)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    buf = out.read_bytes()
    k = int(np.frombuffer(buf, np.int64, 1)[0])
    got = np.frombuffer(buf, np.float32, 3 * k, 8).reshape(k, 3)
    ref = reference.load_pcd(p, xyz.shape[0])
    assert k == ref.shape[0] and np.array_equal(got.view(np.int32), ref.view(np.int32))


@pytest.mark.gpu
def test_dropin_load_errors_like_reference(tmp_path, reference):
    """A missing file, a header without z and a short binary payload: -1, as
    the reference returns."""
    import subprocess
    exe = _build_driver(tmp_path)
    xyz = _xyz()[:100]
    good = tmp_path / "g.pcd"
    write_pcd(str(good), xyz, "binary", False)
    data = good.read_bytes()
    noz = tmp_path / "noz.pcd"
    noz.write_bytes(data.replace(b"FIELDS x y z", b"FIELDS x y w"))
    short = tmp_path / "short.pcd"
    short.write_bytes(data[:-5])
    for p in (tmp_path / "missing.pcd", noz, short):
        assert reference.load_pcd(str(p), 100) is None
        out = tmp_path / "out.bin"
        r = subprocess.run([exe, "load", str(p), str(out)], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert int(np.frombuffer(out.read_bytes(), np.int64, 1)[0]) == -1


@pytest.mark.gpu
def test_pcd_capacity_error(tmp_path, gpu_ctx):
    """Capacity below the point count: RVP_ERR_CAPACITY, the count reported,
    nothing written."""
    import ctypes as C
    import torch
    from rvpoint_b200 import _lib
    xyz = _xyz()
    p = str(tmp_path / "c.pcd")
    write_pcd(p, xyz, "binary", True)
    x, y, z = (torch.full((100,), 7.0, device="cuda") for _ in range(3))
    n = C.c_size_t(0)
    st = gpu_ctx.L.rvp_pcd_load(gpu_ctx.h, p.encode(), 1, C.c_void_p(x.data_ptr()),
                                C.c_void_p(y.data_ptr()), C.c_void_p(z.data_ptr()), 100,
                                C.byref(n))
    assert st == _lib.RVP_ERR_CAPACITY and n.value == xyz.shape[0]
    assert bool((x == 7.0).all())
