"""GPU: the allocation-free plane split, rvp_extract_plane_noalloc.

It serves callers that cannot allocate device memory at call time (a
control loop that forbids allocation once started, a host framework that
owns every device buffer): they pass device inputs and outputs, and the
library's only scratch is a fixed array inside it. Its results must equal
those of the allocating entry point, rvp_extract_plane, bit for bit (the
tolerance every plane-extraction test here uses), on two calls in a row
that share that array, and the oracle's extract_plane (ransac_plane.cpp:
327-383) on several models and sizes, up to the size limit. The file sorts
last so that a run stopping at the first failure has already run every
other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LIMIT = 1 << 24  # RVP_NOALLOC_MAX_POINTS: 8192 tiles of 2048 points


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _split(lib, ctx, torch, cloud, model, thresh, outliers=True):
    """One call through the C ABI; returns (status, inliers, outliers, counts)
    as host arrays."""
    ptr = lambda t: C.c_void_p(t.data_ptr()) if t is not None else None  # noqa: E731
    n = cloud.n
    x, y, z = (_dev(cloud.x, torch), _dev(cloud.y, torch), _dev(cloud.z, torch))
    m = _dev(np.asarray(model, np.float32), torch)
    ins = torch.full((max(n, 1), 3), float("nan"), device="cuda")
    outs = torch.full((max(n, 1), 3), float("nan"), device="cuda") if outliers else None
    counts = torch.full((2,), -1, dtype=torch.int64, device="cuda")
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    st = lib.rvp_extract_plane_noalloc(ctx.h, ptr(x), ptr(y), ptr(z), n, ptr(m), thresh,
                                       ptr(ins), ptr(outs), ptr(counts))
    torch.cuda.synchronize()
    ni, no = (int(v) for v in counts.cpu())
    return (st, ins[:max(ni, 0)].cpu().numpy(),
            outs[:max(no, 0)].cpu().numpy() if outliers else None, (ni, no))


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.int32)


def test_noalloc_split_matches_allocating_entry_point_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api
    from rvpoint_b200 import datasets as D

    lib = _lib.load()
    ctx = api.Context(0)
    cases = [(D.room_cloud(n=150_000, seed=501), np.array([0, 0, 1, -0.001], np.float32), 0.01),
             (D.room_cloud(n=61_777, seed=502), np.array([1, 0, 0, -0.002], np.float32), 0.02)]
    for cloud, model, thresh in cases:
        st, ins, outs, (ni, no) = _split(lib, ctx, torch, cloud, model, thresh)
        assert st == _lib.RVP_OK
        ref_in, ref_out = api.extract_plane_inliers_outliers_rvv(cloud, model, thresh, ctx=ctx)
        assert (ni, no) == (len(ref_in), len(ref_out))
        assert ni > 0 and no > 0
        assert np.array_equal(_bits(ins), _bits(ref_in))
        assert np.array_equal(_bits(outs), _bits(ref_out))
    ctx.close()


@pytest.mark.parametrize("n,seed", [(2048 * 5, 1), (2048 * 7 + 1, 2), (99_999, 3), (1, 4)])
def test_noalloc_split_matches_oracle(restatement, n, seed):
    """Sizes on and off the 2048-point tile boundary, three models each."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api
    from rvpoint_b200 import datasets as D

    lib = _lib.load()
    ctx = api.Context(0)
    cloud = D.room_cloud(n=max(n, 1000), seed=600 + seed).subset(np.arange(n))
    models = [np.array([0, 0, 1, -0.001], np.float32), np.array([0, 1, 0, -0.5], np.float32),
              np.array([0.6, 0.0, 0.8, -1.2], np.float32)]
    for model in models:
        st, ins, outs, (ni, no) = _split(lib, ctx, torch, cloud, model, 0.01)
        assert st == _lib.RVP_OK
        a, b = restatement.extract_plane(cloud, model, 0.01)
        assert (ni, no) == (len(a), len(b))
        assert np.array_equal(_bits(ins), _bits(a)) and np.array_equal(_bits(outs), _bits(b))
    ctx.close()


def test_noalloc_split_at_the_size_limit(restatement):
    """Exactly 8192 full tiles, against the oracle; the call asks the library
    for no allocation (every allocation through its allocator fails during
    the call) and the device's free memory does not drop."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api
    from rvpoint_b200 import datasets as D

    lib = _lib.load()
    ctx = api.Context(0)
    rng = np.random.default_rng(77)
    xy = rng.uniform(0.0, 10.0, size=(LIMIT, 2)).astype(np.float32)
    z = np.where(rng.uniform(size=LIMIT) < 0.5, 0.3 * xy[:, 0] + rng.normal(0, 0.01, LIMIT),
                 rng.uniform(-2.0, 5.0, LIMIT)).astype(np.float32)
    cloud = D.Cloud(np.ascontiguousarray(xy[:, 0]), np.ascontiguousarray(xy[:, 1]), z)
    model = np.array([-0.3, 0.0, 1.0, 0.0], np.float32) / np.float32(np.sqrt(1.09))
    _split(lib, ctx, torch, D.Cloud(cloud.x[:4096], cloud.y[:4096], cloud.z[:4096]), model, 0.02)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    lib.rvp_debug_fail_allocation(0)
    try:
        st, ins, outs, (ni, no) = _split(lib, ctx, torch, cloud, model, 0.02)
    finally:
        lib.rvp_debug_fail_allocation(-1)
    assert st == _lib.RVP_OK
    a, b = restatement.extract_plane(cloud, model, 0.02)
    assert (ni, no) == (len(a), len(b)) and ni > LIMIT // 3
    assert np.array_equal(_bits(ins), _bits(a)) and np.array_equal(_bits(outs), _bits(b))
    del ins, outs
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    assert torch.cuda.mem_get_info()[0] >= free0 - (1 << 20)
    ctx.close()


def test_noalloc_empty_cloud_and_no_outlier_output(restatement):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api
    from rvpoint_b200 import datasets as D

    lib = _lib.load()
    ctx = api.Context(0)
    model = np.array([0, 0, 1, -0.001], np.float32)
    st, _, _, counts = _split(lib, ctx, torch, D.Cloud(*(np.zeros(0, np.float32),) * 3), model,
                              0.01)
    assert st == _lib.RVP_OK and counts == (0, 0)
    cloud = D.room_cloud(n=30_001, seed=611)
    st, ins, _, (ni, no) = _split(lib, ctx, torch, cloud, model, 0.01, outliers=False)
    assert st == _lib.RVP_OK
    a, b = restatement.extract_plane(cloud, model, 0.01)
    assert (ni, no) == (len(a), len(b))
    assert np.array_equal(_bits(ins), _bits(a))
    ctx.close()


def test_noalloc_keeps_the_callers_current_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api
    from rvpoint_b200 import datasets as D

    lib = _lib.load()
    ctx = api.Context(0)
    before = torch.cuda.current_device()
    st, _, _, _ = _split(lib, ctx, torch, D.room_cloud(n=5000, seed=612),
                         np.array([0, 0, 1, 0], np.float32), 0.01)
    assert st == _lib.RVP_OK and torch.cuda.current_device() == before
    ctx.close()


def test_noalloc_rejects_clouds_above_the_limit():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api

    lib = _lib.load()
    ctx = api.Context(0)
    m = torch.zeros(4, device="cuda")
    counts = torch.zeros(2, dtype=torch.int64, device="cuda")
    p = C.c_void_p(m.data_ptr())
    st = lib.rvp_extract_plane_noalloc(ctx.h, p, p, p, LIMIT + 1, p, 0.1, None, None,
                                       C.c_void_p(counts.data_ptr()))
    assert st == _lib.RVP_ERR_INVALID_ARG
    ctx.close()
