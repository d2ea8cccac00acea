"""GPU: the allocation-free plane split, rvp_extract_plane_noalloc.

It serves callers that cannot allocate device memory at call time (a
control loop that forbids allocation once started, a host framework that
owns every device buffer): they pass device inputs and outputs, and the
library's only scratch is a fixed array inside it. Its results must equal
those of the allocating entry point, rvp_extract_plane, bit for bit (the
tolerance every plane-extraction test here uses), on two calls in a row
that share that array. The file sorts last so that a run stopping at the
first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, torch):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_noalloc_split_matches_allocating_entry_point_twice():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import _lib, api
    from rvpoint_b200 import datasets as D

    lib = _lib.load()
    ctx = api.Context(0)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    cases = [(D.room_cloud(n=150_000, seed=501), np.array([0, 0, 1, -0.001], np.float32), 0.01),
             (D.room_cloud(n=61_777, seed=502), np.array([1, 0, 0, -0.002], np.float32), 0.02)]
    for cloud, model, thresh in cases:
        n = cloud.n
        x, y, z = (_dev(cloud.x, torch), _dev(cloud.y, torch), _dev(cloud.z, torch))
        m = _dev(model, torch)
        ins = torch.full((n, 3), float("nan"), device="cuda")
        outs = torch.full((n, 3), float("nan"), device="cuda")
        counts = torch.zeros(2, dtype=torch.int64, device="cuda")
        ctx.set_stream(torch.cuda.current_stream().cuda_stream)
        st = lib.rvp_extract_plane_noalloc(ctx.h, ptr(x), ptr(y), ptr(z), n, ptr(m), thresh,
                                           ptr(ins), ptr(outs), ptr(counts))
        assert st == _lib.RVP_OK
        torch.cuda.synchronize()
        ni, no = (int(v) for v in counts.cpu())
        ref_in, ref_out = api.extract_plane_inliers_outliers_rvv(cloud, model, thresh, ctx=ctx)
        assert (ni, no) == (len(ref_in), len(ref_out))
        assert ni > 0 and no > 0
        assert np.array_equal(ins[:ni].cpu().numpy().view(np.int32), ref_in.view(np.int32))
        assert np.array_equal(outs[:no].cpu().numpy().view(np.int32), ref_out.view(np.int32))


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
    st = lib.rvp_extract_plane_noalloc(ctx.h, p, p, p, (1 << 24) + 1, p, 0.1, None, None,
                                       C.c_void_p(counts.data_ptr()))
    assert st == _lib.RVP_ERR_INVALID_ARG
