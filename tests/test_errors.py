"""Error paths of the C ABI on the GPU, made on the host: allocation failures
injected through the library's own allocator hook (rvp_debug_fail_allocation)
and output buffers below the result size. Each must return its status, leave
no device memory behind, and let the same call succeed afterwards.
"""
import ctypes as C

import numpy as np
import pytest

from rvpoint_b200 import datasets as D

pytestmark = pytest.mark.gpu


def live(L):
    d, p = C.c_longlong(0), C.c_longlong(0)
    L.rvp_debug_live_bytes(C.byref(d), C.byref(p))
    return d.value, p.value


@pytest.fixture
def lib(gpu_ctx):
    L = gpu_ctx.L
    yield L
    L.rvp_debug_fail_allocation(-1)


@pytest.mark.parametrize("after", [0, 1, 7, 20])
def test_pipeline_create_out_of_memory_frees_everything(gpu_ctx, lib, after):
    from rvpoint_b200 import _lib
    from rvpoint_b200 import api
    base = live(lib)
    cfg = _lib.PipelineConfig(0.1, 16, 1.0, 16, 4, 0.0, 0.0, 0.0, 0.05, 1000, 1e-6, 0.99, 0.0,
                              0, 0)
    h = C.c_void_p()
    lib.rvp_debug_fail_allocation(after)
    st = lib.rvp_pipeline_create(gpu_ctx.h, C.byref(cfg), 200_000, 8, C.byref(h))
    lib.rvp_debug_fail_allocation(-1)
    assert st == _lib.RVP_ERR_OOM
    assert not h.value
    assert b"injected" in lib.rvp_last_error(gpu_ctx.h)
    assert live(lib) == base  # nothing leaked
    # the same call succeeds once memory is available, and runs
    p = api.Pipeline(max_points=200_000, max_frames=8)
    b = D.lidar_batch(n_frames=2, seed=3, min_pts=3000, max_pts=6000)
    r = p.run_host(b)
    assert r["sor_offsets"][-1] > 0
    p.close()


def test_hash_build_out_of_memory_then_retry(gpu_ctx, lib, restatement):
    from rvpoint_b200 import _lib
    from rvpoint_b200 import api
    c = D.room_cloud(n=20_000, seed=5)
    h = api.SpatialHash()
    h.setInputCloud(c, 0.05)
    lib.rvp_debug_fail_allocation(0)
    st = lib.rvp_hash_build(h.h)
    lib.rvp_debug_fail_allocation(-1)
    assert st == _lib.RVP_ERR_OOM
    h.build()  # the retry builds the same hash
    offs, idx, d2 = h.radiusSearchBatch(c.x, c.y, c.z, 0.05)
    o2, i2, e2 = restatement.radius_search(c, 0.05, 0.05)
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)
    base = live(lib)
    h.close()
    assert live(lib)[0] < base[0]


def test_radius_search_capacity_then_retry(gpu_ctx, lib, restatement):
    """A capacity below the total: RVP_ERR_CAPACITY, *total and the offsets
    filled, nothing else written; a retry with that capacity gives the exact
    result."""
    from rvpoint_b200 import _lib
    from rvpoint_b200 import api
    c = D.room_cloud(n=20_000, seed=9)
    h = api.SpatialHash()
    h.setInputCloud(c, 0.03)
    h.build()
    o2, i2, e2 = restatement.radius_search(c, 0.03, 0.03)
    nq = c.n
    offs = np.zeros(nq + 1, np.int64)
    cap = int(o2[-1]) // 2
    idx = np.full(cap, -7, np.int32)
    d2 = np.full(cap, -7.0, np.float32)
    total = C.c_size_t(0)
    P = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    st = lib.rvp_hash_radius_search(h.h, P(c.x), P(c.y), P(c.z), nq, 0.03, 0, 0, P(offs), P(idx),
                                    P(d2), cap, C.byref(total))
    assert st == _lib.RVP_ERR_CAPACITY
    assert total.value == int(o2[-1])
    assert np.array_equal(offs, o2)
    assert np.all(idx == -7) and np.all(d2 == -7.0)
    idx = np.zeros(total.value, np.int32)
    d2 = np.zeros(total.value, np.float32)
    st = lib.rvp_hash_radius_search(h.h, P(c.x), P(c.y), P(c.z), nq, 0.03, 0, 0, P(offs), P(idx),
                                    P(d2), total.value, C.byref(total))
    assert st == _lib.RVP_OK
    assert np.array_equal(offs, o2) and np.array_equal(idx, i2)
    assert np.array_equal(d2.view(np.int32), e2.view(np.int32))


def test_one_shot_entry_point_out_of_memory(gpu_ctx, lib, restatement):
    """An entry point that grows the context's scratch: OOM, then the same
    call succeeds with the exact result."""
    from rvpoint_b200 import api
    from rvpoint_b200._lib import RvpError
    c = D.room_cloud(n=30_000, seed=13)
    ctx = api.Context(0)
    lib.rvp_debug_fail_allocation(0)
    with pytest.raises(RvpError) as e:
        api.sor_rvv(c, 16, 1.0, ctx=ctx)
    lib.rvp_debug_fail_allocation(-1)
    assert e.value.status == 2
    out = api.sor_rvv(c, 16, 1.0, ctx=ctx)
    o2, _, _ = restatement.sor_exact(c, 16, 1.0)
    assert np.array_equal(out.view(np.int32), o2.view(np.int32))
    ctx.close()
