"""ctypes binding of librvpoint_b200.so (the C ABI in include/rvpoint_b200.h).

The library is built in-tree (rvpoint_b200/lib/) by rvpoint_b200.build. There
is no fallback: if the shared library is missing or cannot be loaded, every
entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "librvpoint_b200.so")

RVP_OK = 0
RVP_ERR_INVALID_ARG = 1
RVP_ERR_OOM = 2
RVP_ERR_CAPACITY = 3
RVP_ERR_TIMEOUT = 4
RVP_ERR_CUDA = 5
RVP_ERR_NO_DEVICE = 6
MEM_HOST = 0
MEM_DEVICE = 1

STATUS_NAMES = {0: "ok", 1: "invalid argument", 2: "out of memory", 3: "capacity",
                4: "timeout", 5: "CUDA error", 6: "no device"}


class RvpError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class PipelineConfig(C.Structure):
    _fields_ = [("leaf_size", C.c_float), ("sor_k", C.c_int), ("sor_alpha", C.c_float),
                ("normal_k", C.c_int), ("eigen_iters", C.c_int), ("vp_x", C.c_float),
                ("vp_y", C.c_float), ("vp_z", C.c_float), ("ransac_thresh", C.c_float),
                ("ransac_iters", C.c_int), ("ransac_collinear", C.c_float),
                ("ransac_prob", C.c_float), ("cell_size", C.c_float),
                ("block_threads", C.c_int), ("queries_per_warp", C.c_int)]


class PipelineOutputs(C.Structure):
    _fields_ = [("voxel_aos", C.c_void_p), ("voxel_offsets", C.c_void_p),
                ("sor_aos", C.c_void_p), ("sor_offsets", C.c_void_p), ("nx", C.c_void_p),
                ("ny", C.c_void_p), ("nz", C.c_void_p), ("ransac_model", C.c_void_p),
                ("ransac_count", C.c_void_p), ("ransac_iters", C.c_void_p),
                ("sor_mean_dists", C.c_void_p)]


P = C.c_void_p
SZ = C.c_size_t
F = C.c_float
I = C.c_int

# name -> (restype, argtypes)
SIGNATURES = {
    "rvp_context_create": (I, [I, C.POINTER(P)]),
    "rvp_debug_fail_allocation": (I, [C.c_longlong]),
    "rvp_debug_live_bytes": (I, [C.POINTER(C.c_longlong), C.POINTER(C.c_longlong)]),
    "rvp_context_destroy": (I, [P]),
    "rvp_context_set_stream": (I, [P, P]),
    "rvp_context_synchronize": (I, [P]),
    "rvp_last_error": (C.c_char_p, [P]),
    "rvp_status_string": (C.c_char_p, [I]),
    "rvp_context_launch_count": (C.c_uint64, [P]),
    "rvp_version": (C.c_char_p, []),
    "rvp_hash_create": (I, [P, C.POINTER(P)]),
    "rvp_hash_destroy": (I, [P]),
    "rvp_hash_set_primes": (I, [P, C.c_int64, C.c_int64]),
    "rvp_hash_set_input_cloud": (I, [P, P, P, P, SZ, F, I]),
    "rvp_hash_build": (I, [P]),
    "rvp_hash_has_collisions": (I, [P, C.POINTER(I)]),
    "rvp_hash_radius_search": (I, [P, P, P, P, SZ, F, I, I, P, P, P, SZ, C.POINTER(SZ)]),
    "rvp_hash_knn": (I, [P, P, P, P, SZ, I, F, I, P, P, P]),
    "rvp_voxel_grid": (I, [P, P, P, P, SZ, F, I, P, P, C.POINTER(SZ)]),
    "rvp_sor": (I, [P, P, P, P, SZ, I, F, I, P, C.POINTER(SZ), P, P]),
    "rvp_sor_spatial_hash": (I, [P, I, F, F, I, P, C.POINTER(SZ), P, P]),
    "rvp_normals_radius": (I, [P, F, F, F, F, I, I, P, P, P]),
    "rvp_normals_knn": (I, [P, P, P, P, SZ, I, F, F, F, I, I, P, P, P]),
    "rvp_normals_knn_precise": (I, [P, P, P, P, SZ, I, F, F, F, C.c_double, I, P, P, P, P, P]),
    "rvp_ransac_plane": (I, [P, P, P, P, SZ, F, I, F, F, P, I, P, C.POINTER(I), C.POINTER(I), P]),
    "rvp_extract_plane": (I, [P, P, P, P, SZ, P, F, I, P, P, C.POINTER(SZ), C.POINTER(SZ)]),
    "rvp_extract_plane_noalloc": (I, [P, P, P, P, SZ, P, F, P, P, P]),
    "rvp_pipeline_create": (I, [P, C.POINTER(PipelineConfig), SZ, I, C.POINTER(P)]),
    "rvp_pipeline_destroy": (I, [P]),
    "rvp_pipeline_run_device": (I, [P, P, P, P, P, I, SZ]),
    "rvp_pipeline_capture": (I, [P, P, P, P, P, I, SZ, C.POINTER(C.c_uint64)]),
    "rvp_pipeline_replay": (I, [P]),
    "rvp_pipeline_copy_outputs": (I, [P] * 10),
    "rvp_pipeline_outputs_get": (I, [P, C.POINTER(PipelineOutputs)]),
    "rvp_pipeline_run_host": (I, [P, P, P, P, P, I, P, P, P, P, P, P, P, P, P]),
    "rvp_pipeline_run_host_batches": (I, [P, I] + [P] * 14),
    "rvp_pipeline_set_timing": (I, [P, I]),
    "rvp_pipeline_set_tuning": (I, [P, F, I, I]),
    "rvp_pipeline_set_search_radius_factor": (I, [P, F]),
    "rvp_pipeline_set_lane_levels": (I, [P, I]),
    "rvp_pipeline_frame_offsets": (I, [P, P, P]),
    "rvp_pipeline_fit_tables": (I, [P]),
    "rvp_pipeline_check": (I, [P]),
    "rvp_pipeline_knn_routed": (I, [P, P]),
    "rvp_pipeline_knn_stats": (I, [P, I, P]),
    "rvp_pipeline_stage_times": (I, [P, C.POINTER(F), I, C.POINTER(I)]),
    # batched RANSAC and the learned proposal
    "rvp_ransac_frames": (I, [P, P, P, P, P, I, I, F, F, F, P, P, P, P]),
    "rvp_ransac_weighted": (I, [P, P, P, P, P, I, P, P, SZ, P, F, C.c_uint64, I, F, F, F, P, P,
                                P, P]),
    "rvp_plane_labels": (I, [P, P, P, P, P, I, SZ, P, F, P]),
    "rvp_euclidean_clusters": (I, [P, P, P, P, SZ, F, I, I, I, P, P, C.POINTER(SZ)]),
    "rvp_octree_create": (I, [P, C.c_int, C.POINTER(P)]),
    "rvp_octree_destroy": (I, [P]),
    "rvp_octree_set_params": (I, [P, C.c_int, C.c_int, C.c_float]),
    "rvp_octree_set_input_cloud": (I, [P, P, P, P, SZ, I]),
    "rvp_octree_build": (I, [P]),
    "rvp_octree_order": (I, [P, I, P]),
    "rvp_octree_radius_search": (I, [P, P, P, P, SZ, C.c_float, I, P, P, P, SZ,
                                     C.POINTER(SZ)]),
    "rvp_sor_octree": (I, [P, C.c_int, C.c_float, C.c_float, I, P, C.POINTER(SZ), P, P]),
    "rvp_normals_octree": (I, [P, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int, I, P,
                               P, P]),
    "rvp_pcd_load": (I, [P, C.c_char_p, I, P, P, P, SZ, C.POINTER(SZ)]),
    "rvp_ransac_preemptive": (I, [P, P, P, P, P, I, P, P, SZ, P, F, C.c_uint64, I, I, F, F, P, P,
                                  P, P]),
    "rvp_scorer_create": (I, [P, SZ, I, C.POINTER(P)]),
    "rvp_scorer_destroy": (I, [P]),
    "rvp_scorer_set_knn": (I, [P, I, F]),
    "rvp_scorer_features": (I, [P, P, P, P, P, I, SZ, F, P, P, SZ, I, P]),
    "rvp_mlp_set_params": (I, [P, P]),
    "rvp_mlp_get_params": (I, [P, P]),
    "rvp_mlp_set_norm": (I, [P, P, P]),
    "rvp_mlp_forward": (I, [P, P, SZ, P]),
    "rvp_mlp_gradients": (I, [P, P, P, SZ, P, C.POINTER(C.c_double)]),
    "rvp_mlp_train_step": (I, [P, P, P, SZ, SZ, C.c_uint64, F, C.POINTER(C.c_double)]),
}

MLP_INPUTS = 8
MLP_HIDDEN = 64
MLP_PARAMS = 4801

_lib = None


def load(path: str = LIB_PATH):
    """Load the shared library (building it first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        from . import build as _build
        _build.build()
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int, ctx=None) -> None:
    if status != RVP_OK:
        msg = ""
        if ctx:
            m = load().rvp_last_error(ctx)
            msg = m.decode() if m else ""
        raise RvpError(status, msg)
