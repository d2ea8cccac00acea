"""CPU: the C-ABI library loads and exports every symbol include/*.h
declares; host-side argument and error handling that needs no kernel."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in os.listdir(inc):
        if f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            names |= set(re.findall(r"^RVP_API\s+[\w\s\*]*?\b(rvp_\w+)\s*\(", txt, re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "rvp_hash_radius_search" in names and "rvp_pipeline_run_device" in names
    assert len(names) >= 29


def test_library_exports_every_declared_symbol():
    from rvpoint_b200 import _lib
    lib = _lib.load()
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing
    # the Python binding covers the same set
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_status_strings_and_version():
    from rvpoint_b200 import _lib
    lib = _lib.load()
    assert lib.rvp_version().decode().startswith("rvpoint_b200")
    assert lib.rvp_status_string(3).decode() == "output capacity too small"


def test_null_arguments_are_rejected_without_a_device():
    from rvpoint_b200 import _lib
    lib = _lib.load()
    assert lib.rvp_context_create(0, None) == _lib.RVP_ERR_INVALID_ARG
    assert lib.rvp_hash_create(None, None) == _lib.RVP_ERR_INVALID_ARG
    assert lib.rvp_voxel_grid(None, None, None, None, 0, 0.1, 0, None, None, None) == \
        _lib.RVP_ERR_INVALID_ARG
    assert lib.rvp_pipeline_destroy(None) == _lib.RVP_ERR_INVALID_ARG


def test_context_without_device_reports_no_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from rvpoint_b200 import _lib
    lib = _lib.load()
    h = C.c_void_p()
    assert lib.rvp_context_create(0, C.byref(h)) == _lib.RVP_ERR_NO_DEVICE


def test_api_fails_loudly_when_library_missing(tmp_path):
    from rvpoint_b200 import _lib
    with pytest.raises(OSError):
        C.CDLL(str(tmp_path / "nope.so"))
    assert os.path.exists(_lib.LIB_PATH)


def test_python_front_end_imports():
    """The host modules load without a device (their module-level code runs)."""
    import importlib
    for m in ("rvpoint_b200.api", "rvpoint_b200.learned", "rvpoint_b200.autotune",
              "rvpoint_b200.sharding", "rvpoint_b200.datasets"):
        importlib.import_module(m)
    from rvpoint_b200 import api
    assert len(api.Pipeline.LEVEL_KERNELS) == 2 * len(api.TIMED_KNN)
