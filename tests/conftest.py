import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def restatement():
    from oracle import oracle as O
    O.build()
    return O.Restatement()


@pytest.fixture(scope="session")
def reference():
    from oracle import oracle as O
    if not O.reference_available():
        pytest.skip("oracle/_ref not built (reference sources absent)")
    return O.Reference()


@pytest.fixture(scope="session")
def gpu_ctx():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from rvpoint_b200 import api
    return api.default_context()
