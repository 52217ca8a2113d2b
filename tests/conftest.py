import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the product library and the oracle when missing (nvcc / g++ are local)."""
    from natureuserinterfacestudio_b200 import build as B
    if not os.path.exists(B.LIB):
        B.build()
    from oracle import oracle as O
    if not os.path.exists(O.ORACLE_SO) or (not O.ref_available() and os.path.isdir(O.REFERENCE_TREE)):
        O.build(reference=True)
    yield


@pytest.fixture(scope="session")
def gpu_ctx():
    if not _gpu_available():
        pytest.skip("no CUDA device")
    from natureuserinterfacestudio_b200 import _lib as L
    ctx = L.Context(0)
    yield ctx
    ctx.close()
