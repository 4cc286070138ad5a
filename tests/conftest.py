import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds the oracle (always) and, when the sources are newer, the
    product library (nvcc cross-compiles without a GPU)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import build as oracle_build  # oracle/build.py
    oracle_build.build_oracle()
    sys.path.pop(0)
    from simcore_b200 import build as product_build  # noqa: F401
    yield
