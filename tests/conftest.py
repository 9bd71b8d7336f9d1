import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REF_OPS = os.path.join(ROOT, "oracle", "_ref", "libfhelium_ref_cpu_ops.so")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 and the built fhelium_b200 library")
    config.addinivalue_line("markers", "slow: long-running (full-size) case")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def ref_ops():
    """The reference's own CPU operators, compiled from its sources by
    oracle/build_ref.sh (absent where the reference sources never were)."""
    if not os.path.exists(REF_OPS):
        pytest.skip("reference CPU operators were not built (oracle/build_ref.sh)")
    import torch
    torch.ops.load_library(REF_OPS)
    return torch.ops
