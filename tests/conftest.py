import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path through the C ABI")


@pytest.fixture(scope="session")
def cuda():
    """Skips when no CUDA device is visible; on a GPU machine the library must load (no fallback)."""
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from ttm_b200 import _lib
    _lib.lib()
    return torch.device("cuda", 0)


@pytest.fixture(scope="session")
def oracle_c():
    from oracle import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def reference():
    from oracle import Reference, REF_SO
    if not os.path.exists(REF_SO):
        pytest.skip("reference build (oracle/_ref) not available")
    try:
        return Reference()
    except OSError as e:
        pytest.skip(f"reference build not loadable here: {e}")
