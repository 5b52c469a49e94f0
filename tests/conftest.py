import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA path through the C ABI")
    config.addinivalue_line("markers", "slow: longer CPU test")


@pytest.fixture(scope="session")
def ref32():
    from oracle import ref32 as r

    r.lib()
    return r


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, loaded through the C ABI; fails (not skips) when the
    build is missing so that a GPU run never passes on a fallback."""
    import torch

    from mountainsort_b200 import _lib

    if not torch.cuda.is_available():
        pytest.fail("gpu test selected but no CUDA device is visible")
    torch.cuda.init()
    return _lib.load()
