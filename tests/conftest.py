import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG_DIR = os.path.join(ROOT, "cuppa-public_b200")
for p in (os.path.join(ROOT, "tests"), PKG_DIR):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def cuda_ok():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("this test needs a CUDA device")
    return True


@pytest.fixture(scope="session")
def pa():
    """The product binding; fails loudly when the library is missing."""
    import cuppa_b200
    cuppa_b200.lib()
    return cuppa_b200
