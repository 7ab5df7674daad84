import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libdagegpu.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def dage():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from dage_b200 import build

    build.build()
    import dage_b200

    dage_b200.load()
    return dage_b200


@pytest.fixture(scope="session")
def dage_host():
    """The package with its library loaded, for host-only entry points
    (no GPU call)."""
    from dage_b200 import build

    build.build()
    import dage_b200

    dage_b200.load()
    return dage_b200
