import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libbgk3d.so")
    config.addinivalue_line("markers", "slow: longer-running test")


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def bgk():
    """The product package with its CUDA library built and loaded."""
    import bgk3d_hit_b200 as B
    from bgk3d_hit_b200 import build

    build.build()
    B.load()
    return B
