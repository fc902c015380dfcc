import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
sys.path.insert(0, REPO)
sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def product_lib():
    """Build (if stale) and load libflexrt_b200.so from the package tree."""
    from flexrt_imaging_reion_b200 import build, _abi
    build.build()
    return _abi.lib()


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import oracle as O
    return O.lib()
