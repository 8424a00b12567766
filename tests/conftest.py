import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the engine through the C ABI")
    config.addinivalue_line("markers", "slow: full-size workloads")


@pytest.fixture(scope="session")
def engine():
    from rtspmspm_b200 import Engine

    e = Engine(0)
    yield e
    e.close()
