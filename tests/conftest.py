import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libccsd_b200.so")
    config.addinivalue_line("markers", "slow: long-running test")


@pytest.fixture(scope="session")
def built_lib():
    """Build (if needed) and load the shared library; host-only entry points work without a GPU."""
    from aquarius_b200 import build as b
    b.build()
    import aquarius_b200 as A
    return A.lib()
