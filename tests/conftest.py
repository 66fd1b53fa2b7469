import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100a GPU (B200)")


@pytest.fixture(scope="session")
def built_lib():
    """Builds libscft_b200.so in-tree if it is missing or stale (nvcc cross-compiles)."""
    from scft_string_b200 import build
    return build.build()
