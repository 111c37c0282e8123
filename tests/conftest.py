import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    """Builds libhush_b200.so and the oracle if they are missing or stale (no-op on the GPU box, where the
    prebuilt files travel with the tree and no source is newer)."""
    from hush_b200 import build

    if not os.path.exists(build.LIB) or not os.path.exists(build.ORACLE_LIB) or os.environ.get("HUSH_REBUILD"):
        build.build()
    yield
