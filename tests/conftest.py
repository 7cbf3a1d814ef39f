"""Shared test setup: the `gpu` marker and in-tree builds of the library and oracle."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TESTS = os.path.dirname(os.path.abspath(__file__))
for _p in (ROOT, TESTS):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build libssmd.so and the oracle if they are missing or stale (CPU-only steps)."""
    from ssmdlbm_b200 import build as pbuild
    from oracle import build as obuild
    pbuild.build()
    obuild.build_oracle()
    obuild.build_oracle_gpu()
    yield
