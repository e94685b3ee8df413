"""Shared test setup: import paths, the `gpu` marker and the device context."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tpt-fem_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libtptfem.so")


@pytest.fixture(scope="session")
def ctx():
    import tpt_fem
    return tpt_fem.Context.default(0)
