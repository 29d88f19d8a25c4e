"""Test configuration: import paths and the `gpu` marker.

`-m "not gpu"` runs on any host (oracle, host logic, library loading and
exports); `-m gpu` runs the parity tests on a B200 through the C ABI.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "turbo-octo-spice_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) and runs the CUDA engine")


@pytest.fixture(scope="session")
def engine():
    from tos_b200 import Engine
    eng = Engine(0)
    yield eng
    eng.close()
