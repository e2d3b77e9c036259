import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) device")


@pytest.fixture(scope="session")
def ctx():
    """One cfdb context for the GPU tests (fails loudly without the library)."""
    from cfdapp_b200 import cfdb
    c = cfdb.Context(0)
    yield c
    c.close()
