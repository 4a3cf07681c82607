import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


@pytest.fixture(scope="session")
def built():
    """Builds (if stale) and loads the native library."""
    from flowcontrast_b200 import build
    build.build()
    import flowcontrast_b200 as fb
    fb.lib()
    return fb


@pytest.fixture(scope="session")
def ctx(built):
    c = built.Context(0)
    yield c
    c.close()
