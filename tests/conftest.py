import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwq3d.so")


@pytest.fixture(scope="session")
def engine():
    """The CUDA engine library; GPU tests fail loudly if it is missing."""
    import underseamodelinglibrary_b200 as u
    lib = u.load_engine()
    import ctypes
    n = ctypes.c_int()
    rc = lib.wq3d_device_count(ctypes.byref(n))
    assert rc == 0 and n.value > 0, "no CUDA device visible to libwq3d"
    return lib
