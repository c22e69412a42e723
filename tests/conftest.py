import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "splatt-stream_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def gpu_available():
    try:
        import splatt_b200 as sb
        lib = sb.Lib(64)
        return lib.L.splatt_b200_init(0) == sb.SPLATT_SUCCESS
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib64():
    import splatt_b200 as sb
    lib = sb.Lib(64)
    lib.init(0)
    return lib


@pytest.fixture(scope="session")
def lib32():
    import splatt_b200 as sb
    lib = sb.Lib(32)
    lib.init(0)
    return lib


@pytest.fixture(scope="session")
def port():
    from oracles import Port
    return Port()
