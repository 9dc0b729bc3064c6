import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import __graft_entry__  # noqa: E402

PKG = __graft_entry__.load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def capi():
    return PKG.capi


@pytest.fixture(scope="session")
def runtime():
    return PKG.runtime


@pytest.fixture(scope="session")
def workloads():
    return PKG.workloads


@pytest.fixture(scope="session")
def orc():
    from oracle import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def gpu_lib():
    if not has_gpu():
        pytest.skip("no CUDA device")
    return PKG.capi.load_library()
