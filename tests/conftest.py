import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line('markers', 'gpu: needs a CUDA device (B200, sm_100a)')
    config.addinivalue_line('markers', 'reference: needs the reference source tree')


@pytest.fixture(scope='session')
def oracle():
    from oracle import oracle as O
    O.build_lib()
    return O


@pytest.fixture
def host_only(monkeypatch):
    """Replaces the device kernels by CPU stand-ins (tests/fake_device.py) to
    test host-side logic without a GPU."""
    import fake_device
    fake_device.install(monkeypatch)
    yield


@pytest.fixture(scope='session')
def tb():
    """The product package with its CUDA library loaded (GPU tests only)."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail('CUDA device required for -m gpu tests')
    import tractor_b200
    from tractor_b200 import _lib, build
    build.build()
    _lib.load()
    return tractor_b200
