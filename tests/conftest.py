"""Shared pytest configuration.

`-m gpu` tests need a CUDA device and call the library through its C ABI;
everything else runs on the CPU (oracle checks, host logic, ABI exports).
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def spb():
    import superman_b200 as S
    if S.device_count() < 1:
        pytest.fail("no CUDA device visible to libsupb200.so")
    return S
