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


GOLDEN = os.path.join(ROOT, "tests", "golden")


def load_golden(name):
    """(matrix, exact, fixture) from tests/golden/<name>.json; exact is a
    Fraction, a (Fraction, Fraction) pair for complex inputs, or an int for
    0/1 inputs."""
    import json
    from fractions import Fraction

    import numpy as np
    g = json.load(open(os.path.join(GOLDEN, name + ".json")))
    n = g["n"]
    if g["kind"] == "complex":
        re = np.array([float.fromhex(h) for h in g["re_hex"]])
        im = np.array([float.fromhex(h) for h in g["im_hex"]])
        return (re + 1j * im).reshape(n, n), (Fraction(g["exact_re"]), Fraction(g["exact_im"])), g
    if g["kind"] == "binary":
        a = np.array([c == "1" for c in g["bits"]], dtype=np.uint8).reshape(n, n)
        return a, int(g["exact"]), g
    a = np.array([float.fromhex(h) for h in g["hex"]]).reshape(n, n)
    return a, Fraction(g["exact"]), g
