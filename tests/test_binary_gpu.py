"""Exact 0/1 permanent (spb_perm_binary) through the C ABI: bit-exact against
the oracle's int128 Ryser and pure-Python Ryser, the committed n=30 fixture,
closed forms that need more than 128 bits, and self-consistency at n=36."""
import math

import numpy as np
import pytest

from conftest import load_golden
from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", list(range(1, 23)))
def test_binary_small_bit_exact(spb, oracle, n):
    a = W.binary_bernoulli(n, seed=300 + n)
    got = spb.perm_binary(a).permanent
    assert got == oracle.binary_u128(a)
    if n <= 12:
        assert got == oracle.ryser_exact(a.astype(int).tolist())


@pytest.mark.parametrize("n", [5, 11, 17])
def test_binary_sparse_and_zero_rows(spb, oracle, n):
    a = (W.uniform(n, n * n).reshape(n, n) < 0.2).astype(np.uint8)
    assert spb.perm_binary(a).permanent == oracle.binary_u128(a)
    a[n // 2, :] = 0  # an empty row: permanent 0
    assert spb.perm_binary(a).permanent == 0


def test_binary_golden_n30(spb, oracle):
    a, exact, g = load_golden("binary_n30_s4")
    r = spb.perm_binary(a)
    assert r.permanent == exact
    # the reference's FP64 result on the same pattern is only close
    ref = float(g["reference"]["value"])
    assert abs(ref - exact) / exact < 1e-8


@pytest.mark.parametrize("n", [10, 21, 33, 34])
def test_binary_all_ones_factorial(spb, n):
    # n! needs 192-bit arithmetic from n = 34 on (34! > 2^127)
    assert spb.perm_binary(np.ones((n, n), dtype=np.uint8)).permanent == math.factorial(n)


def test_binary_identity_and_permutation(spb):
    for n in (1, 2, 7, 40):
        p = np.eye(n, dtype=np.uint8)[np.random.default_rng(n).permutation(n)]
        assert spb.perm_binary(p).permanent == 1


def test_binary_n36_self_consistent(spb):
    """Config C2 (n=36, Bernoulli(0.5) with the identity OR-ed in): the exact
    result must not depend on the launch shape, the row/column order or
    transposition."""
    a = W.binary_bernoulli(36, seed=4)
    base = spb.perm_binary(a).permanent
    assert base > 0
    assert spb.perm_binary(a, unit_bits=5, threads_per_block=256, blocks=97).permanent == base
    rng = np.random.default_rng(36)
    assert spb.perm_binary(a[rng.permutation(36)][:, rng.permutation(36)]).permanent == base
    assert spb.perm_binary(a.T.copy()).permanent == base
