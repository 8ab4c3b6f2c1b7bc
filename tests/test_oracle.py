"""The oracle itself: exact CRT permanent vs brute force / pure-Python Ryser,
reference restatements vs exact, closed forms."""
import math
from fractions import Fraction

import numpy as np
import pytest

from superman_b200 import workloads as W


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7])
def test_exact_matches_brute_force(oracle, n):
    a = W.dense_uniform(n, seed=n)
    want = oracle.brute_perm([[Fraction(v) for v in row] for row in a])
    assert oracle.exact_perm(a) == want


@pytest.mark.parametrize("n", [1, 3, 5, 8])
def test_exact_complex_matches_ryser(oracle, n):
    a = W.haar_block(n, seed=n, N=16)
    want = oracle.ryser_exact([[complex(v) for v in row] for row in a])
    er, ei = oracle.exact_perm_complex(a)
    assert abs(complex(float(er), float(ei)) - want) <= 1e-12 * max(1e-300, abs(want)) + 1e-15


@pytest.mark.parametrize("n", [1, 4, 9, 12])
def test_binary_u128_matches_ryser(oracle, n):
    b = W.binary_bernoulli(n, seed=n)
    assert oracle.binary_u128(b) == oracle.ryser_exact(b.astype(int).tolist())


@pytest.mark.parametrize("n", [2, 6, 11, 16])
def test_reference_restatement_close_to_exact(oracle, n):
    a = W.dense_uniform(n, seed=100 + n)
    ex = oracle.exact_perm(a)
    assert oracle.rel_err(oracle.dense_nw(a, threads=3), ex) < 1e-12
    assert oracle.rel_err(oracle.sparse_nw(a, threads=2), ex) < 1e-12


def test_closed_forms(oracle):
    for n, c in [(5, 0.91), (9, 0.5)]:
        want = math.factorial(n) * Fraction(c) ** n
        assert oracle.exact_perm(np.full((n, n), c)) == want
