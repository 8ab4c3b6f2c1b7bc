"""CPU checks of the oracle's restatement of the reference's sampling
permanent (orc_rasmussen_*): unbiased against exact counts, exact on patterns
with a single perfect matching or none."""
import math

import numpy as np
import pytest

from superman_b200 import workloads as W


@pytest.mark.parametrize("n,seed", [(6, 1), (8, 2), (9, 3), (10, 4)])
def test_sampler_unbiased(oracle, n, seed):
    a = W.binary_bernoulli(n, seed)
    exact = oracle.binary_u128(a)
    est = oracle.rasmussen_samples(a, 0, 200_000, seed=11 + seed)
    se = est.std() / math.sqrt(est.size)
    assert abs(est.mean() - exact) <= 5 * se + FLOAT_REL * exact, (est.mean(), se, exact)


# The draw probabilities are floats (the reference's scaleType), so an
# estimate carries a relative offset of order n * 2^-24 besides its
# sampling error.
FLOAT_REL = 1e-6


def test_sampler_all_ones(oracle):
    n = 7
    est = oracle.rasmussen_samples(np.ones((n, n)), 0, 100_000, seed=5)
    se = est.std() / math.sqrt(est.size)
    assert abs(est.mean() - math.factorial(n)) <= 5 * se + FLOAT_REL * math.factorial(n)


def test_sampler_exact_cases(oracle):
    # one perfect matching: every sample is forced to it, estimate 1
    p = np.eye(9)[np.random.default_rng(3).permutation(9)]
    assert np.all(oracle.rasmussen_samples(p, 0, 100, seed=1) == 1.0)
    # upper triangular: a single matching too, but the scaling has not
    # converged onto it, so samples vary; their mean is 1
    est = oracle.rasmussen_samples(np.triu(np.ones((8, 8))), 0, 200_000, seed=2)
    assert abs(est.mean() - 1.0) <= 5 * est.std() / math.sqrt(est.size) + FLOAT_REL
    # a zero row: no perfect matching
    z = np.ones((6, 6))
    z[2] = 0
    assert np.all(oracle.rasmussen_samples(z, 0, 100, seed=3) == 0.0)


def test_sampler_streams_are_per_sample(oracle):
    """Sample k's estimate does not depend on which batch computes it."""
    a = W.binary_bernoulli(9, 7)
    whole = oracle.rasmussen_samples(a, 0, 64, seed=9)
    tail = oracle.rasmussen_samples(a, 40, 24, seed=9)
    assert np.array_equal(whole[40:], tail)
