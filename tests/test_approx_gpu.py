"""Parity of the sampling permanent (spb_perm_approx, the reference's
approximation algorithm) with the oracle: every sample's estimate equal bit
for bit to the CPU restatement, and the mean within its sampling error of the
exact count."""
import ctypes
import math

import numpy as np
import pytest

from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu

# float draw probabilities (the reference's scaleType): relative offset of
# order n * 2^-24 on top of the sampling error
FLOAT_REL = 1e-6


def block_diag_pattern(blocks):
    n = sum(b.shape[0] for b in blocks)
    a = np.zeros((n, n), dtype=np.uint8)
    o = 0
    for b in blocks:
        m = b.shape[0]
        a[o:o + m, o:o + m] = b
        o += m
    return a


@pytest.mark.parametrize("name,first", [("bern12", 0), ("bern12", 123456), ("sparse40", 7), ("block70", 0)])
def test_samples_bit_exact_vs_oracle(spb, oracle, name, first):
    if name == "bern12":
        a = W.binary_bernoulli(12, 5)
    elif name == "sparse40":
        a = (W.sparse_perm_plus(40, 5) != 0).astype(np.uint8)
    else:  # n = 70 > 63, beyond the exact paths
        a = block_diag_pattern([W.binary_bernoulli(14, 20 + k, p=0.3) for k in range(5)])
    got = spb.approx_samples(a, first, 3000, seed=17)
    want = oracle.rasmussen_samples(a, first, 3000, seed=17)
    assert np.array_equal(got, want), np.flatnonzero(got != want)[:5]
    assert (got > 0).any()


@pytest.mark.parametrize("n,seed", [(12, 1), (16, 2), (20, 3)])
def test_mean_matches_exact(spb, oracle, n, seed):
    a = W.binary_bernoulli(n, seed)
    exact = oracle.binary_u128(a)
    r = spb.perm_approx(a, samples=1 << 20, seed=seed)
    se = r.err_est * abs(r.permanent)
    assert r.gray_steps == 1 << 20
    assert abs(r.permanent - exact) <= 5 * se + FLOAT_REL * exact, (r.permanent, se, exact)


def test_large_block_diagonal(spb, oracle):
    """n = 60: five 12 x 12 blocks; the exact count is the product."""
    blocks = [W.binary_bernoulli(12, 40 + k) for k in range(5)]
    exact = math.prod(oracle.binary_u128(b) for b in blocks)
    r = spb.perm_approx(block_diag_pattern(blocks), samples=1 << 20, seed=3)
    se = r.err_est * abs(r.permanent)
    assert abs(r.permanent - exact) <= 5 * se + FLOAT_REL * exact


def test_launch_shape_independent(spb):
    a = W.binary_bernoulli(14, 9)
    r1 = spb.perm_approx(a, samples=50_000, seed=4)
    r2 = spb.perm_approx(a, samples=50_000, seed=4, blocks=3)
    assert abs(r1.permanent - r2.permanent) <= 1e-12 * abs(r1.permanent)


def test_no_perfect_matching_is_zero(spb):
    a = np.ones((10, 10), dtype=np.uint8)
    a[:, 4] = 0
    assert spb.perm_approx(a, samples=10_000).permanent == 0.0


def test_bad_arguments(spb):
    from superman_b200 import _lib
    ip = ctypes.POINTER(ctypes.c_int)
    cp = np.array([0, 1, 3], dtype=np.int32)
    rw = np.array([0, 1, 5], dtype=np.int32)  # row 5 outside n = 2
    out = _lib.spb_result()
    L = _lib.lib()
    assert L.spb_perm_approx(cp.ctypes.data_as(ip), rw.ctypes.data_as(ip), 2, 100, 1, None,
                             ctypes.byref(out)) == _lib.SPB_ERR_INVALID
    assert L.spb_perm_approx(cp.ctypes.data_as(ip), rw.ctypes.data_as(ip), 2, 0, 1, None,
                             ctypes.byref(out)) == _lib.SPB_ERR_INVALID


def test_pipeline_approximation(spb, oracle, tmp_path):
    """algorithm=approximation through the reference-shaped pipeline (reader,
    pruning, components, selector, sampling driver)."""
    from superman_b200 import _lib
    a = W.binary_bernoulli(14, 31).astype(np.float64)
    exact = oracle.binary_u128(a.astype(np.uint8))
    args = [b"algorithm=approximation", b"approx_samples=400000", b"approx_seed=5"]
    arr = (ctypes.c_char_p * len(args))(*args)
    out = _lib.spb_pipeline_result()
    _lib.check(_lib.lib().spb_perm_pipeline(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 14, arr,
                                            len(args), ctypes.byref(out)))
    assert abs(out.permanent - exact) <= 0.02 * exact
