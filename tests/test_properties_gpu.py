"""Size-independent properties of the permanent at sizes the exact oracle
cannot reach in seconds (n = 24..32), through the C ABI; and the library's
behaviour under injected allocation failures (host-side; no GPU fault)."""
import math

import numpy as np
import pytest

from superman_b200 import _lib
from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu


def rel(a, b):
    return abs(a - b) / abs(b)


def full(r):
    return r.permanent + r.permanent_lo


def test_transpose_invariance_n32(spb):
    a = W.dense_uniform(32, 7)
    r1 = spb.perm_dense(a, precision="dd")
    r2 = spb.perm_dense(np.ascontiguousarray(a.T), precision="dd")
    assert rel(full(r2), full(r1)) <= 3e-13


def test_permutation_invariance_n30(spb):
    a = W.dense_uniform(30, 8)
    rng = np.random.default_rng(8)
    b = a[rng.permutation(30)][:, rng.permutation(30)]
    r1 = spb.perm_dense(a, precision="dd")
    r2 = spb.perm_dense(np.ascontiguousarray(b), precision="dd")
    assert rel(full(r2), full(r1)) <= 3e-13


def test_power_of_two_row_scaling_is_exact_n28(spb):
    """Rows are normalised by exact powers of two, so scaling a row by 2^k
    scales the result by exactly 2^k (both words of the double-double)."""
    a = W.dense_uniform(28, 9)
    b = a.copy()
    b[3] *= 2.0 ** 40
    b[17] *= 2.0 ** -25
    for prec in ("fp64", "dd"):
        r1 = spb.perm_dense(a, precision=prec)
        r2 = spb.perm_dense(b, precision=prec)
        assert r2.permanent == math.ldexp(r1.permanent, 15)
        assert r2.permanent_lo == math.ldexp(r1.permanent_lo, 15)


def test_row_linearity_n24(spb):
    a = W.dense_uniform(24, 10)
    u, v = W.dense_uniform(24, 11)[0], W.dense_uniform(24, 12)[0]
    au, av, aw = a.copy(), a.copy(), a.copy()
    au[5], av[5], aw[5] = u, v, 0.75 * u + 1.25 * v
    pu, pv, pw = (full(spb.perm_dense(x, precision="dd")) for x in (au, av, aw))
    assert rel(pw, 0.75 * pu + 1.25 * pv) <= 1e-13


def test_block_diagonal_product_n30(spb):
    b1, b2 = W.dense_uniform(14, 13), W.dense_uniform(16, 14)
    a = np.zeros((30, 30))
    a[:14, :14], a[14:, 14:] = b1, b2
    prod = full(spb.perm_dense(b1, precision="dd")) * full(spb.perm_dense(b2, precision="dd"))
    # Ryser's sum cancels hard on a block-diagonal matrix; rel_tol is the
    # statistical target of the refinement, the bar is 1e-12
    whole = spb.perm_dense(a, precision="dd")
    assert rel(full(whole), prod) <= 1e-12
    tight = spb.perm_dense(a, precision="dd", rel_tol=1e-15)
    assert tight.refined_units >= whole.refined_units
    assert rel(full(tight), prod) <= 1e-13


def test_complex_conjugation_n24(spb):
    """perm(conj A) = conj perm(A)."""
    c = W.haar_block(24, 15)
    r1 = spb.perm_complex(c, precision="dd")
    r2 = spb.perm_complex(np.conj(c), precision="dd")
    assert abs(r2.permanent - np.conj(r1.permanent)) <= 1e-13 * abs(r1.permanent)


def test_complex_two_term_groups_n34(spb):
    """n = 34 complex runs the two-term groups (n > 32).  perm(A^T) = perm(A);
    a row times i gives i perm(A) (exact in the input); a row times 2 gives
    exactly twice the result (rows are pre-scaled by powers of two, so the
    walk sees the same matrix)."""
    a = W.haar_block(34, 21)
    r1 = spb.perm_complex(a, precision="dd").permanent
    r2 = spb.perm_complex(np.ascontiguousarray(a.T), precision="dd").permanent
    assert abs(r2 - r1) <= 1e-11 * abs(r1)
    b = a.copy()
    b[5] *= 1j
    r3 = spb.perm_complex(b, precision="dd").permanent
    assert abs(r3 - 1j * r1) <= 1e-11 * abs(r1)
    b = a.copy()
    b[9] *= 2.0
    assert spb.perm_complex(b, precision="dd").permanent == 2.0 * r1


def test_injected_allocation_failure_and_recovery(spb):
    L = _lib.lib()
    a = W.dense_uniform(20, 16)
    want = spb.perm_dense(a).permanent
    L.spb_debug_fail_allocations(1)
    with pytest.raises(spb.SupermanError) as e:
        spb.perm_dense(a)
    assert e.value.status == _lib.SPB_ERR_OOM and "injected" in _lib.last_error()
    assert spb.perm_dense(a).permanent == want  # the next call works
    # the double-double mode's second allocation (its refinement list)
    s = np.random.default_rng(3).standard_normal((18, 18))
    want_dd = spb.perm_dense(s, precision="dd", rel_tol=1e-15)
    assert want_dd.refined_units > 0
    L.spb_debug_fail_allocations(2)
    try:
        with pytest.raises(spb.SupermanError) as e:
            spb.perm_dense(s, precision="dd", rel_tol=1e-15)
        assert e.value.status == _lib.SPB_ERR_OOM
    finally:
        L.spb_debug_fail_allocations(0)
    assert full(spb.perm_dense(s, precision="dd", rel_tol=1e-15)) == full(want_dd)


def test_injected_failure_in_server_create(spb):
    from superman_b200.serving import Server
    L = _lib.lib()
    L.spb_debug_fail_allocations(1)
    try:
        with pytest.raises(spb.SupermanError) as e:
            Server()
        assert e.value.status == _lib.SPB_ERR_OOM
    finally:
        L.spb_debug_fail_allocations(0)
    with Server() as srv:  # a later server starts normally
        a = W.dense_uniform(10, 1)
        got = srv.wait(srv.submit(a))["permanent"]
        assert abs(got - spb.perm_dense(a).permanent) <= 1e-13 * abs(got)


def test_edge_values(spb):
    """Zeros give exactly 0; a permanent beyond the double range comes back
    infinite and a NaN entry gives NaN (the reference prints such results as
    'overflowed', main.cpp:122-125); rows are scaled by powers of two, so
    entries near the range limits alone do not overflow the walk."""
    assert spb.perm_dense(np.zeros((12, 12))).permanent == 0.0
    z = W.dense_uniform(22, 5)
    z[7] = 0.0
    assert spb.perm_dense(z).permanent == 0.0
    big = np.full((20, 20), 1e300)
    assert np.isinf(spb.perm_dense(big).permanent)
    tiny = np.full((12, 12), 1e-300)  # 12! * 1e-3600 underflows to 0
    assert spb.perm_dense(tiny).permanent == 0.0
    # rows at 2^900 and 2^-900 whose scales cancel: the result is in range
    scaled = np.full((12, 12), 0.75)
    scaled[:6] *= 2.0 ** 900
    scaled[6:] *= 2.0 ** -900
    r = spb.perm_dense(scaled)
    assert abs(r.permanent - math.factorial(12) * 0.75 ** 12) <= 1e-13 * r.permanent
    nan = W.dense_uniform(10, 6)
    nan[3, 4] = np.nan
    assert np.isnan(spb.perm_dense(nan).permanent)
