"""Parity of the dense real / complex CUDA path (through the C ABI) with the
oracle: the exact CRT permanent and the reference-algorithm restatement."""
import numpy as np
import pytest

from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu

# FP64 products with double-double accumulation: relative error against the
# exact value.  At n <= 20 the cancellation factor of U[0,1) inputs is below
# ~1e2, so 1e-13 holds with margin.
REL_TOL_SMALL = 1e-13


@pytest.mark.parametrize("n", list(range(1, 21)))
def test_dense_uniform_small_exact(spb, oracle, n):
    a = W.dense_uniform(n, seed=1000 + n)
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a)
    assert oracle.rel_err(r.permanent, exact) <= REL_TOL_SMALL, (r.permanent, float(exact))


@pytest.mark.parametrize("n", [1, 2, 3, 5, 8, 13, 16])
def test_dense_signed_small_vs_brute(spb, oracle, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n))
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a)
    # signed entries cancel harder; compare against the magnitude of the terms
    scale = float(np.prod(np.abs(a).sum(axis=1)))
    assert abs(r.permanent - float(exact)) <= 1e-13 * scale


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 12, 16, 20])
def test_complex_haar_small_exact(spb, oracle, n):
    a = W.haar_block(n, seed=77 + n, N=64)
    er, ei = oracle.exact_perm_complex(a)
    r = spb.perm_complex(a)
    scale = float(np.prod(np.abs(a).sum(axis=1)))
    err = abs(r.permanent - complex(float(er), float(ei)))
    assert err <= 1e-13 * scale


@pytest.mark.parametrize("unit_bits,threads,blocks", [(2, 32, 1), (3, 64, 3), (5, 128, 7), (7, 96, 2)])
def test_dense_shape_invariance(spb, oracle, unit_bits, threads, blocks):
    a = W.dense_uniform(18, seed=5)
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a, unit_bits=unit_bits, threads_per_block=threads, blocks=blocks)
    assert oracle.rel_err(r.permanent, exact) <= REL_TOL_SMALL


@pytest.mark.parametrize("small_call", [0, -1])
@pytest.mark.parametrize("precision", ["fp64", "dd"])
@pytest.mark.parametrize("unit_bits", [9, 10])
def test_dense_wide_units(spb, oracle, unit_bits, precision, small_call):
    # Tables of 2^9 and 2^10 entries per row: every level above 32 entries
    # takes several passes of the setup kernel's per-row warp (small_call=-1
    # keeps the separate kernels; 2^10 does not fit the fused call anyway).
    a = W.dense_uniform(18, seed=6)
    exact = oracle.exact_perm(a)
    if precision == "dd" and unit_bits == 10:
        # both table words of 2^10 x 18 entries (295 KB) exceed the
        # refinement's shared memory: refused before any launch
        with pytest.raises(spb.SupermanError) as e:
            spb.perm_dense(a, precision=precision, unit_bits=unit_bits, small_call=small_call)
        assert "use fewer unit bits" in str(e.value)
        return
    r = spb.perm_dense(a, precision=precision, unit_bits=unit_bits, small_call=small_call)
    assert oracle.rel_err(r.permanent, exact) <= REL_TOL_SMALL


@pytest.mark.parametrize("unit_bits", [7, 8])
def test_complex_wide_units(spb, oracle, unit_bits):
    # (2^9 would need 2 parts x 2 words x 2^9 x 16 doubles, 262 KB, in the
    # refinement's shared memory: refused like the real case below)
    a = W.haar_block(16, seed=91, N=64)
    er, ei = oracle.exact_perm_complex(a)
    r = spb.perm_complex(a, precision="dd", unit_bits=unit_bits)
    scale = float(np.prod(np.abs(a).sum(axis=1)))
    assert abs(r.permanent - complex(float(er), float(ei))) <= 1e-13 * scale


def test_dense_unit_bits_too_wide(spb):
    # 2^14 table entries per row do not fit the walk's shared memory: a clean
    # error before any launch.
    a = W.dense_uniform(18, seed=7)
    with pytest.raises(spb.SupermanError) as e:
        spb.perm_dense(a, unit_bits=14)
    assert "shared memory" in str(e.value)


def test_dense_known_answers(spb):
    # perm(c J_n) = n! c^n  (ExampleMatrices/dense.mtx is 0.91 J_45)
    import math
    for n, c in [(10, 0.91), (16, 0.5), (21, 1.0)]:
        r = spb.perm_dense(np.full((n, n), c))
        want = math.factorial(n) * c ** n
        assert abs(r.permanent - want) <= 1e-12 * want
    # identity / permutation -> 1, diagonal -> product
    assert spb.perm_dense(np.eye(17)).permanent == 1.0
    p = np.eye(19)[np.random.default_rng(0).permutation(19)]
    assert spb.perm_dense(p).permanent == 1.0
    d = np.diag(np.arange(1.0, 15.0))
    assert spb.perm_dense(d).permanent == float(math.factorial(14))


def test_dense_n24_exact(spb, oracle):
    a = W.dense_uniform(24, seed=24)
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a)
    err = oracle.rel_err(r.permanent, exact)
    print("n=24 rel err", err)
    assert err <= 1e-12
