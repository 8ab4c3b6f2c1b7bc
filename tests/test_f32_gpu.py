"""The FP32-product variant (SPB_PREC_FP32): error against the exact value
measured and bounded by kappa * n * 2^-24 terms, on the inputs it is offered
for; the call's own error estimate covers the measured error, and a result
whose estimate exceeds the caller's bound (1e-12 unless rel_tol says
otherwise) comes back with SPB_ERR_ACCURACY."""
import numpy as np
import pytest

from superman_b200 import workloads as W
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [3, 5, 8, 13, 17, 20])
def test_f32_real_vs_exact(spb, oracle, n):
    a = W.dense_uniform(n, 600 + n)
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a, precision="fp32", rel_tol=1e-3)
    err = oracle.rel_err(r.permanent, exact)
    # kappa <= ~1e2 for U[0,1) at n <= 20; a term carries ~n ulps of 2^-24
    assert err <= 1e2 * n * 2.0 ** -24, err
    # the estimate is a statistical one: it covers the error with a margin
    assert 0 < r.err_est and err <= 10 * r.err_est, (err, r.err_est)


@pytest.mark.parametrize("name", ["complex_haar_n20_s9", "complex_haar_n28_s6"])
def test_f32_complex_haar_vs_exact(spb, oracle, name):
    a, exact, _ = load_golden(name)
    r = spb.perm_complex(a, precision="fp32", rel_tol=1e-4)
    err = oracle.rel_err(r.permanent, exact)
    print(f"{name}: fp32-product rel err {err:.2e}, estimate {r.err_est:.2e}")
    assert err <= 1e-5
    assert 0 < r.err_est and err <= 10 * r.err_est
    # it is the FP32 path: far from the FP64 walk's 1e-15 agreement
    r64 = spb.perm_complex(a, precision="fp64")
    assert oracle.rel_err(r64.permanent, exact) < err


def test_f32_size_limits(spb):
    from superman_b200 import _lib
    with pytest.raises(spb.SupermanError) as e:
        spb.perm_dense(np.ones((41, 41)), precision="fp32", rel_tol=1e-2)
    assert e.value.status == _lib.SPB_ERR_INVALID
    with pytest.raises(spb.SupermanError) as e:
        spb.perm_dense(np.ones((2, 2)), precision="fp32", rel_tol=1e-2)
    assert e.value.status == _lib.SPB_ERR_INVALID


def test_f32_deterministic(spb):
    a = W.dense_uniform(24, 3)
    r1 = spb.perm_dense(a, precision="fp32", rel_tol=1e-2)
    r2 = spb.perm_dense(a, precision="fp32", rel_tol=1e-2)
    assert (r1.permanent, r1.permanent_lo) == (r2.permanent, r2.permanent_lo)


def test_f32_refused_beyond_the_bound(spb):
    """Without rel_tol the bound is the library's 1e-12, which FP32 products
    cannot meet: the call returns SPB_ERR_ACCURACY with its result and its
    estimate filled in, so the caller can see why."""
    import ctypes
    from superman_b200 import _lib
    a, _, _ = load_golden("complex_haar_n20_s9")
    ri = np.ascontiguousarray(a).view(np.float64)
    out = _lib.spb_result()
    opt = _lib.default_options(precision=_lib.SPB_PREC_FP32)
    st = _lib.lib().spb_perm_dense_c128(ri.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 20,
                                        ctypes.byref(opt), ctypes.byref(out))
    assert st == _lib.SPB_ERR_ACCURACY and out.status == st
    assert out.err_est > 1e-12 and "exceeds the bound" in _lib.last_error()
    want = spb.perm_complex(a, precision="fp64").permanent
    assert abs(complex(out.value, out.imag) - want) <= 1e-5 * abs(want)
    with pytest.raises(spb.SupermanError) as e:
        spb.perm_dense(W.dense_uniform(16, 2), precision="fp32")
    assert e.value.status == _lib.SPB_ERR_ACCURACY
