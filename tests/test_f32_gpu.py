"""The FP32-product variant (SPB_PREC_FP32): error against the exact value
measured and bounded by kappa * n * 2^-24 terms, on the inputs it is offered
for."""
import numpy as np
import pytest

from superman_b200 import workloads as W
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [3, 5, 8, 13, 17, 20])
def test_f32_real_vs_exact(spb, oracle, n):
    a = W.dense_uniform(n, 600 + n)
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a, precision="fp32")
    err = oracle.rel_err(r.permanent, exact)
    # kappa <= ~1e2 for U[0,1) at n <= 20; a term carries ~n ulps of 2^-24
    assert err <= 1e2 * n * 2.0 ** -24, err


@pytest.mark.parametrize("name", ["complex_haar_n20_s9", "complex_haar_n28_s6"])
def test_f32_complex_haar_vs_exact(spb, oracle, name):
    a, exact, _ = load_golden(name)
    r = spb.perm_complex(a, precision="fp32")
    err = oracle.rel_err(r.permanent, exact)
    print(f"{name}: fp32-product rel err {err:.2e}")
    assert err <= 1e-5
    # it is the FP32 path: far from the FP64 walk's 1e-15 agreement
    r64 = spb.perm_complex(a, precision="fp64")
    assert oracle.rel_err(r64.permanent, exact) < err


def test_f32_size_limits(spb):
    with pytest.raises(spb.SupermanError):
        spb.perm_dense(np.ones((41, 41)), precision="fp32")
    with pytest.raises(spb.SupermanError):
        spb.perm_dense(np.ones((2, 2)), precision="fp32")


def test_f32_deterministic(spb):
    a = W.dense_uniform(24, 3)
    r1 = spb.perm_dense(a, precision="fp32")
    r2 = spb.perm_dense(a, precision="fp32")
    assert (r1.permanent, r1.permanent_lo) == (r2.permanent, r2.permanent_lo)
