"""Full-size configurations against the committed exact fixtures
(tests/golden/*.json, made by tests/golden/make_golden.py with the exact CRT
oracle and the reference CPU binary)."""
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

# The accuracy bar for the real/complex paths: relative error against the
# exact rational permanent.
REL_TOL_DD = 1e-12


@pytest.mark.parametrize("name", ["dense_u01_n24_s3", "dense_u01_n32_s7"])
def test_dense_golden_dd(spb, oracle, name):
    a, exact, g = load_golden(name)
    r = spb.perm_dense(a, precision="dd")
    err = oracle.rel_err(r.permanent, exact)
    print(f"{name}: dd rel err {err:.3e}, refined units {r.refined_units}, "
          f"est {r.err_est:.2e}, kernel {r.kernel_s * 1e3:.2f} ms")
    assert err <= REL_TOL_DD
    # The reference CPU result on the same matrix (pinned to the exact value
    # within its own error in test_golden_pins.py) is further from exact.
    ref = g.get("reference")
    if ref:
        assert oracle.rel_err(float(ref["value"]), exact) >= err


@pytest.mark.parametrize("name", ["dense_u01_n24_s3", "dense_u01_n32_s7"])
def test_dense_golden_fp64(spb, oracle, name):
    a, exact, _ = load_golden(name)
    r = spb.perm_dense(a, precision="fp64")
    err = oracle.rel_err(r.permanent, exact)
    print(f"{name}: fp64 rel err {err:.3e}")
    # FP64 products: ~kappa * sqrt(n/6) * 2^-52 (about 3e-12 at n=32)
    assert err <= 2e-11


@pytest.mark.parametrize("name", ["complex_haar_n20_s9", "complex_haar_n28_s6"])
def test_complex_golden(spb, oracle, name):
    a, exact, g = load_golden(name)
    ref = g.get("reference")
    ref_err = oracle.rel_err(complex(float(ref["value_re"]), float(ref["value_im"])), exact) if ref else None
    for prec in ("fp64", "dd"):
        r = spb.perm_complex(a, precision=prec)
        err = oracle.rel_err(r.permanent, exact)
        print(f"{name}: {prec} rel err {err:.3e} refined {r.refined_units} est {r.err_est:.2e} "
              f"(reference CPU {ref_err})")
        assert err <= REL_TOL_DD
        if ref_err is not None:
            assert err <= ref_err


@pytest.mark.parametrize("n", [3, 9, 17, 22])
def test_dd_small_exact(spb, oracle, n):
    from superman_b200 import workloads as W
    a = W.dense_uniform(n, seed=50 + n)
    r = spb.perm_dense(a, precision="dd")
    assert oracle.rel_err(r.permanent, oracle.exact_perm(a)) <= 1e-13
    c = W.haar_block(n, seed=50 + n, N=64)
    rc = spb.perm_complex(c, precision="dd")
    assert oracle.rel_err(rc.permanent, oracle.exact_perm_complex(c)) <= 1e-12


def test_dd_forced_refinement_signed(spb, oracle):
    """A tight tolerance forces many units through the double-double path on
    a signed matrix; the result must stay exact to the tolerance."""
    import numpy as np
    rng = np.random.default_rng(7)
    a = rng.standard_normal((20, 20))
    exact = oracle.exact_perm(a)
    r = spb.perm_dense(a, precision="dd", rel_tol=1e-15)
    assert r.refined_units > 0
    assert oracle.rel_err(r.permanent, exact) <= 1e-12


@pytest.mark.parametrize("name", ["dense_u01_n24_s3", "dense_u01_n32_s7"])
def test_dd_listing_paths_agree(spb, oracle, name):
    """The first pass's unit list and the replay scan select the same units;
    the results agree to far below the tolerance."""
    a, exact, _ = load_golden(name)
    r1 = spb.perm_dense(a, precision="dd")
    r2 = spb.perm_dense(a, precision="dd", replay_listing=1)
    assert r1.refined_units == r2.refined_units
    assert r2.launches > 0 and oracle.rel_err(r2.permanent, exact) <= REL_TOL_DD
    assert abs((r1.permanent + r1.permanent_lo) - (r2.permanent + r2.permanent_lo)) <= 1e-15 * abs(r1.permanent)


def test_dd_parallel_scan_signed(spb, oracle):
    """Many units to refine (tight tolerance, signed entries): the threshold
    falls below the first pass's list, so the parallel scan lists them; the
    replay scan must select the same units."""
    import numpy as np
    rng = np.random.default_rng(21)
    a = rng.standard_normal((22, 22))
    exact = oracle.exact_perm(a)
    r1 = spb.perm_dense(a, precision="dd", rel_tol=1e-16)
    r2 = spb.perm_dense(a, precision="dd", rel_tol=1e-16, replay_listing=1)
    assert r1.refined_units == r2.refined_units > 0
    assert oracle.rel_err(r1.permanent, exact) <= 1e-12
    assert oracle.rel_err(r2.permanent, exact) <= 1e-12
