"""Parity of the sparse entry point spb_perm_sparse_f64 (row-compacted walk)
with the oracle: exact CRT permanents, and the exact n=40 sparse fixture
through its decomposition pieces."""
import numpy as np
import pytest

from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu


def csc(a):
    n = a.shape[0]
    cptrs, rows, vals = [0], [], []
    for c in range(n):
        for r in range(n):
            if a[r, c] != 0:
                rows.append(r)
                vals.append(a[r, c])
        cptrs.append(len(rows))
    return np.array(cptrs), np.array(rows), np.array(vals)


@pytest.mark.parametrize("n", [4, 5, 7, 10, 13, 16])
def test_sparse_forced_small_exact(spb, oracle, n):
    a = W.sparse_perm_plus(n, 300 + n, extra=2)
    exact = oracle.exact_perm(a)
    r = spb.perm_sparse(a, walk="always")
    assert r.active_rows < n
    assert oracle.rel_err(r.permanent, exact) <= 1e-13, (r.permanent, float(exact))


@pytest.mark.parametrize("n,seed", [(20, 1), (22, 2), (24, 3)])
@pytest.mark.parametrize("precision", ["fp64", "dd"])
def test_sparse_auto_exact(spb, oracle, n, seed, precision):
    a = W.sparse_perm_plus(n, seed)
    exact = oracle.exact_perm(a)
    r = spb.perm_sparse(a, precision=precision)
    assert r.active_rows < n
    assert oracle.rel_err(r.permanent, exact) <= 1e-13


def test_sparse_walks_agree_signed(spb, oracle):
    """Signed values: the compacted and the dense walk both match the exact
    value to the terms' magnitude."""
    a = W.sparse_perm_plus(22, 8)
    rng = np.random.default_rng(8)
    a = a * np.where(rng.random(a.shape) < 0.5, -1.0, 1.0)
    exact = float(oracle.exact_perm(a))
    scale = float(np.prod(np.abs(a).sum(axis=1)))
    rc = spb.perm_sparse(a, walk="always")
    rd = spb.perm_sparse(a, walk="never")
    assert rc.active_rows < 22 and rd.active_rows == 22
    assert abs(rc.permanent - exact) <= 1e-14 * scale
    assert abs(rd.permanent - exact) <= 1e-14 * scale


def test_sparse_dd_refinement_signed(spb, oracle):
    """A tight tolerance sends units of the compacted walk through the
    double-double refinement; the result stays exact to the tolerance."""
    a = W.sparse_perm_plus(22, 9, extra=4)
    rng = np.random.default_rng(9)
    a = a * np.where(rng.random(a.shape) < 0.5, -1.0, 1.0)
    exact = oracle.exact_perm(a)
    r = spb.perm_sparse(a, precision="dd", rel_tol=1e-15, walk="always")
    assert r.active_rows < 22 and r.refined_units > 0
    assert oracle.rel_err(r.permanent, exact) <= 1e-12
    # the replay scan (the walk's own unit bases) selects the same units
    r2 = spb.perm_sparse(a, precision="dd", rel_tol=1e-15, walk="always", replay_listing=1)
    assert r2.refined_units == r.refined_units
    assert oracle.rel_err(r2.permanent, exact) <= 1e-12


def test_sparse_csc_input_matches_dense_input(spb):
    a = W.sparse_perm_plus(24, 11)
    r1 = spb.perm_sparse(a)
    r2 = spb.perm_sparse(csc(a))
    assert (r1.permanent, r1.permanent_lo) == (r2.permanent, r2.permanent_lo)


def test_sparse_deterministic_and_shape_invariant(spb, oracle):
    a = W.sparse_perm_plus(23, 12)
    exact = oracle.exact_perm(a)
    r1 = spb.perm_sparse(a)
    r2 = spb.perm_sparse(a)
    assert (r1.permanent, r1.permanent_lo) == (r2.permanent, r2.permanent_lo)
    for threads, blocks in [(64, 3), (160, 11)]:
        r = spb.perm_sparse(a, threads_per_block=threads, blocks=blocks)
        assert oracle.rel_err(r.permanent, exact) <= 1e-13


def test_sparse_n40_pieces_sum_to_exact(spb, oracle):
    """The decomposition pieces of the n=40 fixture, each on the compacted
    walk, sum to its exact permanent."""
    from conftest import load_golden
    from test_host_pipeline import decompose
    a, exact, _ = load_golden("sparse_n40_s5")
    total = 0.0
    for p in decompose(a):
        r = spb.perm_sparse(p, precision="dd")
        assert r.active_rows < p.shape[0]
        total += r.permanent + r.permanent_lo
    assert oracle.rel_err(total, exact) <= 1e-13


def test_sparse_zero_column(spb):
    """A zero column makes the permanent 0; the dense walk then runs and its
    terms cancel to rounding level."""
    a = W.sparse_perm_plus(21, 4)
    a[:, 7] = 0.0
    r = spb.perm_sparse(a)
    assert r.active_rows == 21
    assert abs(r.permanent) <= 1e-15 * float(np.prod(np.abs(a).sum(axis=1)))


def test_sparse_bad_arguments(spb):
    import ctypes
    from superman_b200 import _lib
    cp, rw, vl = csc(W.sparse_perm_plus(6, 1))
    bad = cp.copy()
    bad[3], bad[4] = bad[4], bad[3] - 1  # decreasing pointers
    with pytest.raises(spb.SupermanError):
        spb.perm_sparse((bad, rw, vl))
    rw2 = rw.copy()
    rw2[0] = 9
    with pytest.raises(spb.SupermanError):
        spb.perm_sparse((cp, rw2, vl))
    with pytest.raises(spb.SupermanError):
        spb.perm_sparse((np.array([0]), rw, vl))
