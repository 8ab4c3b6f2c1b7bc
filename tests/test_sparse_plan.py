"""Host logic of the row-compacted sparse walk (CPU only): the plan
spb_perm_sparse_f64 would run — row and column orders, active rows, low
columns — checked for the properties the walk relies on."""
import ctypes

import numpy as np
import pytest

from superman_b200 import _lib
from superman_b200 import workloads as W

IP = ctypes.POINTER(ctypes.c_int)
DP = ctypes.POINTER(ctypes.c_double)


def plan(a, mode=0):
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    na, w = ctypes.c_int(), ctypes.c_int()
    ro, co = (ctypes.c_int * n)(), (ctypes.c_int * n)()
    assert _lib.lib().spb_sparse_plan(a.ctypes.data_as(DP), n, mode, ctypes.byref(na), ctypes.byref(w), ro, co) == 0
    return na.value, w.value, list(ro), list(co)


def check_plan(a, na, w, ro, co):
    n = a.shape[0]
    assert sorted(ro) == list(range(n)) and sorted(co) == list(range(n))
    if na == n:
        return
    assert 1 <= na < n and 2 <= w <= n - 2
    p = a[np.ix_(ro, co)]
    low = p[:, :w] != 0
    assert not low[na:].any(), "inactive rows must be zero in the low columns"
    assert low[:na].any(axis=1).all(), "every active row has a low-column nonzero"


@pytest.mark.parametrize("n,seed", [(20, 1), (24, 2), (30, 3), (40, 5), (63, 9)])
def test_plan_sparse_auto_compacts(n, seed):
    a = W.sparse_perm_plus(n, seed)
    na, w, ro, co = plan(a)
    check_plan(a, na, w, ro, co)
    assert na < n // 2, (n, na, w)


def test_plan_dense_keeps_dense_walk():
    a = W.dense_uniform(30, seed=4)
    na, w, ro, co = plan(a)
    assert na == 30 and ro == list(range(30)) and co == list(range(30))


def test_plan_modes():
    a = W.sparse_perm_plus(12, 3)
    assert plan(a, mode=0)[0] == 12          # below the automatic size
    assert plan(a, mode=1)[0] == 12          # never
    na, w, ro, co = plan(a, mode=2)          # always
    assert na < 12
    check_plan(a, na, w, ro, co)
    z = a.copy()
    z[:, 4] = 0.0                            # zero column: the dense walk (result 0)
    assert plan(z, mode=2)[0] == 12


def test_plan_pieces_of_sparse40():
    from test_host_pipeline import decompose
    for p in decompose(W.sparse_perm_plus(40, 5)):
        na, w, ro, co = plan(p)
        check_plan(p, na, w, ro, co)
        assert na < p.shape[0]


@pytest.mark.parametrize("seed", range(6))
def test_plan_permutation_keeps_permanent(oracle, seed):
    """The permuted matrix the walk sees has the same permanent (exact)."""
    a = W.sparse_perm_plus(9, 100 + seed, extra=2)
    na, w, ro, co = plan(a, mode=2)
    check_plan(a, na, w, ro, co)
    assert oracle.exact_perm(a[np.ix_(ro, co)]) == oracle.exact_perm(a)


def test_plan_rejects_bad_arguments():
    a = np.zeros((3, 3))
    na, w = ctypes.c_int(), ctypes.c_int()
    L = _lib.lib()
    assert L.spb_sparse_plan(a.ctypes.data_as(DP), 0, 0, ctypes.byref(na), ctypes.byref(w), None, None) != 0
    assert L.spb_sparse_plan(a.ctypes.data_as(DP), 64, 0, ctypes.byref(na), ctypes.byref(w), None, None) != 0


def test_plan_table_budget():
    """A block-diagonal matrix invites many low columns (they touch few rows);
    the plan keeps the low-column table within 64 KB (2^w * n doubles)."""
    a = np.zeros((30, 30))
    a[:14, :14] = W.dense_uniform(14, 13)
    a[14:, 14:] = W.dense_uniform(16, 14)
    na, w, ro, co = plan(a)
    check_plan(a, na, w, ro, co)
    assert (1 << w) * 30 * 8 <= 64 * 1024
