"""Host-side C++ layer through the C ABI, on the CPU (no GPU calls):
the .mtx reader, perfect-matching pruning and DecomposePerman."""
import ctypes
import math
import os
from fractions import Fraction

import numpy as np
import pytest

from superman_b200 import _lib
from superman_b200 import workloads as W

DP = ctypes.POINTER(ctypes.c_double)


def read(path, binary=False, undirected=False, complex_=False, max_n=64):
    L = _lib.lib()
    n = ctypes.c_int()
    sp = ctypes.c_double()
    out = np.zeros(max_n * max_n * (2 if complex_ else 1))
    st = L.spb_read_matrix(path.encode(), int(binary), int(undirected), int(complex_),
                           out.ctypes.data_as(DP), max_n, ctypes.byref(n), ctypes.byref(sp))
    if st != 0:
        return st, None, None
    k = n.value
    a = out[: k * k * (2 if complex_ else 1)]
    a = a.view(np.complex128).reshape(k, k) if complex_ else a.reshape(k, k)
    return st, a.copy(), sp.value


def test_reader_mtx_one_based_and_comments(tmp_path):
    p = tmp_path / "m.mtx"
    p.write_text("%%MatrixMarket matrix coordinate real general\n% comment\n3 3 4\n1 1 2.5\n2 3 -1\n3 2 4\n1 2 0\n")
    st, a, sp = read(str(p))
    assert st == 0
    want = np.array([[2.5, 0, 0], [0, 0, -1], [0, 4, 0]])
    assert np.array_equal(a, want)
    assert sp == pytest.approx(100 * 3 / 9)


def test_reader_zero_based_binary_undirected(tmp_path):
    p = tmp_path / "m.txt"  # not .mtx: 0-based indices
    p.write_text("3 3 3\n0 1\n1 2\n0 0\n")
    st, a, _ = read(str(p), binary=True, undirected=True)
    assert st == 0
    # mirrored entries, all 1; then pruning keeps only entries on perfect matchings
    full = np.array([[1, 1, 0], [1, 0, 1], [0, 1, 0]], dtype=float)
    assert a[2, 1] == 1 and a[1, 2] == 1
    assert np.all((a == 0) | (full == 1))


def test_reader_errors(tmp_path):
    L = _lib.lib()
    p = tmp_path / "ns.mtx"
    p.write_text("3 4 1\n1 1 1\n")
    assert read(str(p))[0] == _lib.SPB_ERR_NOT_SQUARE
    assert "not square" in _lib.last_error()
    q = tmp_path / "oob.mtx"
    q.write_text("2 2 1\n3 1 1\n")
    assert read(str(q))[0] == _lib.SPB_ERR_IO
    assert read(str(tmp_path / "missing.mtx"))[0] == _lib.SPB_ERR_IO
    assert "could not be opened" in _lib.last_error()
    del L


def test_reader_complex(tmp_path):
    p = tmp_path / "c.mtx"
    p.write_text("2 2 3\n1 1 0 1\n1 2 2 0\n2 2 1 -1\n")
    st, a, _ = read(str(p), complex_=True)
    assert st == 0
    assert np.array_equal(a, np.array([[1j, 2], [0, 1 - 1j]]))


def prune(a):
    L = _lib.lib()
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros_like(a)
    ok = ctypes.c_int()
    assert L.spb_dm_prune(a.ctypes.data_as(DP), a.shape[0], out.ctypes.data_as(DP), ctypes.byref(ok)) == 0
    return out, ok.value


@pytest.mark.parametrize("seed", range(6))
def test_dm_prune_keeps_permanent(oracle, seed):
    n = 9
    rng = np.random.default_rng(seed)
    a = (rng.random((n, n)) < 0.3) * rng.integers(1, 5, (n, n)).astype(float)
    a += np.eye(n)[rng.permutation(n)]  # guarantees a perfect matching
    pr, ok = prune(a)
    assert ok == 1
    assert np.all((pr == 0) | (pr == a))
    assert oracle.exact_perm(pr) == oracle.exact_perm(a)
    # every kept entry lies on a perfect matching: removing it changes the permanent
    for (i, j) in zip(*np.nonzero(pr)):
        b = pr.copy()
        b[i, j] = 0
        assert oracle.exact_perm(b) != oracle.exact_perm(pr)


def test_dm_prune_structurally_singular():
    a = np.zeros((4, 4))
    a[0, :] = 1
    a[1, 0] = a[2, 0] = a[3, 0] = 1  # rows 1-3 all need column 0
    pr, ok = prune(a)
    assert ok == 0 and not pr.any()


# ----------------------------------------------------------- decomposition --

def band_perm(a, b):
    """Exact permanent of a matrix whose nonzeros satisfy |i - j| <= b, by DP
    over rows with the used columns of the window as state."""
    n = len(a)
    states = {0: Fraction(1)}  # bitmask over columns i-b .. i+b (bit k <-> column i-b+k)
    for i in range(n):
        nxt = {}
        for mask, v in states.items():
            for k in range(2 * b + 1):
                j = i - b + k
                if j < 0 or j >= n or (mask >> k) & 1 or a[i][j] == 0:
                    continue
                m2 = mask | (1 << k)
                if (m2 & 1) == 0 and i - b >= 0:
                    continue  # column i-b would never be used again
                nm = m2 >> 1
                nxt[nm] = nxt.get(nm, Fraction(0)) + v * Fraction(a[i][j])
        states = nxt
    return sum(states.values(), Fraction(0))


def decompose(a):
    L = _lib.lib()
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    cnt = ctypes.c_int()
    assert L.spb_decompose(a.ctypes.data_as(DP), n, ctypes.byref(cnt), None, None, 0, 0) == 0
    sizes = (ctypes.c_int * max(1, cnt.value))()
    data = np.zeros(max(1, cnt.value * n * n))
    assert L.spb_decompose(a.ctypes.data_as(DP), n, ctypes.byref(cnt), sizes, data.ctypes.data_as(DP),
                           cnt.value, data.size) == 0
    out, off = [], 0
    for k in range(cnt.value):
        m = sizes[k]
        out.append(data[off: off + m * m].reshape(m, m))
        off += m * m
    return out


def perm_any(p):
    """Exact permanent of a piece: band DP on its bandwidth."""
    nz = np.nonzero(p)
    b = int(np.max(np.abs(nz[0] - nz[1]))) if len(nz[0]) else 0
    assert b <= 6, b
    return band_perm(p.tolist(), max(b, 0))


@pytest.mark.parametrize("n,b,seed", [(34, 1, 1), (36, 1, 2), (33, 2, 3)])
def test_decompose_sum_of_pieces(n, b, seed):
    rng = np.random.default_rng(seed)
    a = np.zeros((n, n))
    for i in range(n):
        for j in range(max(0, i - b), min(n, i + b + 1)):
            if i == j or rng.random() < 0.7:
                a[i, j] = float(rng.integers(1, 4))
    pieces = decompose(a)
    assert pieces and all(p.shape[0] <= 30 for p in pieces)
    total = sum((perm_any(p) for p in pieces), Fraction(0))
    assert total == band_perm(a.tolist(), b)


def test_decompose_small_is_one_piece():
    a = W.dense_uniform(12, 1)
    pieces = decompose(a)
    assert len(pieces) == 1 and np.array_equal(pieces[0], a)


# ---------------------------------------------------------------- orderings --
def reorder(a, order, param=0):
    L = _lib.lib()
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = np.zeros_like(a)
    st = L.spb_reorder(a.ctypes.data_as(DP), a.shape[0], order.encode(), param, out.ctypes.data_as(DP))
    assert st == 0, _lib.last_error()
    return out


def _is_permuted_copy(a, b):
    """b equals a with rows and columns permuted (row and column multisets)."""
    ra = sorted(tuple(sorted(r)) for r in a)
    rb = sorted(tuple(sorted(r)) for r in b)
    ca = sorted(tuple(sorted(c)) for c in a.T)
    cb = sorted(tuple(sorted(c)) for c in b.T)
    return ra == rb and ca == cb and np.isclose(a.sum(), b.sum())


@pytest.mark.parametrize("order,param", [("colSort", 0), ("colSort", 1), ("rowSort", 0), ("rowSort", 1),
                                         ("skipOrder", 0), ("UTOrder", 0), ("colIndexMinimizationOrder", 0),
                                         ("alphaOrder", 2), ("alphaOrder", 3), ("randomOrder", 42)])
def test_orderings_keep_permanent(oracle, order, param):
    a = W.sparse_perm_plus(9, 3, extra=2)
    b = reorder(a, order, param)
    assert _is_permuted_copy(a, b)
    assert oracle.exact_perm(b) == oracle.exact_perm(a)


def test_utorder_triangularises():
    """A row/column-shuffled upper-triangular pattern comes back upper
    triangular."""
    rng = np.random.default_rng(4)
    t = np.triu(rng.random((10, 10)) + 0.5)
    p, q = rng.permutation(10), rng.permutation(10)
    b = reorder(t[p][:, q], "UTOrder")
    assert _is_permuted_copy(t, b)
    # the column with one nonzero comes first with its row, which covers every
    # column; then the next, and so on: the result is upper triangular again
    assert np.count_nonzero(np.tril(b != 0, -1)) == 0


def test_alpha_order_is_a_permutation():
    """Unlike the reference's final loop, every row keeps a distinct place."""
    a = W.sparse_perm_plus(13, 8, extra=3)
    for alpha in (2, 3, 4, 5):
        assert _is_permuted_copy(a, reorder(a, "alphaOrder", alpha))


def test_random_order_repeatable():
    a = W.sparse_perm_plus(8, 2)
    assert np.array_equal(reorder(a, "randomOrder", 7), reorder(a, "randomOrder", 7))
    with pytest.raises(AssertionError):
        reorder(a, "noSuchOrder")
