"""The reference's top-level flow through the C ABI (spb_perm_pipeline,
spb_perm_file) and the superman command-line front end, on the GPU."""
import ctypes
import math
import os
import re
import subprocess

import numpy as np
import pytest

from superman_b200 import _lib
from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def pipeline(a, *args):
    a = np.ascontiguousarray(a, dtype=np.float64)
    arr = (ctypes.c_char_p * max(1, len(args)))(*[x.encode() for x in args])
    out = _lib.spb_pipeline_result()
    st = _lib.lib().spb_perm_pipeline(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.shape[0], arr,
                                      len(args), ctypes.byref(out))
    return st, out


def test_pipeline_dense_matches_direct(spb, oracle):
    a = W.dense_uniform(18, seed=18)
    st, out = pipeline(a)
    assert st == 0
    assert out.components == 1 and out.pieces == 1
    assert oracle.rel_err(out.permanent, oracle.exact_perm(a)) <= 1e-13


def test_pipeline_block_diagonal_is_product(spb, oracle):
    b1, b2 = W.dense_uniform(7, 1), W.dense_uniform(9, 2)
    a = np.zeros((16, 16))
    a[:7, :7] = b1
    a[7:, 7:] = b2
    rng = np.random.default_rng(3)
    p, q = rng.permutation(16), rng.permutation(16)
    st, out = pipeline(a[p][:, q], "calculation_precision=dd")
    assert st == 0 and out.components == 2
    want = oracle.exact_perm(b1) * oracle.exact_perm(b2)
    assert oracle.rel_err(out.permanent, want) <= 1e-13


def test_pipeline_structurally_singular_is_zero(spb):
    a = W.dense_uniform(10, 4)
    a[:, 3] = 0.0
    st, out = pipeline(a)
    assert st == 0 and out.permanent == 0.0


def test_pipeline_binary_exact(spb, oracle):
    a = W.binary_bernoulli(22, seed=9).astype(np.float64)
    st, out = pipeline(a, "binary=true")
    assert st == 0
    assert out.permanent == float(oracle.binary_u128(a))


def test_pipeline_decomposes_sparse_n34(spb, oracle):
    a = W.sparse_perm_plus(34, seed=11)
    st, out = pipeline(a, "algorithm=xshared_mshared")
    assert st == 0 and out.pieces >= 1
    assert out.avg_n <= 30


def test_pipeline_mode_errors(spb):
    a = W.dense_uniform(5, 1)
    st, _ = pipeline(a, "mode=cpu")
    assert st == _lib.SPB_ERR_INVALID and "unavailable" in _lib.last_error()
    st, _ = pipeline(a, "algorithm=no_such_algorithm")
    assert st == _lib.SPB_ERR_INVALID and "UNKNOWN ALGORITHM" in _lib.last_error()
    st, _ = pipeline(a, "approx_samples=many")
    assert st == _lib.SPB_ERR_INVALID and "approx_samples" in _lib.last_error()


def write_mtx(path, a):
    n = a.shape[0]
    lines = [f"{i + 1} {j + 1} {float(a[i, j])!r}" for i in range(n) for j in range(n) if a[i, j] != 0]
    path.write_text(f"{n} {n} {len(lines)}\n" + "\n".join(lines) + "\n")


def test_cli_closed_form(spb, tmp_path):
    """ExampleMatrices/dense.mtx is 0.91*J_45; the same closed form at n=20."""
    p = tmp_path / "dense.mtx"
    write_mtx(p, np.full((20, 20), 0.91))
    exe = os.path.join(ROOT, "superman_b200", "superman")
    out = subprocess.run([exe, f"filename={p}", "mode=single_gpu"], capture_output=True, text=True,
                         timeout=120, check=True).stdout
    m = re.search(r"Permanent: (\S+) - Computed in: (\S+) seconds", out)
    assert m, out
    want = math.factorial(20) * 0.91 ** 20
    assert abs(float(m.group(1)) - want) <= 1e-12 * want
    assert "Submatrix count: 1" in out


def test_cli_complex(spb, tmp_path):
    """ExampleMatrices/complex.mtx is i*J_40 (permanent 40!); here i*J_12 = 12!."""
    p = tmp_path / "c.mtx"
    n = 12
    p.write_text(f"{n} {n} {n * n}\n" + "\n".join(f"{i + 1} {j + 1} 0 1" for i in range(n) for j in range(n)) + "\n")
    exe = os.path.join(ROOT, "superman_b200", "superman")
    out = subprocess.run([exe, f"filename={p}", "complex=true"], capture_output=True, text=True, timeout=120,
                         check=True).stdout
    m = re.search(r"Permanent: \(([^,]+),([^)]+)\)", out)
    assert m, out
    assert abs(float(m.group(1)) - math.factorial(12)) <= 1e-12 * math.factorial(12)
    assert abs(float(m.group(2))) <= 1e-12 * math.factorial(12)


@pytest.mark.parametrize("args", [(), ("calculation_precision=dd",), ("algorithm=xshared_mshared",),
                                  ("algorithm=xshared_mshared", "calculation_precision=dd")])
def test_pipeline_sparse_n40_golden(spb, oracle, args):
    """Config C3 (n=40: random permutation + 3 extra nonzeros per row, values
    U[0.5,1.5)) through pruning, components, decomposition and the GPU walks,
    against the exact value (oracle/decompose.py); the reference CPU binary's
    sparse path is 6.4e-12 away from it."""
    from conftest import load_golden
    a, exact, g = load_golden("sparse_n40_s5")
    st, out = pipeline(a, *args)
    assert st == 0, _lib.last_error()
    err = oracle.rel_err(out.permanent, exact)
    print(args, "pieces", out.pieces, "avg n", out.avg_n, "rel err", err, "time", out.time_s)
    assert err <= 1e-12
    ref_err = oracle.rel_err(float(g["reference"]["value"]), exact)
    assert ref_err < 1e-9
