"""The exact oracle pinned to the reference itself (CPU only).

Each golden fixture (tests/golden/*.json) holds the exact permanent computed
by the oracle (CRT over the modular NW-Ryser; int128 Ryser for 0/1 input) and
the output of the reference's own CPU program on the same matrix.  The
reference computes in FP64 (Algorithms/CPU/Dense/dpNaivePerman.h:46-142,
Algorithms/Complex/cpuComputeComplex.h:34-142, Algorithms/CPU/Sparse/
spNaivePerman.h:46-172), so its value carries its own rounding error.  A
wrong exact value would show up as a much larger gap, so each test bounds
the gap by twice the error measured when the fixture was made:

    dense U[0,1) n=24  9.1e-12      complex Haar n=20  1.4e-12
    dense U[0,1) n=32  7.0e-7       complex Haar n=28  1.6e-10
    0/1 n=30           1.5e-10      sparse n=40        6.4e-12

When the reference program is built here (oracle/_ref), it is also run
again on each fixture with the fixture's thread count (the same chunking;
its last digits still vary with the order of its `omp atomic` merge,
dpNaivePerman.h:135-136) and held to the same bound.  The sparse fixture
also pins the decomposition: the number of pieces and their mean size and
nonzero count that the reference prints (main.cpp:117-121) must equal ours.
"""
import os
import tempfile
from fractions import Fraction

import numpy as np
import pytest

from conftest import load_golden

# pinned reference error against the exact value, per fixture
PINNED = {
    "dense_u01_n24_s3": 9.1e-12,
    "dense_u01_n32_s7": 7.0e-7,
    "complex_haar_n20_s9": 1.4e-12,
    "complex_haar_n28_s6": 1.6e-10,
    "binary_n30_s4": 1.5e-10,
    "sparse_n40_s5": 6.4e-12,
}


def _reference_value(ref):
    if "value_re" in ref:
        return complex(float(ref["value_re"]), float(ref["value_im"]))
    return float(ref["value"])


def _exact(exact):
    return Fraction(exact) if isinstance(exact, int) else exact


@pytest.mark.parametrize("name", sorted(PINNED))
def test_fixture_reference_within_its_error_of_exact(oracle, name):
    _, exact, g = load_golden(name)
    err = oracle.rel_err(_reference_value(g["reference"]), _exact(exact))
    assert err <= 2 * PINNED[name], (name, err)


def _write_mtx(path, a, kind):
    n = a.shape[0]
    rows = []
    for i in range(n):
        for j in range(n):
            v = a[i, j]
            if v == 0:
                continue
            if kind == "binary":
                rows.append(f"{i + 1} {j + 1}")
            elif kind == "complex":
                rows.append(f"{i + 1} {j + 1} {float(v.real)!r} {float(v.imag)!r}")
            else:
                rows.append(f"{i + 1} {j + 1} {float(v)!r}")
    with open(path, "w") as f:
        f.write(f"{n} {n} {len(rows)}\n" + "\n".join(rows) + "\n")


def _have_reference(oracle):
    return os.path.exists(oracle.ref_binary_path())


@pytest.mark.parametrize("name", sorted(PINNED))
def test_reference_rerun_within_its_error_of_exact(oracle, name):
    if not _have_reference(oracle):
        pytest.skip("the reference CPU program (oracle/_ref) is not built on this machine")
    a, exact, g = load_golden(name)
    kind = g["kind"]
    extra = {"complex": ["complex=true"], "binary": ["binary=true"]}.get(kind, [])
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.mtx")
        _write_mtx(p, a, kind)
        v, _ = oracle.run_reference(p, threads=g["reference"]["threads"], extra=extra, timeout=600)
    err = oracle.rel_err(v, _exact(exact))
    assert err <= 2 * PINNED[name], (name, err)


def _our_decomposition(a):
    import superman_b200 as S
    comps, pieces = S.plan_pieces(a)
    sizes = [p.shape[0] for _, p in pieces]
    nnz = [int(np.count_nonzero(p)) for _, p in pieces]
    return comps, len(pieces), float(np.mean(sizes)), float(np.mean(nnz))


def test_decomposition_matches_the_fixture():
    a, _, g = load_golden("sparse_n40_s5")
    ref = g["reference"]
    _, count, avg_n, avg_nnz = _our_decomposition(a)
    assert count == ref["pieces"]
    assert avg_n == pytest.approx(ref["avg_n"], abs=1e-3)
    assert avg_nnz == pytest.approx(ref["avg_nnz"], abs=1e-3)


def test_decomposition_matches_a_reference_run(oracle):
    if not _have_reference(oracle):
        pytest.skip("the reference CPU program (oracle/_ref) is not built on this machine")
    a, exact, _ = load_golden("sparse_n40_s5")
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.mtx")
        _write_mtx(p, a, "sparse")
        ref = oracle.run_reference_stats(p, timeout=600)
    _, count, avg_n, avg_nnz = _our_decomposition(a)
    assert count == ref["pieces"]
    assert avg_n == pytest.approx(ref["avg_n"], abs=1e-3)
    assert avg_nnz == pytest.approx(ref["avg_nnz"], abs=1e-3)
    assert oracle.rel_err(ref["permanent"], exact) <= 2 * PINNED["sparse_n40_s5"]
