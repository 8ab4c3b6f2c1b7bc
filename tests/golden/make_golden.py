"""Generates the golden fixtures in tests/golden/ (run in the build container,
where the reference sources and the oracle are available).

Each fixture is a JSON file holding
  * the input matrix exactly (float.hex per entry, so no generator or LAPACK
    difference between machines can change it),
  * the exact permanent from the oracle (CRT over the modular NW-Ryser for
    real/complex inputs, int128 plain Ryser for 0/1 inputs) as a rational
    "num/den" string,
  * when the reference CPU binary is built (oracle/_ref), its own output on
    the same matrix file and the thread count it used.

Usage:  python tests/golden/make_golden.py [case ...] [--threads T]
Cases:  dense_u01_n24_s3 dense_u01_n28_s28 dense_u01_n32_s7 complex_haar_n28_s6
        complex_haar_n20_s9 binary_n30_s4 binary_n36_s4 sparse_n40_s5
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from superman_b200 import workloads as W  # noqa: E402


def write_mtx(path, a, complex_=False, binary=False):
    n = a.shape[0]
    rows = []
    for i in range(n):
        for j in range(n):
            v = a[i, j]
            if v == 0:
                continue
            if binary:
                rows.append(f"{i + 1} {j + 1}")
            elif complex_:
                rows.append(f"{i + 1} {j + 1} {float(v.real)!r} {float(v.imag)!r}")
            else:
                rows.append(f"{i + 1} {j + 1} {float(v)!r}")
    with open(path, "w") as f:
        f.write(f"{n} {n} {len(rows)}\n")
        f.write("\n".join(rows) + "\n")


def reference_run(a, threads, complex_=False, binary=False, stats=False):
    """The reference program's output on `a`; with stats, also its
    decomposition line (piece count, mean size and nonzeros)."""
    if not os.path.exists(O.ref_binary_path()):
        return None
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "m.mtx")
        write_mtx(p, a, complex_=complex_, binary=binary)
        extra = []
        if complex_:
            extra.append("complex=true")
        if binary:
            extra.append("binary=true")
        if stats:
            st = O.run_reference_stats(p, threads=threads, extra=extra)
            val, secs = st["permanent"], st["seconds"]
        else:
            val, secs = O.run_reference(p, threads=threads, extra=extra)
    out = {"threads": threads, "seconds": secs}
    if stats:
        out.update(pieces=st["pieces"], avg_n=st["avg_n"], avg_nnz=st["avg_nnz"])
    if complex_:
        out["value_re"] = repr(val.real)
        out["value_im"] = repr(val.imag)
    else:
        out["value"] = repr(float(val))
    return out


def frac_str(f):
    return f"{f.numerator}/{f.denominator}"


def case_matrix(name):
    kind, *rest = name.split("_")
    parts = dict((p[0], int(p[1:])) for p in name.split("_")[-2:])
    n, seed = parts["n"], parts["s"]
    if name.startswith("dense_u01"):
        return "dense", W.dense_uniform(n, seed)
    if name.startswith("complex_haar"):
        return "complex", W.haar_block(n, seed)
    if name.startswith("binary"):
        return "binary", W.binary_bernoulli(n, seed)
    if name.startswith("sparse"):
        return "sparse", W.sparse_perm_plus(n, seed)
    raise ValueError(name)


def make(name, threads):
    kind, a = case_matrix(name)
    t0 = time.time()
    fx = {"name": name, "kind": kind, "n": int(a.shape[0])}
    if kind == "complex":
        fx["re_hex"] = [float(v.real).hex() for v in a.ravel()]
        fx["im_hex"] = [float(v.imag).hex() for v in a.ravel()]
        er, ei = O.exact_perm_complex(a, threads=threads)
        fx["exact_re"], fx["exact_im"] = frac_str(er), frac_str(ei)
        fx["reference"] = reference_run(a, threads, complex_=True)
    elif kind == "binary":
        fx["bits"] = "".join("1" if v else "0" for v in a.ravel())
        fx["exact"] = str(O.binary_u128(a, threads=threads))
        fx["reference"] = reference_run(a.astype(np.float64), threads, binary=True)
    else:
        fx["hex"] = [float(v).hex() for v in a.ravel()]
        if kind == "sparse":
            # exact folds (oracle/decompose.py) then exact CRT on the pieces
            import decompose as D
            fx["exact"] = frac_str(D.exact_perm_sparse(a))
        else:
            fx["exact"] = frac_str(O.exact_perm(a, threads=threads))
        fx["reference"] = reference_run(a, threads, stats=kind == "sparse")
    fx["oracle_seconds"] = time.time() - t0
    with open(os.path.join(HERE, name + ".json"), "w") as f:
        json.dump(fx, f, indent=0)
    print(name, "done in", round(fx["oracle_seconds"], 1), "s", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cases", nargs="*")
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    args = ap.parse_args()
    cases = args.cases or ["dense_u01_n24_s3", "complex_haar_n20_s9", "binary_n30_s4"]
    for c in cases:
        make(c, args.threads)


if __name__ == "__main__":
    main()
