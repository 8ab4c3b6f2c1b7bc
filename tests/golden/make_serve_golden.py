"""Exact permanents of a sample of the seeded serving stream, for the accuracy
checks of the serving loop (tests/test_serve_gpu.py and the `serve` bench
workload).  Run in the build container, where the oracle is built:

    python tests/golden/make_serve_golden.py [--threads T]

The stream is superman_b200.workloads.ServeStream(8, 32, 20000, seed=2026):
n uniform in [8, 32], half real U[0, 1) matrices, half blocks of Haar-random
256 x 256 unitaries.  The sample is the first request of each size in SIZES
and of each kind; its exact permanent comes from the oracle's CRT over the
modular NW-Ryser (Gaussian integers for complex input) and is stored as a
rational "num/den" string, with the SHA-256 of the matrix's float64 bytes so
that a consumer can confirm it rebuilt the same matrix.  The file is written
after every entry (cheapest first), so an interrupted run keeps what it
finished; a rerun skips the entries already present.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import oracle as O  # noqa: E402
from superman_b200 import workloads as W  # noqa: E402

STREAM = {"n_lo": 8, "n_hi": 32, "count": 20000, "seed": 2026}
SIZES = [8, 14, 20, 21, 24, 26, 28, 29, 30, 31, 32]
OUT = os.path.join(HERE, "serve_sample.json")


def frac_str(f):
    return f"{f.numerator}/{f.denominator}"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count())
    ap.add_argument("--max-n", type=int, default=32)
    args = ap.parse_args()
    s = W.ServeStream(STREAM["n_lo"], STREAM["n_hi"], STREAM["count"], STREAM["seed"])
    data = {"stream": STREAM, "entries": []}
    if os.path.exists(OUT):
        data = json.load(open(OUT))
    have = {e["index"] for e in data["entries"]}
    # cheapest first: real before complex at each size
    todo = [(n, c) for n in SIZES if n <= args.max_n for c in (False, True)]
    for n, cplx in todo:
        i = s.first_index(n, cplx)
        if i < 0 or i in have:
            continue
        a = s.matrix(i)
        t0 = time.time()
        e = {"index": i, "n": n, "kind": "complex" if cplx else "real", "sha256": W.matrix_sha256(a)}
        if cplx:
            er, ei = O.exact_perm_complex(a, threads=args.threads)
            e["exact_re"], e["exact_im"] = frac_str(er), frac_str(ei)
        else:
            e["exact"] = frac_str(O.exact_perm(a, threads=args.threads))
        e["oracle_seconds"] = round(time.time() - t0, 1)
        data["entries"].append(e)
        data["entries"].sort(key=lambda x: (x["n"], x["kind"]))
        with open(OUT + ".tmp", "w") as f:
            json.dump(data, f, indent=0)
        os.replace(OUT + ".tmp", OUT)
        print(f"request {i}: n={n} {e['kind']} done in {e['oracle_seconds']} s", flush=True)


if __name__ == "__main__":
    main()
