"""TEST INFRASTRUCTURE ONLY — the checker, never the product.

Python side of the oracle: a ctypes loader for ``oracle/_build/liboracle.so``
(the C restatement of the reference's NW-Ryser), exact rational permanents by
CRT over the modular NW-Ryser, and pure-Python exact cross-checks for small n.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s cpu_baseline leg
may import this module.

Exactness: every finite double is num/2^k, so scaling row r by the largest
denominator 2^s_r in that row gives an integer matrix K with
perm(A) = perm(K) / 2^(sum s_r).  perm(K) is found modulo enough 62-bit primes
to exceed twice the bound prod_r sum_j |K_rj|, then recombined by CRT.  This
stands in for the GMP rational permanent named by the reference's arbitrary
precision path (Algorithms/CPU/Dense/dpArbitraryPerman.h:47-176), whose GMP
headers are not available here.
"""
from __future__ import annotations

import ctypes
import itertools
import math
import os
import subprocess
from fractions import Fraction
from functools import lru_cache

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_REF_BIN = os.path.join(_HERE, "_ref", "superman_ref")


def build() -> None:
    """Compile liboracle.so (and the reference CPU binary when its sources exist)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    if not os.path.exists(_LIB_PATH):
        build()
    L = ctypes.CDLL(_LIB_PATH)
    dp = ctypes.POINTER(ctypes.c_double)
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.orc_dense_nw.restype = ctypes.c_double
    L.orc_dense_nw.argtypes = [dp, ctypes.c_int, ctypes.c_int]
    L.orc_sparse_nw.restype = ctypes.c_double
    L.orc_sparse_nw.argtypes = [dp, ctypes.c_int, ctypes.c_int]
    L.orc_complex_nw.restype = None
    L.orc_complex_nw.argtypes = [dp, ctypes.c_int, ctypes.c_int, dp, dp]
    L.orc_binary_ryser_u128.restype = None
    L.orc_binary_ryser_u128.argtypes = [ctypes.POINTER(ctypes.c_uint8), ctypes.c_int,
                                        ctypes.c_int, u64p]
    L.orc_perm_mod_primes.restype = None
    L.orc_perm_mod_primes.argtypes = [u64p, ctypes.c_int, u64p, ctypes.c_int, ctypes.c_int, u64p]
    L.orc_perm_mod_primes_gauss.restype = None
    L.orc_perm_mod_primes_gauss.argtypes = [u64p, u64p, ctypes.c_int, u64p, ctypes.c_int,
                                            ctypes.c_int, u64p, u64p]
    ip = ctypes.POINTER(ctypes.c_int)
    fp = ctypes.POINTER(ctypes.c_float)
    L.orc_rasmussen_init.restype = None
    L.orc_rasmussen_init.argtypes = [ctypes.c_int, ip, ip, ip, ip, fp, fp]
    L.orc_rasmussen_samples.restype = None
    L.orc_rasmussen_samples.argtypes = [ctypes.c_int, ip, ip, ip, ip, fp, fp, ctypes.c_uint64,
                                        ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, dp]
    return L


def _threads(threads):
    return threads if threads else (os.cpu_count() or 1)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _u64ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64))


# ------------------------------------------------- reference restatements --

def dense_nw(a, threads=None) -> float:
    """Algorithms/CPU/Dense/dpNaivePerman.h:46-142 on a row-major n x n array."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    return lib().orc_dense_nw(_dptr(a), a.shape[0], _threads(threads))


def sparse_nw(a, threads=None) -> float:
    """Algorithms/CPU/Sparse/spNaivePerman.h:46-172 (columns as given)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    return lib().orc_sparse_nw(_dptr(a), a.shape[0], _threads(threads))


def complex_nw(a, threads=None) -> complex:
    """Algorithms/Complex/cpuComputeComplex.h:34-142."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    re, im = ctypes.c_double(), ctypes.c_double()
    ri = a.view(np.float64)
    lib().orc_complex_nw(_dptr(ri), a.shape[0], _threads(threads), ctypes.byref(re),
                         ctypes.byref(im))
    return complex(re.value, im.value)


def binary_u128(a, threads=None) -> int:
    """Exact perm of a 0/1 matrix by plain Ryser mod 2^128 (signed result)."""
    a = np.ascontiguousarray(np.asarray(a) != 0, dtype=np.uint8)
    out = (ctypes.c_uint64 * 2)()
    lib().orc_binary_ryser_u128(a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), a.shape[0],
                                _threads(threads), out)
    v = out[0] | (out[1] << 64)
    return v - (1 << 128) if v >> 127 else v


# ------------------------------------------------------------ exact (CRT) --

def _is_prime(n: int) -> bool:
    if n < 2:
        return False
    small = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)
    for p in small:
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for b in small:  # deterministic for n < 3.3e24
        x = pow(b, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


@lru_cache(maxsize=1)
def _prime_pool(count: int = 256):
    out, c = [], (1 << 62) - 1
    while len(out) < count:
        if _is_prime(c):
            out.append(c)
        c -= 2
    return tuple(out)


def _primes_for(bound_bits: int):
    need = bound_bits + 2
    pool = _prime_pool()
    out, bits = [], 0
    for p in pool:
        out.append(p)
        bits += p.bit_length() - 1
        if bits >= need:
            return out
    raise ValueError("entries too wide for the prime pool")


def _crt_signed(residues, primes) -> int:
    x, m = 0, 1
    for r, p in zip(residues, primes):
        # solve x' = x (mod m), x' = r (mod p)
        t = ((r - x) * pow(m, -1, p)) % p
        x += m * t
        m *= p
    if x > m // 2:
        x -= m
    return x


def _integerize_rows(rows):
    """rows: list of lists of Fractions-as-(num, den) -> (K rows, total shift)."""
    K, shift = [], 0
    for row in rows:
        dens = [d for (_, d) in row]
        dmax = max(dens) if dens else 1
        shift += dmax.bit_length() - 1
        K.append([num * (dmax // d) for (num, d) in row])
    return K, shift


def exact_perm(a, threads=None) -> Fraction:
    """Exact rational permanent of a real float64 matrix."""
    a = np.asarray(a, dtype=np.float64)
    n = a.shape[0]
    if n == 0:
        return Fraction(1)
    rows = [[float(v).as_integer_ratio() for v in a[i]] for i in range(n)]
    K, shift = _integerize_rows(rows)
    bound_bits = sum(max(1, sum(abs(v) for v in row)).bit_length() for row in K) + 1
    primes = _primes_for(bound_bits)
    kmod = np.array([[[v % p for v in row] for row in K] for p in primes], dtype=np.uint64)
    pr = np.array(primes, dtype=np.uint64)
    out = np.zeros(len(primes), dtype=np.uint64)
    lib().orc_perm_mod_primes(_u64ptr(kmod), n, _u64ptr(pr), len(primes), _threads(threads),
                              _u64ptr(out))
    val = _crt_signed([int(v) for v in out], primes)
    return Fraction(val, 1 << shift)


def exact_perm_fractions(a, threads=None) -> Fraction:
    """Exact permanent of a matrix of Fractions (or ints): each row is scaled
    by the lcm of its denominators, the integer permanent found by CRT."""
    n = len(a)
    if n == 0:
        return Fraction(1)
    K, scale = [], 1
    for row in a:
        row = [Fraction(v) for v in row]
        den = 1
        for v in row:
            den = den * v.denominator // math.gcd(den, v.denominator)
        scale *= den
        K.append([int(v * den) for v in row])
    bound_bits = sum(max(1, sum(abs(v) for v in row)).bit_length() for row in K) + 1
    primes = _primes_for(bound_bits)
    kmod = np.array([[[v % p for v in row] for row in K] for p in primes], dtype=np.uint64)
    pr = np.array(primes, dtype=np.uint64)
    out = np.zeros(len(primes), dtype=np.uint64)
    lib().orc_perm_mod_primes(_u64ptr(kmod), n, _u64ptr(pr), len(primes), _threads(threads),
                              _u64ptr(out))
    return Fraction(_crt_signed([int(v) for v in out], primes), scale)


def exact_perm_complex(a, threads=None):
    """Exact (re, im) permanent of a complex128 matrix, as two Fractions."""
    a = np.asarray(a, dtype=np.complex128)
    n = a.shape[0]
    if n == 0:
        return Fraction(1), Fraction(0)
    K_re, K_im, shift = [], [], 0
    for i in range(n):
        pr_ = [float(v.real).as_integer_ratio() for v in a[i]]
        pi_ = [float(v.imag).as_integer_ratio() for v in a[i]]
        dmax = max([d for _, d in pr_] + [d for _, d in pi_])
        shift += dmax.bit_length() - 1
        K_re.append([num * (dmax // d) for num, d in pr_])
        K_im.append([num * (dmax // d) for num, d in pi_])
    bound_bits = sum(max(1, sum(abs(x) + abs(y) for x, y in zip(r1, r2))).bit_length()
                     for r1, r2 in zip(K_re, K_im)) + 1
    primes = _primes_for(bound_bits)
    kre = np.array([[[v % p for v in row] for row in K_re] for p in primes], dtype=np.uint64)
    kim = np.array([[[v % p for v in row] for row in K_im] for p in primes], dtype=np.uint64)
    pr = np.array(primes, dtype=np.uint64)
    ore = np.zeros(len(primes), dtype=np.uint64)
    oim = np.zeros(len(primes), dtype=np.uint64)
    lib().orc_perm_mod_primes_gauss(_u64ptr(kre), _u64ptr(kim), n, _u64ptr(pr), len(primes),
                                    _threads(threads), _u64ptr(ore), _u64ptr(oim))
    vre = _crt_signed([int(v) for v in ore], primes)
    vim = _crt_signed([int(v) for v in oim], primes)
    return Fraction(vre, 1 << shift), Fraction(vim, 1 << shift)


# ------------------------------------------------- pure Python, small n ----

def rasmussen_samples(a, first: int, count: int, seed: int, threads=None):
    """Estimates of samples first .. first+count-1 of the sequential
    importance sampler on the nonzero pattern of `a` (orc_rasmussen_samples)."""
    import numpy as np
    pat = np.asarray(a) != 0
    n = pat.shape[0]
    rptr = np.zeros(n + 1, dtype=np.int32)
    rptr[1:] = np.cumsum(pat.sum(axis=1))
    col = np.ascontiguousarray(np.nonzero(pat)[1], dtype=np.int32)
    cptr = np.zeros(n + 1, dtype=np.int32)
    cptr[1:] = np.cumsum(pat.sum(axis=0))
    row = np.ascontiguousarray(np.nonzero(pat.T)[1], dtype=np.int32)
    L = lib()
    ip = ctypes.POINTER(ctypes.c_int)
    fp = ctypes.POINTER(ctypes.c_float)
    rv = np.zeros(n, dtype=np.float32)
    cv = np.zeros(n, dtype=np.float32)
    args = [x.ctypes.data_as(ip) for x in (rptr, col, cptr, row)]
    L.orc_rasmussen_init(n, *args, rv.ctypes.data_as(fp), cv.ctypes.data_as(fp))
    out = np.zeros(count)
    L.orc_rasmussen_samples(n, *args, rv.ctypes.data_as(fp), cv.ctypes.data_as(fp), seed, first, count,
                            _threads(threads), out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


def brute_perm(a):
    """Sum over all permutations, exact for int/Fraction entries (n <= 8)."""
    n = len(a)
    total = 0
    for p in itertools.permutations(range(n)):
        t = 1
        for i in range(n):
            t *= a[i][p[i]]
        total += t
    return total


def ryser_exact(a):
    """Plain Ryser with exact Python arithmetic (n <= ~14); entries int/Fraction/complex."""
    n = len(a)
    if n == 0:
        return 1
    total = 0
    for mask in range(1, 1 << n):
        prod = 1
        for i in range(n):
            s = 0
            for j in range(n):
                if mask >> j & 1:
                    s += a[i][j]
            prod *= s
        total += (-1) ** bin(mask).count("1") * prod
    return (-1) ** n * total


def rel_err(approx, exact) -> float:
    """|approx - exact| / |exact| evaluated exactly, returned as float."""
    if isinstance(exact, tuple):
        er, ei = exact
        ar, ai = Fraction(approx.real), Fraction(approx.imag)
        num = (ar - er) ** 2 + (ai - ei) ** 2
        den = er ** 2 + ei ** 2
        return math.sqrt(float(num / den)) if den else float("inf")
    d = Fraction(approx) - exact
    return float(abs(d) / abs(exact)) if exact else float(abs(d))


# ------------------------------------------------- reference CPU binary ----

def ref_binary_path() -> str:
    return _REF_BIN


def run_reference_stats(mtx_path: str, threads=None, extra=(), timeout=3600) -> dict:
    """Like run_reference, plus the decomposition line the reference prints
    (main.cpp:117-121): {"permanent", "seconds", "pieces", "avg_n", "avg_nnz"}."""
    import re
    import tempfile
    work = tempfile.mkdtemp(prefix="spb_ref_")
    os.makedirs(os.path.join(work, "build"), exist_ok=True)
    args = [_REF_BIN, "pid=2", f"repo_dir={work}/", f"filename={mtx_path}", "mode=cpu",
            f"thread_count={_threads(threads)}", *extra]
    out = subprocess.run(args, check=True, capture_output=True, text=True, timeout=timeout).stdout
    m = re.search(r"Submatrix count: (\d+) - Average N: (\S+) - Average NNZ: (\S+)", out)
    p = re.search(r"Permanent: (\S+) - Computed in: (\S+) seconds", out)
    if m is None or p is None:
        raise RuntimeError("unexpected reference output: " + out[-400:])
    return {"permanent": float(p.group(1)), "seconds": float(p.group(2)), "pieces": int(m.group(1)),
            "avg_n": float(m.group(2)), "avg_nnz": float(m.group(3))}


def run_reference(mtx_path: str, threads=None, extra=(), timeout=3600):
    """Run the reference's own CPU program on a matrix file; returns
    (permanent as float or complex, seconds).  Needs oracle/_ref built.
    Each run gets a fresh mailbox directory: the reference blocks while an
    unread mailbox file exists (CommonFiles/Helpers.h:71-116)."""
    import re
    import tempfile
    work = tempfile.mkdtemp(prefix="spb_ref_")
    os.makedirs(os.path.join(work, "build"), exist_ok=True)
    args = [_REF_BIN, "pid=2", f"repo_dir={work}/", f"filename={mtx_path}", "mode=cpu",
            f"thread_count={_threads(threads)}", *extra]
    out = subprocess.run(args, check=True, capture_output=True, text=True,
                         timeout=timeout).stdout
    m2 = re.search(r"Permanent: \(([^,]+),([^)]+)\) - Computed in: (\S+) seconds", out)
    if m2 is not None:
        return complex(float(m2.group(1)), float(m2.group(2))), float(m2.group(3))
    m = re.search(r"Permanent: (\S+) - Computed in: (\S+) seconds", out)
    if m is None:
        raise RuntimeError("unexpected reference output: " + out[-400:])
    return float(m.group(1)), float(m.group(2))
