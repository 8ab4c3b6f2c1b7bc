"""superman_b200 — B200-native (sm_100a) exact matrix permanents.

Python host mirror of SUPerman's permanent API over the C ABI in
include/superman_b200.h.  The compute path is libsupb200.so (hand-written CUDA
for sm_100a); there is no CPU fallback.

    from superman_b200 import perm_dense, perm_complex
    r = perm_dense(a)          # Result(time, permanent, ...)
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import SPB_PREC_DD, SPB_PREC_FP64, SupermanError

__all__ = ["Result", "plan_pieces", "perm_dense", "perm_sparse", "perm_complex", "perm_binary", "perm_approx",
           "approx_samples", "SupermanError", "SPB_PREC_FP64", "SPB_PREC_DD", "device_count"]

_PREC = {"fp64": SPB_PREC_FP64, "kahan": SPB_PREC_FP64, "dd": SPB_PREC_DD, "fp32": 2}
_SPARSE_WALK = {"auto": 0, "never": 1, "always": 2}


@dataclass
class Result:
    """Mirror of the reference's Result record {time, permanent}
    (CommonFiles/Result.h:29-37) with the extra fields the C ABI reports."""
    time: float
    permanent: complex | float
    permanent_lo: float = 0.0
    imag_lo: float = 0.0
    kernel_s: float = 0.0
    err_est: float = 0.0
    gray_steps: int = 0
    refined_units: int = 0
    launches: int = 0
    active_rows: int = 0


def device_count() -> int:
    return _lib.lib().spb_device_count()


def _options(precision, device, **shape):
    p = _PREC[precision] if isinstance(precision, str) else int(precision)
    return _lib.default_options(device=device, precision=p, **shape)


def _to_result(r: _lib.spb_result, complex_: bool) -> Result:
    val = complex(r.value, r.imag) if complex_ else r.value
    return Result(time=r.elapsed_s, permanent=val, permanent_lo=r.value_lo, imag_lo=r.imag_lo,
                  kernel_s=r.kernel_s, err_est=r.err_est, gray_steps=r.gray_steps,
                  refined_units=r.refined_units, launches=r.launches, active_rows=r.active_rows)


def perm_dense(a, precision="fp64", device: int = 0, **shape) -> Result:
    """Permanent of a dense real n x n matrix (1 <= n <= 63)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("perm_dense needs a square 2-D array")
    out = _lib.spb_result()
    opt = _options(precision, device, **shape)
    st = _lib.lib().spb_perm_dense_f64(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       a.shape[0], ctypes.byref(opt), ctypes.byref(out))
    _lib.check(st)
    return _to_result(out, False)


def perm_sparse(a, precision="fp64", device: int = 0, walk: str = "auto", **shape) -> Result:
    """Permanent of a sparse real n x n matrix (1 <= n <= 63), given dense or
    as a (cptrs, rows, cvals) compressed-column triple like the reference's
    SparseMatrix.  walk: "auto" (cost model), "never" (dense walk) or
    "always" (row-compacted walk whenever the pattern allows);
    Result.active_rows tells which ran."""
    if isinstance(a, tuple):
        cptrs, rows, cvals = a
        cptrs = np.ascontiguousarray(cptrs, dtype=np.int32)
        rows = np.ascontiguousarray(rows, dtype=np.int32)
        cvals = np.ascontiguousarray(cvals, dtype=np.float64)
        n = cptrs.size - 1
    else:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.ndim != 2 or a.shape[0] != a.shape[1]:
            raise ValueError("perm_sparse needs a square 2-D array or a (cptrs, rows, cvals) triple")
        n = a.shape[0]
        r_idx, c_idx = np.nonzero(a.T)  # column-major order: (column, row) pairs
        cptrs = np.zeros(n + 1, dtype=np.int32)
        np.add.at(cptrs, r_idx + 1, 1)
        cptrs = np.cumsum(cptrs).astype(np.int32)
        rows = np.ascontiguousarray(c_idx, dtype=np.int32)
        cvals = np.ascontiguousarray(a.T[r_idx, c_idx], dtype=np.float64)
    out = _lib.spb_result()
    opt = _options(precision, device, **shape)
    opt.sparse_walk = _SPARSE_WALK[walk]
    ip = ctypes.POINTER(ctypes.c_int)
    st = _lib.lib().spb_perm_sparse_f64(cptrs.ctypes.data_as(ip), rows.ctypes.data_as(ip),
                                        cvals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), n,
                                        ctypes.byref(opt), ctypes.byref(out))
    _lib.check(st)
    return _to_result(out, False)


def _csc_pattern(a):
    """(cptrs, rows) of the nonzero pattern of a square matrix, or the
    pattern part of a (cptrs, rows[, vals]) triple."""
    if isinstance(a, tuple):
        return np.ascontiguousarray(a[0], dtype=np.int32), np.ascontiguousarray(a[1], dtype=np.int32)
    a = np.asarray(a)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("needs a square 2-D array or a compressed-column tuple")
    c_idx, r_idx = np.nonzero(a.T)
    cptrs = np.zeros(a.shape[0] + 1, dtype=np.int64)
    np.add.at(cptrs, c_idx + 1, 1)
    return np.cumsum(cptrs).astype(np.int32), np.ascontiguousarray(r_idx, dtype=np.int32)


def perm_approx(a, samples: int = 1_000_000, seed: int = 1, device: int = 0, **shape) -> Result:
    """Monte-Carlo estimate of the permanent of the nonzero pattern of `a`
    (its number of perfect matchings), any n up to 2^20; the mirror of the
    reference's approximation algorithm.  Result.err_est is the relative
    standard error of the mean."""
    cptrs, rows = _csc_pattern(a)
    out = _lib.spb_result()
    opt = _lib.default_options(device=device, **shape)
    ip = ctypes.POINTER(ctypes.c_int)
    st = _lib.lib().spb_perm_approx(cptrs.ctypes.data_as(ip), rows.ctypes.data_as(ip), cptrs.size - 1,
                                    samples, seed, ctypes.byref(opt), ctypes.byref(out))
    _lib.check(st)
    return _to_result(out, False)


def approx_samples(a, first: int, count: int, seed: int = 1) -> np.ndarray:
    """The individual estimates of samples first .. first+count-1 of
    perm_approx(a, seed=seed)."""
    cptrs, rows = _csc_pattern(a)
    est = np.zeros(count)
    ip = ctypes.POINTER(ctypes.c_int)
    _lib.check(_lib.lib().spb_approx_samples(cptrs.ctypes.data_as(ip), rows.ctypes.data_as(ip), cptrs.size - 1,
                                             first, count, seed, est.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
    return est


def plan_pieces(a):
    """The pieces the reference's real-matrix flow computes for `a` (pruning,
    connected components, DecomposePerman per component), without computing
    them: (components, [(component, piece matrix)]).  The permanent of `a` is
    the product over components of the sum of their pieces' permanents; a
    component without pieces contributes 0.  CPU only."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    n = a.shape[0]
    dp = ctypes.POINTER(ctypes.c_double)
    ip = ctypes.POINTER(ctypes.c_int)
    comps, count = ctypes.c_int(), ctypes.c_int()
    L = _lib.lib()
    _lib.check(L.spb_plan_pieces(a.ctypes.data_as(dp), n, ctypes.byref(comps), ctypes.byref(count),
                                 None, None, None, 0, 0))
    k = count.value
    sizes = np.zeros(max(k, 1), dtype=np.int32)
    owner = np.zeros(max(k, 1), dtype=np.int32)
    data = np.zeros(max(k * n * n, 1))
    _lib.check(L.spb_plan_pieces(a.ctypes.data_as(dp), n, ctypes.byref(comps), ctypes.byref(count),
                                 sizes.ctypes.data_as(ip), owner.ctypes.data_as(ip), data.ctypes.data_as(dp),
                                 k, data.size))
    out, off = [], 0
    for i in range(k):
        m = int(sizes[i])
        out.append((int(owner[i]), data[off:off + m * m].reshape(m, m).copy()))
        off += m * m
    return comps.value, out


def perm_binary(a, device: int = 0, **shape) -> Result:
    """Exact permanent of a 0/1 n x n matrix (1 <= n <= 63); Result.permanent
    is a Python int."""
    a = np.ascontiguousarray(np.asarray(a) != 0, dtype=np.uint8)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("perm_binary needs a square 2-D array")
    out = _lib.spb_result()
    limbs = (ctypes.c_uint32 * 10)()
    opt = _lib.default_options(device=device, **shape)
    st = _lib.lib().spb_perm_binary(a.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), a.shape[0],
                                    ctypes.byref(opt), limbs, ctypes.byref(out))
    _lib.check(st)
    v = 0
    for i in reversed(range(10)):
        v = (v << 32) | limbs[i]
    if v >> 319:
        v -= 1 << 320
    res = _to_result(out, False)
    res.permanent = v
    return res


def perm_complex(a, precision="fp64", device: int = 0, **shape) -> Result:
    """Permanent of a dense complex128 n x n matrix (1 <= n <= 63)."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    if a.ndim != 2 or a.shape[0] != a.shape[1]:
        raise ValueError("perm_complex needs a square 2-D array")
    out = _lib.spb_result()
    opt = _options(precision, device, **shape)
    ri = a.view(np.float64)
    st = _lib.lib().spb_perm_dense_c128(ri.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        a.shape[0], ctypes.byref(opt), ctypes.byref(out))
    _lib.check(st)
    return _to_result(out, True)
