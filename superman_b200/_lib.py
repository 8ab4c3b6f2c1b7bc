"""ctypes binding of libsupb200.so, the C ABI declared in include/superman_b200.h.

The library is built in-tree (``make -C superman_b200/csrc``) and loaded from
the package directory.  There is no fallback: if the shared object is missing
or a call fails, a ``SupermanError`` is raised.
"""
from __future__ import annotations

import ctypes
import os
from functools import lru_cache

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libsupb200.so")

# enum spb_status
SPB_OK = 0
SPB_ERR_INVALID = 1
SPB_ERR_CUDA = 2
SPB_ERR_NO_DEVICE = 3
SPB_ERR_OOM = 4
SPB_ERR_OVERFLOW = 5
SPB_ERR_TIMEOUT = 6
SPB_ERR_CANCELLED = 7
SPB_ERR_BUSY = 8
SPB_ERR_IO = 9
SPB_ERR_NOT_SQUARE = 10
SPB_ERR_ACCURACY = 11

# enum spb_precision
SPB_PREC_FP64 = 0
SPB_PREC_DD = 1
SPB_PREC_FP32 = 2


class SupermanError(RuntimeError):
    """A C-ABI call returned a non-OK status."""

    def __init__(self, status: int, message: str):
        super().__init__(f"[{status}] {message}")
        self.status = status


class spb_options(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int),
        ("precision", ctypes.c_int),
        ("rel_tol", ctypes.c_double),
        ("unit_bits", ctypes.c_int),
        ("threads_per_block", ctypes.c_int),
        ("blocks", ctypes.c_int),
        ("stream", ctypes.c_void_p),
        ("sparse_walk", ctypes.c_int),
        ("replay_listing", ctypes.c_int),
        ("small_call", ctypes.c_int),
        ("skip_timing", ctypes.c_int),
    ]


class spb_result(ctypes.Structure):
    _fields_ = [
        ("value", ctypes.c_double),
        ("value_lo", ctypes.c_double),
        ("imag", ctypes.c_double),
        ("imag_lo", ctypes.c_double),
        ("elapsed_s", ctypes.c_double),
        ("kernel_s", ctypes.c_double),
        ("device_s", ctypes.c_double),
        ("err_est", ctypes.c_double),
        ("gray_steps", ctypes.c_uint64),
        ("refined_units", ctypes.c_uint64),
        ("status", ctypes.c_int),
        ("launches", ctypes.c_int),
        ("active_rows", ctypes.c_int),
    ]


class spb_pipeline_result(ctypes.Structure):
    _fields_ = [
        ("permanent", ctypes.c_double),
        ("imag", ctypes.c_double),
        ("time_s", ctypes.c_double),
        ("avg_n", ctypes.c_double),
        ("avg_nnz", ctypes.c_double),
        ("components", ctypes.c_int),
        ("pieces", ctypes.c_int),
        ("algorithm", ctypes.c_int),
        ("status", ctypes.c_int),
    ]


class spb_server_config(ctypes.Structure):
    _fields_ = [
        ("device", ctypes.c_int),
        ("batch_max_n", ctypes.c_int),
        ("max_batch", ctypes.c_int),
        ("slots", ctypes.c_int),
        ("max_wait_s", ctypes.c_double),
        ("admit_bytes", ctypes.c_size_t),
        ("precision", ctypes.c_int),
        ("use_graphs", ctypes.c_int),
        ("large_workers", ctypes.c_int),
        ("split", ctypes.c_int),
    ]


class spb_request_result(ctypes.Structure):
    _fields_ = [
        ("re", ctypes.c_double), ("re_lo", ctypes.c_double),
        ("im", ctypes.c_double), ("im_lo", ctypes.c_double),
        ("submit_s", ctypes.c_double), ("done_s", ctypes.c_double),
        ("n", ctypes.c_int), ("is_complex", ctypes.c_int), ("status", ctypes.c_int),
    ]


class spb_server_stats(ctypes.Structure):
    _fields_ = [(k, ctypes.c_uint64) for k in (
        "submitted", "completed", "rejected", "cancelled", "batches", "batched_requests",
        "graph_launches", "graphs_captured", "large_launches")] + [("queued_bytes", ctypes.c_size_t)] + [
        (k, ctypes.c_uint64) for k in ("split_requests", "pieces", "mid_to_large")] + [
        ("pool_bytes", ctypes.c_size_t)]


_DP = ctypes.POINTER(ctypes.c_double)
_OP = ctypes.POINTER(spb_options)
_RP = ctypes.POINTER(spb_result)

# name -> (restype, argtypes); every symbol include/superman_b200.h declares.
SIGNATURES = {
    "spb_default_options": (None, [_OP]),
    "spb_last_error": (ctypes.c_char_p, []),
    "spb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "spb_version": (ctypes.c_int, []),
    "spb_device_count": (ctypes.c_int, []),
    "spb_perm_dense_f64": (ctypes.c_int, [_DP, ctypes.c_int, _OP, _RP]),
    "spb_sparse_plan": (ctypes.c_int, [_DP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int)]),
    "spb_perm_approx": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                       ctypes.c_uint64, ctypes.c_uint64, _OP, _RP]),
    "spb_approx_samples": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                          ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, _DP]),
    "spb_perm_sparse_f64": (ctypes.c_int, [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _DP,
                                           ctypes.c_int, _OP, _RP]),
    "spb_perm_dense_f64_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _OP, _RP]),
    "spb_perm_dense_c128": (ctypes.c_int, [_DP, ctypes.c_int, _OP, _RP]),
    "spb_perm_dense_c128_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _OP, _RP]),
    "spb_perm_batch_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_void_p, ctypes.c_void_p]),
    "spb_perm_binary": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint8), ctypes.c_int, _OP,
                                       ctypes.POINTER(ctypes.c_uint32), _RP]),
    "spb_perm_dense_f64_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                                  ctypes.c_void_p]),
    "spb_perm_pipeline": (ctypes.c_int, [_DP, ctypes.c_int, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                         ctypes.POINTER(spb_pipeline_result)]),
    "spb_perm_file": (ctypes.c_int, [ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                     ctypes.POINTER(spb_pipeline_result)]),
    "spb_read_matrix": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, _DP,
                                       ctypes.c_int, ctypes.POINTER(ctypes.c_int), _DP]),
    "spb_reorder": (ctypes.c_int, [_DP, ctypes.c_int, ctypes.c_char_p, ctypes.c_ulonglong, _DP]),
    "spb_dm_prune": (ctypes.c_int, [_DP, ctypes.c_int, _DP, ctypes.POINTER(ctypes.c_int)]),
    "spb_decompose": (ctypes.c_int, [_DP, ctypes.c_int, ctypes.POINTER(ctypes.c_int),
                                     ctypes.POINTER(ctypes.c_int), _DP, ctypes.c_int, ctypes.c_size_t]),
    "spb_plan_pieces": (ctypes.c_int, [_DP, ctypes.c_int, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), _DP,
                                       ctypes.c_int, ctypes.c_size_t]),
    "spb_server_default_config": (None, [ctypes.POINTER(spb_server_config)]),
    "spb_server_create": (ctypes.c_int, [ctypes.POINTER(spb_server_config), ctypes.POINTER(ctypes.c_void_p)]),
    "spb_server_submit": (ctypes.c_int, [ctypes.c_void_p, _DP, ctypes.c_int, ctypes.c_int,
                                         ctypes.POINTER(ctypes.c_uint64)]),
    "spb_server_submit_many": (ctypes.c_int, [ctypes.c_void_p, _DP, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(ctypes.c_int), ctypes.c_int,
                                              ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_int)]),
    "spb_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(spb_request_result)]),
    "spb_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_double,
                                       ctypes.POINTER(spb_request_result)]),
    "spb_server_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "spb_server_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(spb_server_stats)]),
    "spb_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "spb_now": (ctypes.c_double, []),
    "spb_debug_fail_allocations": (None, [ctypes.c_int]),
    "spb_measure_pipe_peak": (ctypes.c_int, [ctypes.c_int, ctypes.c_int,
                                             ctypes.POINTER(ctypes.c_double)]),
}


@lru_cache(maxsize=1)
def lib() -> ctypes.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build it with `make -C superman_b200/csrc -j` "
            "(or __graft_entry__.build()); there is no CPU fallback")
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def last_error() -> str:
    return lib().spb_last_error().decode()


def check(status: int) -> None:
    if status != SPB_OK:
        raise SupermanError(status, f"{lib().spb_status_string(status).decode()}: {last_error()}")


def default_options(**kw) -> spb_options:
    o = spb_options()
    lib().spb_default_options(ctypes.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o
