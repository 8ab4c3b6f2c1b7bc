"""The C ABI library loads on a machine without a GPU and exports every
symbol include/superman_b200.h declares; status/error plumbing works without
a device.  No compute calls here."""
import ctypes
import os
import re

import numpy as np

from superman_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "superman_b200.h")).read()
    return sorted(set(re.findall(r"SPB_API\s+[\w\s\*]+?\b(spb_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    syms = declared_symbols()
    assert "spb_perm_dense_f64" in syms and "spb_perm_dense_c128" in syms
    assert len(syms) >= 8


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    # the Python binding types every declared symbol too
    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_status_strings_and_defaults():
    L = _lib.lib()
    assert L.spb_status_string(0) == b"ok"
    assert L.spb_status_string(_lib.SPB_ERR_OVERFLOW) == b"result overflow"
    o = _lib.default_options()
    assert o.device == 0 and o.precision == _lib.SPB_PREC_FP64
    assert L.spb_version() >= 100


def test_invalid_arguments_are_rejected_without_a_device():
    L = _lib.lib()
    r = _lib.spb_result()
    a = np.zeros((4, 4))
    p = a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    assert L.spb_perm_dense_f64(p, 0, None, ctypes.byref(r)) == _lib.SPB_ERR_INVALID
    assert L.spb_perm_dense_f64(p, 64, None, ctypes.byref(r)) == _lib.SPB_ERR_INVALID
    assert L.spb_perm_dense_f64(None, 4, None, ctypes.byref(r)) == _lib.SPB_ERR_INVALID
    assert "n=64" in _lib.last_error() or "1 <= n" in _lib.last_error()
