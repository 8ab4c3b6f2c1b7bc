"""Python handle on the serving loop of libsupb200 (spb_server_* in
include/superman_b200.h): submit permanents of mixed size and type, poll or
wait for them; small ones are batched on the GPU, large ones run the
whole-GPU walk, concurrently."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


class Server:
    def __init__(self, device=0, batch_max_n=20, max_batch=2048, slots=4, max_wait_s=200e-6,
                 admit_bytes=256 << 20, precision="fp64", use_graphs=True):
        cfg = _lib.spb_server_config(device=device, batch_max_n=batch_max_n, max_batch=max_batch, slots=slots,
                                     max_wait_s=max_wait_s, admit_bytes=admit_bytes,
                                     precision=_lib.SPB_PREC_DD if precision == "dd" else _lib.SPB_PREC_FP64,
                                     use_graphs=0 if use_graphs else -1)
        self._h = ctypes.c_void_p()
        _lib.check(_lib.lib().spb_server_create(ctypes.byref(cfg), ctypes.byref(self._h)))

    def submit(self, a) -> int:
        """Queues one matrix; returns its ticket.  Raises SupermanError with
        status SPB_ERR_BUSY when admission refuses it."""
        a = np.asarray(a)
        is_c = np.iscomplexobj(a)
        buf = np.ascontiguousarray(a, dtype=np.complex128 if is_c else np.float64)
        flat = buf.view(np.float64) if is_c else buf
        t = ctypes.c_uint64()
        _lib.check(_lib.lib().spb_server_submit(self._h, flat.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                a.shape[0], int(is_c), ctypes.byref(t)))
        return t.value

    def submit_many(self, mats):
        """Queues a list of matrices in one C call; returns their tickets (0
        where admission refused one)."""
        flat, ns, cx = [], [], []
        for a in mats:
            a = np.asarray(a)
            c = np.iscomplexobj(a)
            b = np.ascontiguousarray(a, dtype=np.complex128 if c else np.float64)
            flat.append((b.view(np.float64) if c else b).ravel())
            ns.append(a.shape[0])
            cx.append(int(c))
        buf = np.concatenate(flat) if flat else np.zeros(1)
        k = len(ns)
        n_arr = (ctypes.c_int * max(1, k))(*ns)
        c_arr = (ctypes.c_int * max(1, k))(*cx)
        t_arr = (ctypes.c_uint64 * max(1, k))()
        got = ctypes.c_int()
        _lib.check(_lib.lib().spb_server_submit_many(self._h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                     n_arr, c_arr, k, t_arr, ctypes.byref(got)))
        return [t_arr[i] for i in range(k)]

    def poll(self, ticket):
        """The request's result dict when done, else None."""
        r = _lib.spb_request_result()
        st = _lib.lib().spb_server_poll(self._h, ticket, ctypes.byref(r))
        if st == _lib.SPB_ERR_BUSY:
            return None
        _lib.check(st)
        return self._dict(r)

    def wait(self, ticket, timeout_s=60.0):
        r = _lib.spb_request_result()
        _lib.check(_lib.lib().spb_server_wait(self._h, ticket, timeout_s, ctypes.byref(r)))
        return self._dict(r)

    def cancel(self, ticket):
        _lib.check(_lib.lib().spb_server_cancel(self._h, ticket))

    def stats(self) -> dict:
        s = _lib.spb_server_stats()
        _lib.check(_lib.lib().spb_server_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if self._h:
            _lib.lib().spb_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @staticmethod
    def _dict(r):
        val = complex(r.re + r.re_lo, r.im + r.im_lo) if r.is_complex else r.re + r.re_lo
        return {"permanent": val, "submit_s": r.submit_s, "done_s": r.done_s, "n": r.n,
                "status": r.status, "latency_s": r.done_s - r.submit_s}


def now() -> float:
    return _lib.lib().spb_now()
