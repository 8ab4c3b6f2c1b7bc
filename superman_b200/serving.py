"""Python handle on the serving loop of libsupb200 (spb_server_* in
include/superman_b200.h): submit permanents of mixed size and type, poll or
wait for them; admission by device pool memory, small ones batched on the
GPU, large ones on the whole-GPU walk, concurrently; real matrices with
zeros decomposed into independent pieces."""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib


_PREC = {"fp64": _lib.SPB_PREC_FP64, "dd": _lib.SPB_PREC_DD, "fp32": _lib.SPB_PREC_FP32}


class Server:
    """Defaults follow spb_server_default_config: whole-GPU requests in
    double-double refinement mode (<= 1e-12 relative at n=32), a 256 MiB
    device pool for admitted matrices, batched launches up to n=24, two
    concurrent whole-GPU workers, real matrices with zeros decomposed."""

    def __init__(self, device=0, batch_max_n=24, max_batch=2048, slots=4, max_wait_s=200e-6,
                 admit_bytes=256 << 20, precision="dd", use_graphs=True, large_workers=2, split=True):
        cfg = _lib.spb_server_config(device=device, batch_max_n=batch_max_n, max_batch=max_batch, slots=slots,
                                     max_wait_s=max_wait_s, admit_bytes=admit_bytes, precision=_PREC[precision],
                                     use_graphs=0 if use_graphs else -1, large_workers=large_workers,
                                     split=0 if split else -1)
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

    def submit_flat(self, buf, ns, is_complex):
        """Queues len(ns) matrices already packed one after another in the
        float64 array `buf` (row-major, complex ones as interleaved re/im),
        with sizes ns and flags is_complex (int32 arrays); returns their
        tickets (0 where admission refused one).  No per-matrix Python work,
        for clients that keep their requests packed."""
        buf = np.ascontiguousarray(buf, dtype=np.float64)
        ns = np.ascontiguousarray(ns, dtype=np.int32)
        cx = np.ascontiguousarray(is_complex, dtype=np.int32)
        k = int(ns.size)
        t_arr = (ctypes.c_uint64 * max(1, k))()
        got = ctypes.c_int()
        ip = ctypes.POINTER(ctypes.c_int)
        _lib.check(_lib.lib().spb_server_submit_many(self._h, buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                     ns.ctypes.data_as(ip), cx.ctypes.data_as(ip), k, t_arr,
                                                     ctypes.byref(got)))
        return list(t_arr[:k])

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
