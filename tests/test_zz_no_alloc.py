"""The allocation-free dense entry point, spb_perm_dense_f64_noalloc, against
the allocating one, spb_perm_dense_f64.

Some callers cannot let a library allocate device memory: programs that hand
all of device memory to their own pool allocator up front, and request loops
that cannot take cudaFree's device-wide synchronisation or a mid-request
allocation failure.  The variant keeps its working memory in one fixed device
array inside the library, so each call here passes only device input and
output buffers (allocated by the caller, torch in this test).

Both entry points run the FP64 walk with the same launch shape, so their
results agree to the tolerance of the other dense parity tests (in practice
bit for bit), at every size the fixed array takes, 40 included.

This file is collected last on purpose: it runs after every other GPU test in
a full run, and it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from superman_b200 import _lib
from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu

# Same bound as the other dense parity tests (FP64 products, double-double sum).
REL_TOL = 1e-13


def _call(L, d_a, n, d_out):
    return L.spb_perm_dense_f64_noalloc(ctypes.c_void_p(d_a.data_ptr()), n,
                                        ctypes.c_void_p(d_out.data_ptr()), None)


@pytest.mark.parametrize("n", [1, 5, 20, 28, 32, 36, 40])
def test_noalloc_matches_allocating_entry_twice(spb, n):
    import torch
    L = _lib.lib()
    a = W.dense_uniform(n, seed=900 + n)
    want = spb.perm_dense(a).permanent
    d_a = torch.from_numpy(a).cuda()
    outs = [torch.full((2,), float("nan"), dtype=torch.float64, device="cuda") for _ in range(2)]
    torch.cuda.synchronize()
    # two calls in a row on the same stream; the second reuses the array the
    # first left behind
    for d_out in outs:
        _lib.check(_call(L, d_a, n, d_out))
    torch.cuda.synchronize()
    for d_out in outs:
        hi, lo = d_out.cpu().numpy()
        assert abs(hi - want) <= REL_TOL * abs(want), (hi, want)
        assert abs(lo) <= abs(hi) * 2.0 ** -52


def test_noalloc_calls_allocate_nothing(spb):
    """With every library allocation set to fail, the calls still succeed, and
    the device's free memory does not move across them (the set-up, which
    loads the kernels, happened in a first call)."""
    import torch
    L = _lib.lib()
    sizes = [12, 24, 33, 40]
    mats = [torch.from_numpy(W.dense_uniform(n, seed=950 + n)).cuda() for n in sizes]
    outs = [torch.zeros(2, dtype=torch.float64, device="cuda") for _ in sizes]
    _lib.check(_call(L, mats[0], sizes[0], outs[0]))  # set-up on this device
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    L.spb_debug_fail_allocations(1 << 30)
    try:
        sts = [_call(L, d_a, n, d_out) for d_a, n, d_out in zip(mats, sizes, outs)]
        torch.cuda.synchronize()
    finally:
        L.spb_debug_fail_allocations(0)
    free1, _ = torch.cuda.mem_get_info()
    assert sts == [_lib.SPB_OK] * len(sizes), sts
    assert free1 == free0, (free0, free1)
    for n, d_out in zip(sizes, outs):
        hi = float(d_out[0])
        want = spb.perm_dense(W.dense_uniform(n, seed=950 + n)).permanent
        assert abs(hi - want) <= REL_TOL * abs(want), (n, hi, want)


def test_noalloc_rejects_sizes_beyond_its_array(spb):
    import torch
    L = _lib.lib()
    d_a = torch.zeros((41, 41), dtype=torch.float64, device="cuda")
    d_out = torch.zeros(2, dtype=torch.float64, device="cuda")
    st = _call(L, d_a, 41, d_out)
    assert st == _lib.SPB_ERR_INVALID
    assert "1..40" in _lib.last_error()
