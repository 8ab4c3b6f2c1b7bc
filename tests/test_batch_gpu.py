"""Batched small permanents (spb_perm_batch_dev, one warp per matrix) through
the C ABI: each matrix of a batch against the exact oracle and against the
single-matrix entry point."""
import ctypes

import numpy as np
import pytest

from superman_b200 import _lib
from superman_b200 import workloads as W

pytestmark = pytest.mark.gpu


def run_batch(mats, is_complex):
    import torch
    mats = np.ascontiguousarray(mats)
    count, n = mats.shape[0], mats.shape[1]
    flat = mats.view(np.float64) if is_complex else mats
    d_in = torch.from_numpy(flat.copy()).cuda()
    comps = 2 if is_complex else 1
    d_out = torch.full((count * 2 * comps,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().spb_perm_batch_dev(ctypes.c_void_p(d_in.data_ptr()), n, int(is_complex), count,
                                             ctypes.c_void_p(d_out.data_ptr()), None))
    torch.cuda.synchronize()
    o = d_out.cpu().numpy().reshape(count, comps, 2)
    if is_complex:
        return o[:, 0, 0] + 1j * o[:, 1, 0]
    return o[:, 0, 0]


@pytest.mark.parametrize("n", [1, 2, 3, 4, 7, 8, 12, 16])
def test_batch_real_exact(spb, oracle, n):
    count = 37
    mats = np.stack([W.dense_uniform(n, seed=1000 * n + k) for k in range(count)])
    got = run_batch(mats, False)
    for k in range(count):
        assert oracle.rel_err(got[k], oracle.exact_perm(mats[k])) <= 1e-13


@pytest.mark.parametrize("n", [18, 20, 22, 24])
def test_batch_real_matches_single(spb, n):
    count = 9
    rng = np.random.default_rng(n)
    mats = np.stack([W.dense_uniform(n, seed=77 * n + k) for k in range(count - 1)] +
                    [rng.standard_normal((n, n))])
    got = run_batch(mats, False)
    for k in range(count):
        want = spb.perm_dense(mats[k]).permanent
        scale = float(np.prod(np.abs(mats[k]).sum(axis=1)))
        assert abs(got[k] - want) <= 1e-13 * max(abs(want), 1e-300) or abs(got[k] - want) <= 1e-14 * scale


@pytest.mark.parametrize("n", [1, 2, 5, 11, 16, 20, 21, 23, 24])
def test_batch_complex(spb, oracle, n):
    count = 6
    mats = np.stack([W.haar_block(n, seed=500 + k, N=64) for k in range(count)])
    got = run_batch(mats, True)
    for k in range(count):
        if n <= 16:
            want = oracle.exact_perm_complex(mats[k])
            err = oracle.rel_err(got[k], want)
        else:
            s = spb.perm_complex(mats[k]).permanent
            err = abs(got[k] - s) / abs(s)
        assert err <= 1e-12


def test_batch_empty_and_invalid(spb):
    import torch
    L = _lib.lib()
    d = torch.zeros(4, dtype=torch.float64, device="cuda")
    assert L.spb_perm_batch_dev(ctypes.c_void_p(d.data_ptr()), 5, 0, 0, ctypes.c_void_p(d.data_ptr()), None) == 0
    assert L.spb_perm_batch_dev(ctypes.c_void_p(d.data_ptr()), 25, 0, 1, ctypes.c_void_p(d.data_ptr()),
                                None) == _lib.SPB_ERR_INVALID
