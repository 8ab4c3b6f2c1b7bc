"""The fused small-matrix call (one cooperative kernel for real 4 <= n <= 26:
tables, walk, threshold and double-double refinement) against the same call
made of separate kernels, and against the exact value."""
import numpy as np
import pytest

from superman_b200 import workloads as W
from conftest import load_golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [4, 5, 9, 13, 17, 20, 22, 24, 25])
def test_fused_equals_separate_fp64(spb, n):
    """FP64 mode at one launch shape: the same walk, unit split and reduction
    order, so the same bits.  At the default shapes (the fused call spreads
    n >= 19 over every SM with smaller CTAs) the unit split differs, so only
    the value is compared."""
    a = W.dense_uniform(n, 700 + n)
    f = spb.perm_dense(a, precision="fp64", threads_per_block=448, blocks=148)
    s = spb.perm_dense(a, precision="fp64", threads_per_block=448, blocks=148, small_call=-1)
    assert f.launches == 1 and s.launches >= 2
    assert (f.permanent, f.permanent_lo) == (s.permanent, s.permanent_lo)
    fd = spb.perm_dense(a, precision="fp64")
    sd = spb.perm_dense(a, precision="fp64", small_call=-1)
    assert fd.launches == 1
    assert abs(fd.permanent - sd.permanent) <= 1e-13 * abs(sd.permanent)


@pytest.mark.parametrize("n,threads", [(12, 96), (20, 160), (20, 384), (22, 448), (24, 448), (24, 384)])
def test_fused_launch_shapes(spb, oracle, n, threads):
    """CTAs of fewer threads: the grid takes the units in passes (thread t
    owns units t, t + T, ...), one launch, exact to the bar."""
    a = W.dense_uniform(n, 720 + n)
    r = spb.perm_dense(a, precision="dd", threads_per_block=threads)
    assert r.launches == 1
    assert oracle.rel_err(r.permanent + r.permanent_lo, oracle.exact_perm(a)) <= 1e-13


@pytest.mark.parametrize("n", [6, 12, 18, 21, 24, 25, 26])
def test_fused_dd_matches_separate_and_exact(spb, oracle, n):
    a = W.dense_uniform(n, 710 + n)
    f = spb.perm_dense(a, precision="dd")
    s = spb.perm_dense(a, precision="dd", small_call=-1)
    assert f.launches == 1
    assert f.refined_units == s.refined_units
    assert abs(f.permanent - s.permanent) <= 1e-15 * abs(s.permanent)
    # rel_tol (1e-13 by default) is a statistical target: this n=26 matrix
    # lands at 2.0e-13 on both paths, inside the 1e-12 bar
    bar = 1e-13 if n <= 25 else 1e-12
    assert oracle.rel_err(f.permanent + f.permanent_lo, oracle.exact_perm(a)) <= bar


def test_fused_dd_golden_n24(spb, oracle):
    a, exact, _ = load_golden("dense_u01_n24_s3")
    f = spb.perm_dense(a, precision="dd")
    assert f.launches == 1 and f.refined_units > 0
    assert oracle.rel_err(f.permanent, exact) <= 1e-13


def test_fused_dd_forced_refinement_signed(spb, oracle):
    """Signed entries and a tight tolerance: many units refined inside the
    fused call, still exact to the bar."""
    rng = np.random.default_rng(31)
    a = rng.standard_normal((20, 20))
    f = spb.perm_dense(a, precision="dd", rel_tol=1e-16)
    s = spb.perm_dense(a, precision="dd", rel_tol=1e-16, small_call=-1)
    assert f.launches == 1 and f.refined_units == s.refined_units > 0
    exact = oracle.exact_perm(a)
    assert oracle.rel_err(f.permanent, exact) <= 1e-12
    assert abs(f.permanent - s.permanent) <= 1e-14 * abs(exact)


def test_fused_device_input_and_edge_values(spb):
    """Device-resident input, a zero row (permanent 0) and rows scaled far
    apart go through the fused call like the separate kernels."""
    import ctypes
    import torch
    from superman_b200 import _lib
    a = W.dense_uniform(16, 3)
    d = torch.from_numpy(a).cuda()
    out = _lib.spb_result()
    opt = _lib.default_options(precision=_lib.SPB_PREC_DD)
    _lib.check(_lib.lib().spb_perm_dense_f64_dev(ctypes.c_void_p(d.data_ptr()), 16, ctypes.byref(opt),
                                                 ctypes.byref(out)))
    assert out.launches == 1
    want = spb.perm_dense(a, precision="dd", small_call=-1).permanent
    assert abs(out.value - want) <= 1e-15 * abs(want)
    z = W.dense_uniform(14, 4)
    z[5] = 0.0
    assert spb.perm_dense(z, sparse_walk=1).permanent == 0.0
    sc = np.full((12, 12), 0.75)
    sc[:6] *= 2.0 ** 900
    sc[6:] *= 2.0 ** -900
    r = spb.perm_dense(sc, precision="dd")
    import math
    assert abs(r.permanent - math.factorial(12) * 0.75 ** 12) <= 1e-13 * r.permanent


def test_fused_graph_replay_reads_each_matrix(spb, oracle):
    """Repeated calls of one size replay the fused call as a CUDA graph, which
    copies the matrix from the library's page-locked staging area: every call
    must see its own matrix (host input) or its own device pointer."""
    import ctypes
    import torch
    from superman_b200 import _lib
    mats = [W.dense_uniform(20, 900 + k) for k in range(3)]
    want = [spb.perm_dense(m, precision="dd", small_call=-1).permanent for m in mats]
    for _ in range(3):  # first sight runs directly, then the graph replays
        for m, w in zip(mats, want):
            r = spb.perm_dense(m, precision="dd")
            assert r.launches == 1
            assert abs(r.permanent - w) <= 1e-15 * abs(w)
    devs = [torch.from_numpy(m).cuda() for m in mats[:2]]
    opt = _lib.default_options(precision=_lib.SPB_PREC_DD)
    out = _lib.spb_result()
    for _ in range(3):
        for d, w in zip(devs, want[:2]):
            _lib.check(_lib.lib().spb_perm_dense_f64_dev(ctypes.c_void_p(d.data_ptr()), 20, ctypes.byref(opt),
                                                         ctypes.byref(out)))
            assert abs(out.value - w) <= 1e-15 * abs(w)
            assert out.device_s > 0.0 and out.kernel_s > 0.0 and out.kernel_s <= out.device_s
    assert oracle.rel_err(want[0], oracle.exact_perm(mats[0])) <= 1e-13


@pytest.mark.parametrize("n", [16, 24, 26, 28])
def test_skip_timing_same_result(spb, n):
    """skip_timing drops the device timing only: the same permanent (to the
    last bits the order of the refinement's corrections can move), with
    kernel_s reported as 0 (fused call at n <= 26, separate kernels above)."""
    a = W.dense_uniform(n, 930 + n)
    t = spb.perm_dense(a, precision="dd")
    for _ in range(3):  # direct, then graph-replayed for the fused call
        u = spb.perm_dense(a, precision="dd", skip_timing=1)
        assert abs(u.permanent - t.permanent) <= 1e-15 * abs(t.permanent)
        assert u.kernel_s == 0.0
    assert t.kernel_s > 0.0


def test_skip_timing_complex(spb):
    """skip_timing on the complex entry point: the same value, no device
    timing."""
    c = W.haar_block(14, seed=14, N=32)
    t = spb.perm_complex(c, precision="dd")
    u = spb.perm_complex(c, precision="dd", skip_timing=1)
    assert abs(u.permanent - t.permanent) <= 1e-14 * abs(t.permanent)
    assert u.kernel_s == 0.0 and t.kernel_s > 0.0
