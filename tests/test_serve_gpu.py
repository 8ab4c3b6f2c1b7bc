"""The serving loop (spb_server_*) through the C ABI: every result in a mixed
stream equals the same matrix computed alone, with and without captured
graphs; served results of the seeded serving stream (n up to 32, real and
complex) match their exact permanents; real matrices with zeros are served
as decomposed pieces and match the reference flow; mid-size requests go to
whichever path their queue favours; admission, cancellation and shutdown
behave."""
import json
import os

import numpy as np
import pytest

from superman_b200 import SupermanError, _lib
from superman_b200 import workloads as W
from superman_b200.serving import Server

pytestmark = pytest.mark.gpu

REL_TOL = 1e-12  # same bar as the single-matrix parity tests


def mixed_stream(count, n_lo, n_hi, seed):
    rng = np.random.default_rng(seed)
    unitaries = [W.haar_unitary(64, seed + k) for k in range(3)]
    out = []
    for i in range(count):
        n = int(rng.integers(n_lo, n_hi + 1))
        if rng.random() < 0.5:
            out.append(W.dense_uniform(n, seed * 100000 + i))
        else:
            u = unitaries[i % 3]
            r0, c0 = rng.integers(0, 64 - n + 1, size=2)
            out.append(np.ascontiguousarray(u[r0:r0 + n, c0:c0 + n]))
    return out


def alone(spb, a):
    return spb.perm_complex(a).permanent if np.iscomplexobj(a) else spb.perm_dense(a).permanent


@pytest.mark.parametrize("use_graphs", [True, False])
def test_mixed_stream_matches_alone(spb, use_graphs):
    mats = mixed_stream(240, 3, 26, seed=7)
    with Server(max_batch=64, use_graphs=use_graphs) as srv:
        tickets = [srv.submit(a) for a in mats]
        results = [srv.wait(t, timeout_s=120) for t in tickets]
        st = srv.stats()
    for a, r in zip(mats, results):
        assert r["status"] == 0
        want = alone(spb, a)
        assert abs(r["permanent"] - want) <= REL_TOL * abs(want), (a.shape, r["permanent"], want)
        assert r["latency_s"] >= 0
    assert st["completed"] == len(mats)
    assert st["batches"] >= 1 and st["large_launches"] >= 1
    if use_graphs:
        assert st["graph_launches"] <= st["batches"]
    else:
        assert st["graph_launches"] == 0 and st["graphs_captured"] == 0


def test_repeated_shape_is_replayed_from_a_graph(spb):
    """A batch shape is captured once it has been used a few times; the
    replayed batches give the same results as the single calls."""
    mats = [W.dense_uniform(12, 300 + k) for k in range(16)]
    with Server(max_batch=64) as srv:
        results = [srv.wait(srv.submit(a), timeout_s=120) for a in mats]
        st = srv.stats()
    assert st["graphs_captured"] >= 1 and st["graph_launches"] >= 1
    for a, r in zip(mats, results):
        want = spb.perm_dense(a).permanent
        assert abs(r["permanent"] - want) <= REL_TOL * abs(want)


def test_same_matrix_alone_and_in_batch(spb):
    a = W.dense_uniform(16, 99)
    with Server(max_batch=256) as srv:
        t_alone = srv.submit(a)
        r_alone = srv.wait(t_alone)
        others = [srv.submit(W.dense_uniform(16, 1000 + k)) for k in range(100)]
        t_mix = srv.submit(a)
        more = [srv.submit(W.dense_uniform(16, 2000 + k)) for k in range(100)]
        r_mix = srv.wait(t_mix)
        for t in others + more:
            srv.wait(t)
    assert r_mix["permanent"] == r_alone["permanent"]  # bit-identical: own warp, own reduction


def test_admission_refuses_beyond_budget(spb):
    with Server(admit_bytes=16 * 1024) as srv:
        big = W.dense_uniform(46, 1)  # 16.9 KB
        with pytest.raises(SupermanError) as e:
            srv.submit(big)
        assert e.value.status == _lib.SPB_ERR_BUSY
        assert srv.stats()["rejected"] == 1
        t = srv.submit(W.dense_uniform(10, 2))
        assert srv.wait(t)["status"] == 0


def test_cancel_and_shutdown(spb):
    srv = Server()
    ts = [srv.submit(W.dense_uniform(29, k)) for k in range(4)]
    srv.cancel(ts[-1])
    r = srv.wait(ts[-1])
    assert r["status"] in (0, _lib.SPB_ERR_CANCELLED)
    for t in ts[:-1]:
        assert srv.wait(t)["status"] == 0
    # queued work at shutdown is cancelled, not left hanging
    for k in range(8):
        srv.submit(W.dense_uniform(28, 50 + k))
    srv.close()


def test_invalid_ticket_and_sizes(spb):
    with Server() as srv:
        with pytest.raises(SupermanError) as e:
            srv.poll(123456789)
        assert e.value.status == _lib.SPB_ERR_INVALID
        with pytest.raises(SupermanError):
            srv.submit(np.zeros((64, 64)))


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _serve_sample():
    """(matrix, exact, entry) for each request of the seeded serving stream
    whose exact permanent is in tests/golden/serve_sample.json."""
    from fractions import Fraction
    g = json.load(open(os.path.join(GOLDEN, "serve_sample.json")))
    cfg = g["stream"]
    stream = W.ServeStream(cfg["n_lo"], cfg["n_hi"], cfg["count"], cfg["seed"])
    out = []
    for e in g["entries"]:
        a = stream.matrix(e["index"])
        assert W.matrix_sha256(a) == e["sha256"], f"request {e['index']} rebuilt differently"
        ex = (Fraction(e["exact_re"]), Fraction(e["exact_im"])) if e["kind"] == "complex" else Fraction(e["exact"])
        out.append((a, ex, e))
    return out


def test_served_stream_sample_matches_exact(spb, oracle):
    """Config C5's accuracy bar: the sampled requests (n = 8 .. 32, real U[0,1)
    and Haar-unitary blocks), served in a mix with other requests of the same
    stream, are within 1e-12 of their exact permanents."""
    sample = _serve_sample()
    assert max(e["n"] for _, _, e in sample) >= 29
    stream = W.ServeStream(8, 32, 20000)
    fill = [stream.matrix(i) for i in range(400, 520) if stream.meta[i][0] <= 24]
    with Server() as srv:
        tickets = []
        for k, (a, _, _) in enumerate(sample):
            tickets.append(srv.submit(a))
            for b in fill[k * 4:(k + 1) * 4]:
                srv.submit(b)
        results = [srv.wait(t, timeout_s=300) for t in tickets]
    worst = 0.0
    for (a, exact, e), r in zip(sample, results):
        assert r["status"] == 0
        err = oracle.rel_err(r["permanent"], exact)
        worst = max(worst, err)
        assert err <= REL_TOL, (e["index"], e["n"], e["kind"], err)
    print(f"served sample: {len(sample)} requests, max rel err vs exact {worst:.2e}")


def test_sparse_request_is_decomposed_and_matches_pipeline(spb, oracle):
    """Config C3's n=40 matrix served as one request: the server prunes and
    decomposes it as the reference's main flow does (3 pieces of n=30) and
    returns the product over components of the sum of the pieces; it equals
    the synchronous pipeline and the exact value."""
    import ctypes
    from conftest import load_golden
    a, exact, _ = load_golden("sparse_n40_s5")
    out = _lib.spb_pipeline_result()
    arr = (ctypes.c_char_p * 1)(b"calculation_precision=dd")
    _lib.check(_lib.lib().spb_perm_pipeline(a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), 40, arr, 1,
                                            ctypes.byref(out)))
    with Server() as srv:
        r = srv.wait(srv.submit(a), timeout_s=120)
        st = srv.stats()
    assert r["status"] == 0
    assert st["split_requests"] == 1 and st["pieces"] == out.pieces == 3
    assert abs(r["permanent"] - out.permanent) <= REL_TOL * abs(out.permanent)
    assert oracle.rel_err(r["permanent"], exact) <= REL_TOL


def test_decomposed_components_multiply(spb, oracle):
    """A block-diagonal matrix with zeros is served as its components'
    product; a matrix without a perfect matching is served as 0."""
    rng = np.random.default_rng(5)
    a = np.zeros((18, 18))
    a[:10, :10] = rng.random((10, 10))
    a[10:, 10:] = rng.random((8, 8))
    p = rng.permutation(18)
    a = a[p][:, rng.permutation(18)]
    z = rng.random((12, 12))
    z[:, 3] = 0.0  # an empty column: no perfect matching
    with Server() as srv:
        ra = srv.wait(srv.submit(a))
        rz = srv.wait(srv.submit(z))
        st = srv.stats()
    assert st["split_requests"] == 2
    assert ra["status"] == 0 and oracle.rel_err(ra["permanent"], oracle.exact_perm(a)) <= REL_TOL
    assert rz["status"] == 0 and rz["permanent"] == 0.0


def test_mid_size_requests_take_the_favoured_path(spb):
    """A lone n=22 request runs as a whole-GPU call; a burst of n=21 requests
    of one shape is batched.  Both match their single calls."""
    lone = W.dense_uniform(22, 77)
    burst = [W.dense_uniform(21, 800 + k) for k in range(64)]
    with Server(max_wait_s=1e-3) as srv:
        r_lone = srv.wait(srv.submit(lone), timeout_s=60)
        st0 = srv.stats()
        ts = srv.submit_many(burst)
        rs = [srv.wait(t, timeout_s=120) for t in ts]
        st1 = srv.stats()
    assert st0["mid_to_large"] >= 1 and st0["large_launches"] >= 1
    assert st1["batched_requests"] >= 16
    want = spb.perm_dense(lone, precision="dd").permanent
    assert abs(r_lone["permanent"] - want) <= REL_TOL * abs(want)
    for a, r in zip(burst, rs):
        want = spb.perm_dense(a).permanent
        assert abs(r["permanent"] - want) <= REL_TOL * abs(want)


def test_admission_counts_device_pool_bytes(spb):
    """Admission reserves each request's matrix in the device pool until it
    completes: a pool of 64 KiB takes eight 32 x 32 real matrices (8 KiB
    each) at most while they are queued, and frees them on completion."""
    mats = [W.dense_uniform(32, 60 + k) for k in range(12)]
    with Server(admit_bytes=64 * 1024, large_workers=1) as srv:
        got = srv.submit_many(mats)
        admitted = [t for t in got if t]
        st = srv.stats()
        assert 1 <= len(admitted) <= 8
        assert st["rejected"] == len(mats) - len(admitted)
        assert st["pool_bytes"] >= 64 * 1024
        for t in admitted:
            assert srv.wait(t, timeout_s=120)["status"] == 0
        assert srv.stats()["queued_bytes"] == 0
        # room again once they completed
        assert srv.wait(srv.submit(mats[-1]), timeout_s=120)["status"] == 0
