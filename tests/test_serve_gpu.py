"""The serving loop (spb_server_*) through the C ABI: every result in a mixed
stream equals the same matrix computed alone, with and without captured
graphs; admission, cancellation and shutdown behave."""
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
