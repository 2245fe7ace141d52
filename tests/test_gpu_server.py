"""Serving: continuous batching of arriving queries.

Queries submitted while others run are admitted at the next superstep and
share its kernels; each result must equal the same query run alone
(SSSP identical to hyt_sssp, PPR identical to a one-query batch), and a
short query that arrives after a long one must be able to finish first.
"""
from __future__ import annotations

import threading
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served(hyt):
    csrs = [hyt.rmat(s, 16, 40 + s) for s in (10, 12, 14, 16)]
    graphs = [hyt.Graph(c) for c in csrs]
    yield csrs, graphs
    for g in graphs:
        g.close()


def _drain(srv, n, timeout_s=60.0):
    got = []
    t0 = time.time()
    while len(got) < n and time.time() - t0 < timeout_s:
        got += srv.poll(256, wait_ms=50)
    assert len(got) == n, (len(got), n, srv.stats())
    return got


def test_server_results_equal_alone(hyt, gpu, served):
    csrs, graphs = served
    rng = np.random.default_rng(3)
    reqs = []
    for i in range(80):
        gi = int(rng.integers(0, len(graphs)))
        kind = "sssp" if rng.random() < 0.7 else "ppr"
        src = int(hyt.pick_sources(csrs[gi].row_offsets, 500 + i, 1)[0])
        reqs.append((gi, kind, src))
    gaps = rng.exponential(0.0005, len(reqs))
    with hyt.Server(graphs) as srv:
        tickets = {}

        def client():  # open-loop arrivals, ~1 every 0.5 ms
            for r, gap in zip(reqs, gaps):
                tickets[srv.submit(*r)] = r
                time.sleep(float(gap))

        th = threading.Thread(target=client)
        th.start()
        got = _drain(srv, len(reqs))
        th.join()
        st = srv.stats()
    assert st["completed"] == len(reqs) and st["max_running"] > 1
    with hyt.Batch(graphs) as b:
        for c in got:
            assert c["status"] == 0
            gi, kind, src = tickets[c["ticket"]]
            alone, res, _ = b.run([{"graph": gi, "kind": kind, "source": src}])
            assert np.array_equal(c["out"].view(np.uint32), alone[0].view(np.uint32)), (gi, kind, src)
            if kind == "ppr":  # SSSP round counts depend on in-round propagation order; distances do not
                assert c["result"]["iterations"] == res[0]["iterations"]
            else:
                single, _ = graphs[gi].sssp(src)
                assert np.array_equal(c["out"], single)
            assert c["latency_ms"] >= c["queue_ms"] >= 0.0


def test_server_packs_equal_alone(hyt, gpu, served):
    """Queries on graphs at or above pack_min_edges run in packs of up to 8
    (hyt_sssp_multi / hyt_ppr_multi) next to the engine's queries on the
    smaller graphs.  SSSP labels equal hyt_sssp's; a packed PPR equals the
    same query packed alone (hyt_ppr_multi's result does not depend on its
    companions) and lies within L1 1e-5 of hyt_ppr (both are within 1e-5 of
    the FP64 definition)."""
    csrs, graphs = served
    rng = np.random.default_rng(11)
    reqs = []
    for i in range(60):
        gi = int(rng.integers(0, len(graphs)))
        kind = "sssp" if rng.random() < 0.6 else "ppr"
        src = int(hyt.pick_sources(csrs[gi].row_offsets, 900 + i, 1)[0])
        reqs.append((gi, kind, src))
    # the two larger graphs pack, the two smaller go through the engine
    with hyt.Server(graphs, pack_min_edges=csrs[2].num_edges) as srv:
        tickets = {srv.submit(*r): r for r in reqs}
        got = _drain(srv, len(reqs))
        st = srv.stats()
    assert st["packs"] > 0 and st["completed"] == len(reqs)
    assert st["packs"] < sum(1 for g, _, _ in reqs if g >= 2)  # some packs held several queries
    for c in got:
        assert c["status"] == 0
        gi, kind, src = tickets[c["ticket"]]
        if kind == "sssp":
            single, _ = graphs[gi].sssp(src)
            assert np.array_equal(c["out"], single), (gi, src)
        elif gi >= 2:
            alone, _ = graphs[gi].ppr_multi([src])
            assert np.array_equal(c["out"].view(np.uint32), alone[0].view(np.uint32)), (gi, src)
            one, _ = graphs[gi].ppr(src)
            assert float(np.abs(c["out"].astype(np.float64) - one).sum()) <= 1e-5


def test_server_short_query_overtakes_long(hyt, gpu, served):
    csrs, graphs = served
    big = len(graphs) - 1
    with hyt.Server(graphs) as srv:
        src = int(hyt.pick_sources(csrs[big].row_offsets, 9, 1)[0])
        # tolerance far below FP32 resolution: runs for thousands of iterations
        t_long = srv.submit(big, "ppr", src, tolerance=1e-30, max_iterations=3000)
        t0 = time.time()
        while srv.stats()["running"] == 0 and time.time() - t0 < 5:
            time.sleep(0.0005)
        small = int(hyt.pick_sources(csrs[0].row_offsets, 9, 1)[0])
        t_short = srv.submit(0, "sssp", small)
        got = _drain(srv, 2)
    order = [c["ticket"] for c in got]
    assert order.index(t_short) < order.index(t_long), got
    assert all(c["status"] == 0 for c in got)


def test_server_budget_queueing_and_rejection(hyt, gpu, served):
    csrs, graphs = served
    # room for about one scale-16 query at a time: the rest wait in the queue
    with hyt.Server(graphs, state_budget_bytes=3 << 20) as srv:
        srcs = hyt.pick_sources(csrs[3].row_offsets, 77, 6)
        for s in srcs:
            srv.submit(3, "sssp", int(s))
        got = _drain(srv, len(srcs))
        st = srv.stats()
    assert all(c["status"] == 0 for c in got)
    assert st["peak_state_bytes"] <= 3 << 20
    for c, s in zip(sorted(got, key=lambda c: c["ticket"]), srcs):
        single, _ = graphs[3].sssp(int(s))
        assert np.array_equal(c["out"], single)
    # a query whose state can never fit completes with HYT_E_OOM
    with hyt.Server(graphs, state_budget_bytes=64 << 10) as srv:
        srv.submit(3, "sssp", int(srcs[0]))
        got = _drain(srv, 1)
    assert got[0]["status"] == hyt.capi.HYT_E_OOM


def test_server_rejects_bad_queries(hyt, gpu, served):
    csrs, graphs = served
    with hyt.Server(graphs) as srv:
        with pytest.raises(hyt.HytError) as e:
            srv.submit(0, "sssp", csrs[0].num_vertices)
        assert e.value.code == hyt.capi.HYT_E_INVALID
        with pytest.raises(hyt.HytError):
            srv.submit(17, "sssp", 0)
        t = srv.submit(0, "ppr", int(hyt.pick_sources(csrs[0].row_offsets, 1, 1)[0]))
        got = _drain(srv, 1)
        assert got[0]["ticket"] == t and got[0]["status"] == 0
