"""Batched queries: many SSSP / personalized-PageRank queries over graphs of
uneven sizes in one CUDA-graph launch.

Bars: SSSP distances identical to the single-query solver and to the
oracle's Dijkstra; PPR within L1 1e-5 of the FP64 oracle and 1e-6 of the
single-query solver; every result identical whether its query runs alone
or in the mix (the engine's per-query sums have a fixed association).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-5


def _inf_u32(d):
    inf = d == np.iinfo(np.uint64).max
    return np.where(inf, 0xFFFFFFFF, d).astype(np.uint32)


@pytest.fixture(scope="module")
def world(hyt):
    specs = [(10, 8, 1), (12, 16, 2), (13, 32, 3), (11, 4, 4), (14, 16, 5), (9, 24, 6)]
    csrs = [hyt.rmat(s, ef, seed) for s, ef, seed in specs]
    csrs.append(hyt.rmat(11, 8, 7, 0, 0))  # unweighted
    graphs = [hyt.Graph(c) for c in csrs]
    rng = np.random.default_rng(11)
    queries = []
    for gi, c in enumerate(csrs):
        for s in hyt.pick_sources(c.row_offsets, 100 + gi, int(rng.integers(1, 7))):
            kind = "sssp" if rng.random() < 0.6 else "ppr"
            queries.append({"graph": gi, "kind": kind, "source": int(s)})
    yield csrs, graphs, queries
    for g in graphs:
        g.close()


def test_batch_matches_single_solvers_and_oracle(hyt, oracle, gpu, world):
    csrs, graphs, queries = world
    with hyt.Batch(graphs) as b:
        outs, res, st = b.run(queries)
    assert st["waves"] == 1 and st["graph_launches"] == 1 and st["supersteps"] > 0
    checked_oracle = 0
    for q, out, r in zip(queries, outs, res):
        c, g = csrs[q["graph"]], graphs[q["graph"]]
        assert r["converged"] == 1, (q, r)
        if q["kind"] == "sssp":
            single, _ = g.sssp(q["source"])
            assert np.array_equal(out, single), q
            if checked_oracle < 6:
                w = c.weights if c.weights is not None else np.ones(c.num_edges, np.uint32)
                assert np.array_equal(out, _inf_u32(oracle.dijkstra(c.row_offsets, c.column_indices, w, q["source"])))
                checked_oracle += 1
        else:
            single, sst = g.ppr(q["source"])
            assert float(np.abs(out.astype(np.float64) - single).sum()) <= 1e-6, q
            assert abs(r["iterations"] - sst["iterations"]) <= 1
            ref, _, _, _ = oracle.ppr_f64(c.row_offsets, c.column_indices, q["source"])
            assert float(np.abs(out.astype(np.float64) - ref).sum()) <= PR_L1_TOL, q


def test_batch_alone_equals_mix(hyt, gpu, world):
    csrs, graphs, queries = world
    with hyt.Batch(graphs) as b:
        mixed, mres, _ = b.run(queries)
        for i in range(0, len(queries), 3):
            alone, ares, _ = b.run([queries[i]])
            if queries[i]["kind"] == "ppr":  # SSSP round counts depend on in-round propagation order
                assert ares[0]["iterations"] == mres[i]["iterations"]
            assert np.array_equal(alone[0].view(np.uint32), mixed[i].view(np.uint32)), queries[i]


def test_batch_waves_host_loop_and_delta(hyt, gpu, world):
    csrs, graphs, queries = world
    with hyt.Batch(graphs) as b:
        ref, _, _ = b.run(queries)
    # a budget that holds only a few queries at a time -> several waves
    with hyt.Batch(graphs, state_budget_bytes=1 << 20) as b:
        outs, _, st = b.run(queries)
    assert st["waves"] > 1
    for x, y in zip(outs, ref):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    # host-driven supersteps and bucketed SSSP give the same answers
    with hyt.Batch(graphs, flags=hyt.capi.HYT_RUN_NO_GRAPH, delta_mult=4, hub_degree=32) as b:
        outs, _, st = b.run(queries)
    assert st["graph_launches"] == 0
    for q, x, y in zip(queries, outs, ref):
        if q["kind"] == "sssp":
            assert np.array_equal(x, y)
        else:
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32))


def test_batch_autotune(hyt, gpu, world):
    csrs, graphs, queries = world
    with hyt.Batch(graphs) as b:
        ref, _, _ = b.run(queries)
        t = b.autotune(queries)
        assert t["delta_mult"] in (0, 2, 8, 32) and t["hub_degree"] in (32, 64, 128, 256)
        outs, _, _ = b.run(queries)
    for q, x, y in zip(queries, outs, ref):
        if q["kind"] == "sssp":
            assert np.array_equal(x, y)
        else:
            assert float(np.abs(x.astype(np.float64) - y).sum()) <= 1e-6


def test_batch_autotune_cache_per_size_class(hyt, gpu, world):
    """A second autotune on a sample of the same size class (here the same
    queries, in another batch handle) reuses the cached choice: same tuning,
    no timing runs."""
    import time

    csrs, graphs, queries = world
    # PPR-only samples: a size class (SSSP share 0) no other test tunes
    ppr = [dict(q, kind="ppr") for q in queries[:24]]
    with hyt.Batch(graphs) as b:
        t0 = time.perf_counter()
        first = b.autotune(ppr)
        t_first = time.perf_counter() - t0
    with hyt.Batch(graphs) as b2:
        t0 = time.perf_counter()
        again = b2.autotune(ppr[::-1])
        t_again = time.perf_counter() - t0
        b2.run(ppr[:4])
    assert again == first
    assert t_again < t_first / 5, (t_again, t_first)


def test_batch_errors(hyt, gpu, world):
    csrs, graphs, queries = world
    pull_only = hyt.Graph(csrs[0], flags=hyt.capi.HYT_GRAPH_PULL)
    with hyt.Batch(graphs + [pull_only]) as b:
        for bad in ({"graph": 99, "kind": "sssp", "source": 0},
                    {"graph": 0, "kind": "sssp", "source": csrs[0].num_vertices},
                    {"graph": len(graphs), "kind": "sssp", "source": 0},
                    {"graph": 0, "kind": "ppr", "source": 0, "restart": 1.5}):
            with pytest.raises(hyt.HytError) as e:
                b.run([bad])
            assert e.value.code == hyt.capi.HYT_E_INVALID
        # the handle stays usable after a rejected batch
        outs, res, _ = b.run(queries[:3])
        assert all(r["converged"] for r in res)
    pull_only.close()
    with pytest.raises(hyt.HytError):
        hyt.Batch([])
