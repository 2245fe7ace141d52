"""Out-of-HBM hybrid transfer: graphs whose edges stay in pinned host memory.

Every engine (resident, ExpTM-Filter, ExpTM-Compaction, ImpTM-Zero-Copy) is
forced in turn with a budget that keeps nothing or only part of the graph
resident, then the cost model chooses freely.  SSSP distances must equal the
oracle's Dijkstra bit for bit; PageRank must stay within L1 1e-5 of the FP64
oracle (the same bar as the in-HBM path).
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-5
MiB = 1 << 20


def _csc(g):
    """CSC of a host CSR by a stable sort on destination (sources ascend)."""
    V = g.num_vertices
    src = np.repeat(np.arange(V, dtype=np.uint32), np.diff(g.row_offsets.astype(np.int64)))
    order = np.argsort(g.column_indices, kind="stable")
    in_src = src[order]
    in_off = np.zeros(V + 1, np.uint64)
    np.cumsum(np.bincount(g.column_indices, minlength=V), out=in_off[1:])
    return in_off, in_src


def _dijkstra(oracle, g, source, weights=None):
    """Oracle distances as the C ABI reports them (uint32, unreachable =
    HYT_DIST_INF_U32)."""
    w = g.weights if weights is None else weights
    d = oracle.dijkstra(g.row_offsets, g.column_indices, w, source)
    inf = d == np.iinfo(np.uint64).max
    assert int(d[~inf].max(initial=0)) < 0xFFFFFFFF
    return np.where(inf, 0xFFFFFFFF, d).astype(np.uint32)


def _hybrid(hyt, g, **kw):
    in_off, in_src = _csc(g)
    return hyt.HybridGraph(g.row_offsets, g.column_indices, g.weights, in_off, in_src, **kw)


def _push_budget(g):
    """Budget whose resident share holds about half of the CSR edge bytes:
    below 8 MiB the engine reserves two 1 MiB staging slots and a 0.5 MiB
    compaction buffer, and keeps the largest partitions in what is left."""
    return 5 * MiB // 2 + g.num_edges * 4


def _pull_budget(g):
    """Same for the CSC side: two 1 MiB slots, half of the 4-byte ids."""
    return 2 * MiB + g.num_edges * 2


ENGINES = ["FILTER", "COMPACTION", "ZERO_COPY"]


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("resident", [False, True])
def test_hybrid_sssp_forced_engines_bit_exact(hyt, oracle, gpu, engine, resident):
    # scale 16 with 2^12-vertex partitions: partition 0 holds ~1/3 of the
    # edges, more than a 1 MiB staging slot, so it is staged in pieces
    g = hyt.rmat(16, 16, 21)
    sources = hyt.pick_sources(g.row_offsets, 5, 2)
    budget = _push_budget(g) if resident else 1
    with _hybrid(hyt, g, flags=hyt.capi.HYT_GRAPH_PUSH, budget_bytes=budget, partition_vertices=1 << 12,
                 force_engine=getattr(hyt.capi, "HYT_ENGINE_" + engine)) as hg:
        info = hg.info()
        assert info["partitions"] == 16
        if resident:
            assert 0 < info["resident_push_partitions"] < 16
        else:
            assert info["resident_push_partitions"] == 0
        for s in sources:
            ref = _dijkstra(oracle, g, int(s))
            d, st, ts = hg.sssp(int(s))
            assert np.array_equal(d, ref), (engine, resident, int(s))
            assert st["converged"] == 1
            n = ts[engine.lower() + "_decisions"]
            assert n > 0, ts
            others = [e for e in ENGINES if e != engine]
            assert all(ts[e.lower() + "_decisions"] == 0 for e in others if e != "ZERO_COPY"), ts
            assert ts["link_bytes"] > 0 and ts["link_gbs"] > 0
            if resident:
                assert ts["resident_decisions"] > 0


@pytest.mark.parametrize("engine", ["FILTER", "ZERO_COPY"])
@pytest.mark.parametrize("resident", [False, True])
def test_hybrid_pagerank_forced_engines(hyt, oracle, gpu, engine, resident):
    g = hyt.rmat(16, 16, 22)
    ref, it_ref, _, conv_ref = oracle.pagerank_f64(g.row_offsets, g.column_indices)
    budget = _pull_budget(g) if resident else 1
    with _hybrid(hyt, g, flags=hyt.capi.HYT_GRAPH_PULL, budget_bytes=budget, partition_vertices=1 << 12,
                 force_engine=getattr(hyt.capi, "HYT_ENGINE_" + engine)) as hg:
        info = hg.info()
        if resident:
            assert 0 < info["resident_pull_partitions"] < 16
        r, st, ts = hg.pagerank()
    l1 = float(np.abs(r.astype(np.float64) - ref).sum())
    assert l1 <= PR_L1_TOL, (engine, resident, l1)
    assert st["converged"] == conv_ref
    assert abs(st["iterations"] - it_ref) <= 1
    assert ts[engine.lower() + "_decisions"] > 0
    assert ts["rounds"] == st["iterations"]
    with hyt.Graph(g) as dg:
        r_hbm, st_hbm = dg.pagerank()
    assert st_hbm["iterations"] == st["iterations"]
    assert float(np.abs(r.astype(np.float64) - r_hbm).sum()) <= 1e-6


def test_hybrid_cost_model_mixed_decisions(hyt, oracle, gpu):
    """AUTO: with a partial budget the model picks per partition per round;
    the result does not depend on what it picked."""
    g = hyt.rmat(16, 16, 23)
    s = int(hyt.pick_sources(g.row_offsets, 9, 1)[0])
    ref = _dijkstra(oracle, g, s)
    pr_ref, _, _, _ = oracle.pagerank_f64(g.row_offsets, g.column_indices)
    with _hybrid(hyt, g, budget_bytes=2 * _push_budget(g), partition_vertices=1 << 12) as hg:
        d, st, ts = hg.sssp(s)
        assert np.array_equal(d, ref)
        decided = ts["resident_decisions"] + ts["filter_decisions"] + ts["compaction_decisions"] + \
            ts["zero_copy_decisions"]
        assert decided > 0 and ts["rounds"] == st["iterations"]
        r, pst, pts = hg.pagerank()
        assert float(np.abs(r.astype(np.float64) - pr_ref).sum()) <= PR_L1_TOL
        info = hg.info()
        assert info["h2d_gbs"] > 1 and info["zero_copy_gbs"] > 0.1 and info["gather_gbs"] > 0


def test_hybrid_everything_resident_moves_nothing(hyt, oracle, gpu):
    g = hyt.rmat(13, 16, 24)
    s = int(hyt.pick_sources(g.row_offsets, 1, 1)[0])
    with _hybrid(hyt, g) as hg:  # default 8 GiB budget holds it all
        info = hg.info()
        assert info["resident_push_partitions"] == info["partitions"] == info["resident_pull_partitions"]
        d, _, ts = hg.sssp(s)
        assert np.array_equal(d, _dijkstra(oracle, g, s))
        assert ts["link_bytes"] == 0
        _, _, pts = hg.pagerank()
        assert pts["link_bytes"] == 0


def test_hybrid_unweighted_and_special(hyt, oracle, gpu):
    g = hyt.rmat(12, 4, 25, 0, 0)  # unweighted, many dangling vertices
    s = int(hyt.pick_sources(g.row_offsets, 3, 1)[0])
    ones = np.ones(g.num_edges, np.uint32)
    for engine in (1, 2, 3):
        with _hybrid(hyt, g, budget_bytes=1, partition_vertices=1 << 8, force_engine=engine) as hg:
            d, _, _ = hg.sssp(s)
            assert np.array_equal(d, _dijkstra(oracle, g, s, ones))
            r, _, _ = hg.pagerank()
            ref, _, _, _ = oracle.pagerank_f64(g.row_offsets, g.column_indices)
            assert float(np.abs(r.astype(np.float64) - ref).sum()) <= PR_L1_TOL


def test_copy_csc_matches_restatement(hyt, gpu):
    g = hyt.rmat(15, 16, 26)
    in_off, in_src = _csc(g)
    with hyt.Graph(g) as dg:
        off, src = dg.copy_csc()
    assert np.array_equal(off, in_off)
    assert np.array_equal(src, in_src)


def test_hybrid_errors(hyt, gpu):
    g = hyt.rmat(10, 8, 27)
    with pytest.raises(hyt.HytError) as e:
        hyt.HybridGraph(g.row_offsets, g.column_indices, g.weights, flags=hyt.capi.HYT_GRAPH_PULL)
    assert e.value.code == hyt.capi.HYT_E_INVALID
    with pytest.raises(hyt.HytError):
        _hybrid(hyt, g, partition_vertices=1000)
    with pytest.raises(hyt.HytError):
        _hybrid(hyt, g, force_engine=7)
    with _hybrid(hyt, g, flags=hyt.capi.HYT_GRAPH_PUSH) as hg:
        with pytest.raises(hyt.HytError):
            hg.pagerank()
        with pytest.raises(hyt.HytError):
            hg.sssp(g.num_vertices)
