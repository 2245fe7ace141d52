"""GPU parity of the vertex-range shard kernels (hyt_shard_*).

One GPU holds every shard of a split here: the shards share the
whole-graph vectors, so their steps (one after another on one stream) need
no exchange, and the results must equal the single-GPU solvers'.
PageRank / personalized PageRank: the same iteration count and L1 <= 1e-6
against hyt_pagerank / hyt_ppr (L1 <= 1e-5 against the FP64 oracle); SSSP:
bit for bit.  The last test runs ShardedGraph through a one-process NCCL
group (the collectives of the multi-GPU path, on one rank)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-5


def _csr(off, cols, w=None):
    import hytgraph_b200 as hyt

    w = None if w is None else np.asarray(w, np.uint32)
    return hyt.CSR(np.asarray(off, np.uint64), np.asarray(cols, np.uint32), w)


def _graphs(hyt):
    out = [(hyt.rmat(14, 16, 21), 0), (hyt.rmat(13, 8, 22), hyt.capi.HYT_GRAPH_HUB_ORDER),
           (hyt.rmat(11, 4, 23, 0, 0), 0)]
    out += [(_csr([0, 0], []), 0), (_csr([0, 0, 0, 0, 0], []), 0), (_csr([0, 1, 2, 3], [1, 2, 0], [1, 1, 1]), 0)]
    n = 20000  # star in and out of vertex 0: long rows split into chunk tasks, hub segments
    off = np.concatenate([[0, n - 1], np.arange(n - 1) + n]).astype(np.uint64)
    cols = np.concatenate([np.arange(1, n), np.zeros(n - 1)]).astype(np.uint32)
    out.append((_csr(off, cols, (np.arange(cols.shape[0]) % 63 + 1).astype(np.uint32)), 0))
    return out


def _pull(dg, parts, personalized=False, source=0, damping=0.85, tol=1e-6, max_iter=100):
    """Every shard of a `parts`-way split, stepped on one GPU."""
    import torch

    from hytgraph_b200.shard import CudaShardKernels, PageRankVectors

    ks = [CudaShardKernels(dg, p, parts) for p in range(parts)]
    V = dg.num_vertices
    rank = [torch.empty(V, dtype=torch.float32, device="cuda") for _ in range(2)]
    contrib = [torch.empty(V, dtype=torch.float32, device="cuda") for _ in range(2)]
    vs = [PageRankVectors(rank, contrib, torch.empty(2, dtype=torch.float64, device="cuda"), damping, personalized,
                          source) for _ in range(parts)]
    for k, v in zip(ks, vs):
        k.pagerank_init(v)
    dangling = sum(float(v.sums[1].item()) for v in vs)
    iters = 0
    for it in range(max_iter):
        for k, v in zip(ks, vs):
            k.pagerank_step(v, it, dangling)
        residual = sum(float(v.sums[0].item()) for v in vs)
        dangling = sum(float(v.sums[1].item()) for v in vs)
        iters = it + 1
        if residual <= float(np.float32(tol)):
            break
    out = ks[0].emit(rank[iters & 1])
    infos = [k.info(1) for k in ks]
    for k in ks:
        k.close()
    return out, iters, infos


def _push(dg, parts, source):
    import torch

    from hytgraph_b200.shard import CudaShardKernels

    ks = [CudaShardKernels(dg, p, parts) for p in range(parts)]
    V = dg.num_vertices
    keys = torch.empty(V + 1, dtype=torch.int32, device="cuda")
    counts = torch.empty(parts, dtype=torch.int64, device="cuda")
    total = torch.empty(1, dtype=torch.int64, device="cuda")
    for k in ks:
        k.sssp_init(keys, source)
    rounds, pulls = 0, 0  # pulls: rounds whose summed frontier asks for a sweep
    while rounds < 4 * V + 1024:
        for p, k in enumerate(ks):
            k.sssp_collect(keys, counts[p:p + 1])
        total.copy_(counts.sum().reshape(1))  # the exchange: one push / pull decision for every shard
        pulls += int(int(total.item()) * 4 > dg.num_edges)
        idle = True
        for k in ks:
            k.sssp_relax(keys, total)
            idle = idle and int(keys[V].item()) == 1
        rounds += 1
        if idle:
            break
    out = ks[0].sssp_labels(keys)
    relaxed = sum(k.info(2)["edges_relaxed"] for k in ks)
    for k in ks:
        k.close()
    return out, rounds, relaxed, pulls


def test_shard_pagerank_matches_single_gpu(hyt, oracle, gpu):
    for g, flags in _graphs(hyt):
        ref, _, _, _ = oracle.pagerank_f64(g.row_offsets, g.column_indices)
        with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | flags) as dg:
            single, st = dg.pagerank()
            for parts in (1, 2, 3, 5):
                r, iters, infos = _pull(dg, parts)
                assert iters == st["iterations"], (g.num_vertices, parts)
                assert float(np.abs(r.astype(np.float64) - single).sum()) <= 1e-6, (g.num_vertices, parts)
                assert float(np.abs(r.astype(np.float64) - ref).sum()) <= PR_L1_TOL
                assert sum(i["edges"] for i in infos) == g.num_edges
                assert [i["vertex_begin"] for i in infos[1:]] == [i["vertex_end"] for i in infos[:-1]]


def test_shard_ppr_matches_single_gpu(hyt, oracle, gpu):
    for g, flags in _graphs(hyt)[:3] + _graphs(hyt)[-1:]:
        with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | flags) as dg:
            for s in hyt.pick_sources(g.row_offsets, 5, 2):
                ref, _, _, _ = oracle.ppr_f64(g.row_offsets, g.column_indices, int(s))
                single, st = dg.ppr(int(s))
                for parts in (2, 3):
                    r, iters, _ = _pull(dg, parts, True, int(s), damping=float(np.float32(1) - np.float32(0.15)))
                    assert iters == st["iterations"]
                    assert float(np.abs(r.astype(np.float64) - single).sum()) <= 1e-6
                    assert float(np.abs(r.astype(np.float64) - ref).sum()) <= PR_L1_TOL


def test_shard_sssp_bit_exact(hyt, oracle, gpu):
    swept = 0
    for g, flags in _graphs(hyt):
        srcs = hyt.pick_sources(g.row_offsets, 9, 2) if g.num_edges else np.zeros(1, np.uint32)
        singles = {}
        with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | flags) as dg:
            for s in srcs:
                single, _ = dg.sssp(int(s))
                singles[int(s)] = single
                for parts in (1, 2, 3, 5):
                    d, rounds, relaxed, pulls = _push(dg, parts, int(s))
                    assert np.array_equal(d, single), (g.num_vertices, int(s), parts, pulls)
                    assert rounds >= 1 and relaxed >= 0
                    swept += pulls
        with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_PUSH) as dp:  # no CSC: push rounds only
            s = int(srcs[0])
            d, _, _, _ = _push(dp, 2, s)
            assert np.array_equal(d, singles[s])
    assert swept > 0  # the R-MAT cases reach dense rounds


def test_shard_float_weights_and_errors(hyt, gpu):
    import torch

    from hytgraph_b200.shard import CudaShardKernels

    g = hyt.rmat(12, 16, 31)
    rng = np.random.default_rng(2)
    gf = hyt.CSR(g.row_offsets, g.column_indices, (rng.random(g.num_edges) * 10).astype(np.float32))
    with hyt.Graph(gf) as dg:
        s = int(hyt.pick_sources(g.row_offsets, 1, 1)[0])
        single, _ = dg.sssp(s)
        d, _, _, _ = _push(dg, 3, s)
        assert np.array_equal(d, single)  # float weights (through the sweeps on dense rounds)
        b = np.zeros(3, np.uint32)
        hyt.capi.check(hyt.capi.lib.hyt_shard_bounds(dg.handle, 1, 2, b.ctypes.data))
        bad = b.copy()
        bad[1] = bad[1] + 1 if bad[1] + 1 < g.num_vertices else bad[1] - 1  # not a tile start
        import ctypes as C

        h = C.c_void_p()
        rc = hyt.capi.lib.hyt_shard_create(dg.handle, 1, bad.ctypes.data, 2, 0, C.byref(h))
        if rc == hyt.capi.HYT_OK:  # the neighbour happened to start a tile too
            hyt.capi.check(hyt.capi.lib.hyt_shard_destroy(h))
        else:
            assert rc == hyt.capi.HYT_E_INVALID
        for args in ((3, b.ctypes.data, 2, 0), (1, b.ctypes.data, 2, 2), (1, None, 2, 0)):
            assert hyt.capi.lib.hyt_shard_create(dg.handle, *args, C.byref(h)) == hyt.capi.HYT_E_INVALID
        k = CudaShardKernels(dg, 0, 2)
        keys = torch.empty(g.num_vertices + 1, dtype=torch.int32, device="cuda")
        with pytest.raises(hyt.HytError) as e:
            k.sssp_init(keys, g.num_vertices)
        assert e.value.code == hyt.capi.HYT_E_INVALID
        k.close()
    with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_PULL) as dp:
        b = np.zeros(3, np.uint32)
        assert hyt.capi.lib.hyt_shard_bounds(dp.handle, 2, 2, b.ctypes.data) == hyt.capi.HYT_E_INVALID


def test_sharded_graph_through_nccl(hyt, oracle, gpu):
    import torch
    import torch.distributed as dist

    g = hyt.rmat(14, 16, 41)
    dist.init_process_group("nccl", store=dist.HashStore(), rank=0, world_size=1,
                            device_id=torch.device("cuda", 0))
    try:
        with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER) as dg:
            with hyt.ShardedGraph(dg) as sg:
                r, st = sg.pagerank()
                single, st1 = dg.pagerank()
                assert st["iterations"] == st1["iterations"] and st["parts"] == 1
                assert float(np.abs(r.astype(np.float64) - single).sum()) <= 1e-6
                s = int(hyt.pick_sources(g.row_offsets, 2, 1)[0])
                d, sst = sg.sssp(s)
                assert np.array_equal(d, dg.sssp(s)[0]) and sst["converged"] == 1
                p, _ = sg.ppr(s)
                assert float(np.abs(p.astype(np.float64) - dg.ppr(s)[0]).sum()) <= 1e-6
                rd = torch.empty(g.num_vertices, dtype=torch.float32, device="cuda")  # device outputs
                dd = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
                sg.pagerank(out=rd)
                sg.sssp(s, out=dd)
                assert np.array_equal(rd.cpu().numpy(), r) and np.array_equal(dd.cpu().numpy().view(np.uint32), d)
    finally:
        dist.destroy_process_group()
