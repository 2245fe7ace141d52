"""GPU parity: the CUDA path through the C ABI against the oracle.

Tolerances: PageRank / personalized PageRank L1 <= 1e-5 against the FP64
oracle (the bar the path is specified to), SSSP bit-exact.
"""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PR_L1_TOL = 1e-5


def _graph_cases(hyt):
    cases = [hyt.rmat(s, ef, seed) for s, ef, seed in [(8, 16, 1), (10, 8, 2), (12, 16, 3), (14, 16, 4), (16, 16, 5)]]
    cases.append(hyt.rmat(11, 4, 6, 0, 0))  # unweighted, many dangling vertices
    return cases


def _csr(off, cols, w=None):
    import hytgraph_b200 as hyt

    w = None if w is None else np.asarray(w, np.float32 if np.asarray(w).dtype.kind == "f" else np.uint32)
    return hyt.CSR(np.asarray(off, np.uint64), np.asarray(cols, np.uint32), w)


def _special_graphs():
    """Edge cases: single vertex, all dangling, 3-cycle, a hub with in- and
    out-degree > 4096 (chunked long rows / hub tasks), warp-sized rows."""
    out = [
        _csr([0, 0], []),
        _csr([0, 0, 0, 0, 0], []),
        _csr([0, 1, 2, 3], [1, 2, 0], [1, 1, 1]),
        _csr([0, 2, 3, 4], [1, 2, 2, 0], [3, 4, 5, 6]),
    ]
    n = 20000  # star in and out of vertex 0
    off = np.concatenate([[0, n - 1], np.arange(n - 1) + n]).astype(np.uint64)
    cols = np.concatenate([np.arange(1, n), np.zeros(n - 1)]).astype(np.uint32)
    w = (np.arange(cols.shape[0]) % 63 + 1).astype(np.uint32)
    out.append(_csr(off, cols, w))
    rng = np.random.default_rng(0)  # rows of 30-40 edges hit the warp path
    V = 3000
    deg = rng.integers(0, 40, V)
    off = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint64)
    cols = rng.integers(0, V, int(off[-1])).astype(np.uint32)
    out.append(_csr(off, cols, rng.integers(1, 64, cols.shape[0]).astype(np.uint32)))
    return out


def test_pagerank_matches_fp64_oracle(hyt, oracle, gpu):
    for g in _graph_cases(hyt) + _special_graphs():
        ref, it_ref, _, conv_ref = oracle.pagerank_f64(g.row_offsets, g.column_indices)
        with hyt.Graph(g) as dg:
            r, st = dg.pagerank()
        l1 = float(np.abs(r.astype(np.float64) - ref).sum())
        assert l1 <= PR_L1_TOL, (g.num_vertices, l1, st)
        assert st["converged"] == conv_ref
        assert abs(st["iterations"] - it_ref) <= 1, (st["iterations"], it_ref)


def test_scale20_parity_with_the_oracle(hyt, oracle, gpu):
    """One step up the scale ladder toward the bench's scale 24: R-MAT scale
    20 edge factor 16 (about 1M vertices, 16M edges), in input and hub
    order: PageRank within L1 1e-5 of the FP64 oracle, SSSP labels of four
    seeded sources equal to Dijkstra's exact labels."""
    g = hyt.rmat(20, 16, 20241203)
    ref, _, _, _ = oracle.pagerank_f64(g.row_offsets, g.column_indices)
    sources = [int(s) for s in hyt.pick_sources(g.row_offsets, 20241203, 4)]
    want = []
    for s in sources:
        d = oracle.dijkstra(g.row_offsets, g.column_indices, g.weights, s)
        want.append(np.where(d == np.iinfo(np.uint64).max, 0xFFFFFFFF, d).astype(np.uint32))
    for flags in (hyt.capi.HYT_GRAPH_ALL, hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER):
        with hyt.Graph(g, flags=flags) as dg:
            r, st = dg.pagerank()
            assert st["converged"]
            l1 = float(np.abs(r.astype(np.float64) - ref).sum())
            assert l1 <= PR_L1_TOL, (flags, l1)
            for s, w in zip(sources, want):
                assert np.array_equal(dg.sssp(s)[0], w), (flags, s)


_RANKS_SCRIPT = """
import sys, numpy as np
sys.path.insert(0, %r)
import hytgraph_b200 as hyt
g = hyt.rmat(20, 16, 7)
with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER) as dg:
    r, st = dg.pagerank()
    p, sp = dg.ppr(12345)
sys.stdout.buffer.write(np.array([st["iterations"], sp["iterations"]], np.uint32).tobytes() + r.tobytes() + p.tobytes())
"""


def test_pagerank_bit_identical_across_runs_grids_and_kernels(hyt, gpu):
    """PageRank and personalized PageRank give the same bits and iteration
    counts on every run and under other persistent grid sizes; on the same
    tiling the bulk-staged kernel gives the register-path kernel's bits: row
    sums and the FP64 residual / dangling sums have fixed association
    orders."""
    import os
    import subprocess
    import sys

    from conftest import ROOT

    g = hyt.rmat(20, 16, 7)
    with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER) as dg:
        runs = [dg.pagerank() for _ in range(10)]
        ppr = [dg.ppr(12345) for _ in range(3)]
    for r, st in runs[1:]:
        assert st["iterations"] == runs[0][1]["iterations"]
        assert np.array_equal(r.view(np.uint32), runs[0][0].view(np.uint32))
    for p, sp in ppr[1:]:
        assert sp["iterations"] == ppr[0][1]["iterations"]
        assert np.array_equal(p.view(np.uint32), ppr[0][0].view(np.uint32))
    want = (np.array([runs[0][1]["iterations"], ppr[0][1]["iterations"]], np.uint32).tobytes() +
            runs[0][0].tobytes() + ppr[0][0].tobytes())
    def ranks(env):
        out = subprocess.run([sys.executable, "-c", _RANKS_SCRIPT % str(ROOT)], capture_output=True,
                             env=dict(os.environ, **env), timeout=600)
        assert out.returncode == 0, out.stderr.decode()[-2000:]
        return out.stdout

    for env in ({"HYT_PR_GRID": "37"}, {"HYT_PR_GRID": "300"}):
        assert ranks(env) == want, env
    # 256-unit tiles: staged kernel (HYT_STAGED=1 selects them) vs register path
    staged = ranks({"HYT_STAGED": "1"})
    assert staged == ranks({"HYT_STAGED": "0", "HYT_PR_TILE": "256"})
    assert staged == ranks({"HYT_STAGED": "1", "HYT_PR_GRID": "37"})


def test_sssp_staged_register_and_skipping_sweeps_agree(hyt, gpu):
    """The bulk-staged pull sweep, the register-path one and the register
    path with row skipping (rows whose label no in-edge can lower are not
    gathered) reach the same labels -- the unique shortest-path fixed point
    -- on a graph whose frontiers trigger pull rounds.  A sweep without
    skipping relaxes every edge, so those solves relax more edges than the
    graph has; skipping relaxes fewer."""
    import os
    import subprocess
    import sys

    from conftest import ROOT

    code = ("import sys, numpy as np; sys.path.insert(0, %r); import hytgraph_b200 as hyt; "
            "g = hyt.rmat(18, 16, 3); src = hyt.pick_sources(g.row_offsets, 3, 3); "
            "dg = hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER); "
            "out = [dg.sssp(int(s)) for s in src]; "
            "sys.stderr.write('edges %%d\\n' %% sum(st['edges_processed'] for _, st in out)); "
            "sys.stdout.buffer.write(b''.join(d.tobytes() for d, _ in out))") % str(ROOT)
    outs, edges = [], []
    for staged, skip in (("1", "0"), ("0", "0"), ("0", "1")):
        env = dict(os.environ, HYT_STAGED=staged, HYT_SSSP_PULL_SKIP=skip)
        r = subprocess.run([sys.executable, "-c", code], capture_output=True, env=env, timeout=600)
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        outs.append(r.stdout)
        edges.append(int(r.stderr.decode().strip().splitlines()[-1].split()[1]))
    g = hyt.rmat(18, 16, 3)
    assert outs[0] == outs[1] == outs[2] and len(outs[0]) > 0
    assert edges[0] > 3 * g.num_edges and edges[1] > 3 * g.num_edges, edges
    assert edges[2] < edges[1], edges


def test_sssp_bit_exact(hyt, oracle, gpu):
    for g in _graph_cases(hyt) + _special_graphs():
        V = g.num_vertices
        srcs = hyt.pick_sources(g.row_offsets, 9, 3) if g.num_edges else np.zeros(1, np.uint32)
        w32 = None if g.weights is None else g.weights.astype(np.float32)
        with hyt.Graph(g) as dg:
            for s in srcs:
                d, st = dg.sssp(int(s))
                ref, _, _ = oracle.sssp(g.row_offsets, g.column_indices, w32, int(s))
                want = np.where(np.isfinite(ref), ref, 0).astype(np.uint64)
                want = np.where(np.isfinite(ref), want, 0xFFFFFFFF).astype(np.uint32)
                assert np.array_equal(d, want), (V, int(s))
                assert st["converged"] == 1


def test_sssp_float_weights_bit_identical_to_reference_float_path(hyt, oracle, gpu):
    g = hyt.rmat(12, 16, 31)
    rng = np.random.default_rng(2)
    wf = (rng.random(g.num_edges) * 10).astype(np.float32)  # non-integer weights
    gf = hyt.CSR(g.row_offsets, g.column_indices, wf)
    with hyt.Graph(gf) as dg:
        for s in hyt.pick_sources(g.row_offsets, 4, 3):
            d, _ = dg.sssp(int(s))
            ref, _, _ = oracle.sssp(g.row_offsets, g.column_indices, wf, int(s))
            assert np.array_equal(d, ref.view(np.uint32))


def test_sssp_modes_and_repeat(hyt, gpu):
    g = hyt.rmat(15, 16, 12)
    s = int(hyt.pick_sources(g.row_offsets, 1, 1)[0])
    with hyt.Graph(g) as dg:
        a, sa = dg.sssp(s)
        b, sb = dg.sssp(s, flags=hyt.capi.HYT_RUN_NO_GRAPH)
        c, sc = dg.sssp(s, flags=hyt.capi.HYT_RUN_PROFILE)
        d, _ = dg.sssp(s)
    assert np.array_equal(a, b) and np.array_equal(a, c) and np.array_equal(a, d)
    assert sa["edges_processed"] >= g.num_edges * 0.5


def test_sssp_errors(hyt, gpu):
    g = hyt.rmat(8, 4, 1)
    with hyt.Graph(g) as dg:
        with pytest.raises(hyt.HytError) as e:
            dg.sssp(g.num_vertices)
        assert e.value.code == hyt.capi.HYT_E_INVALID
    bad = hyt.CSR(g.row_offsets, g.column_indices, -np.ones(g.num_edges, np.float32))
    with hyt.Graph(bad) as dg:  # PageRank ignores weights; SSSP rejects them
        dg.pagerank()
        with pytest.raises(hyt.HytError) as e:
            dg.sssp(0)
        assert "non-negative" in str(e.value)
    with pytest.raises(hyt.HytError) as e:  # malformed CSR is rejected before any kernel reads it
        hyt.Graph(hyt.CSR(np.array([0, 2, 1], np.uint64), np.array([0, 1], np.uint32)))
    assert e.value.code == hyt.capi.HYT_E_INVALID
    with pytest.raises(hyt.HytError):
        hyt.Graph(hyt.CSR(np.array([0, 1], np.uint64), np.array([5], np.uint32)))


def test_device_generator_matches_host(hyt, gpu):
    for scale, ef, seed, wr in [(8, 4, 1, (1, 63)), (12, 16, 7, (1, 63)), (16, 16, 12345, (1, 63)), (10, 8, 3, (0, 0))]:
        h = hyt.rmat(scale, ef, seed, *wr)
        d = hyt.rmat(scale, ef, seed, *wr, device=True)
        assert d.num_edges == h.num_edges
        with hyt.Graph(d) as dg:  # a graph builds straight from device arrays
            assert dg.info()["num_edges"] == h.num_edges
        back = d.download()
        assert np.array_equal(back.row_offsets, h.row_offsets)
        assert np.array_equal(back.column_indices, h.column_indices)
        if h.weights is None:
            assert back.weights is None
        else:
            assert np.array_equal(back.weights, h.weights)
        d.free()


def test_device_resident_inputs_and_outputs(hyt, oracle, gpu):
    import torch

    g = hyt.rmat(12, 16, 8)
    t_off = torch.from_numpy(g.row_offsets.view(np.int64)).cuda()
    t_cols = torch.from_numpy(g.column_indices.view(np.int32)).cuda()
    t_w = torch.from_numpy(g.weights.view(np.int32)).cuda()
    dcsr = hyt.CSR(g.row_offsets, g.column_indices, g.weights)
    dcsr.to_c = lambda: _dev_csr(hyt, g, t_off, t_cols, t_w)
    with hyt.Graph(dcsr) as dg:
        out = torch.empty(g.num_vertices, dtype=torch.float32, device="cuda")
        dg.pagerank(out=out)
        ref, _, _, _ = oracle.pagerank_f64(g.row_offsets, g.column_indices)
        assert np.abs(out.cpu().numpy() - ref).sum() <= PR_L1_TOL
        dd = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
        s = int(hyt.pick_sources(g.row_offsets, 2, 1)[0])
        dg.sssp(s, out=dd)
        h, _ = dg.sssp(s)
        assert np.array_equal(dd.cpu().numpy().view(np.uint32), h)


def _dev_csr(hyt, g, t_off, t_cols, t_w):
    c = hyt.capi.hyt_csr()
    c.num_vertices, c.num_edges = g.num_vertices, g.num_edges
    c.row_offsets, c.column_indices, c.weights = t_off.data_ptr(), t_cols.data_ptr(), t_w.data_ptr()
    c.weight_kind = hyt.capi.HYT_WEIGHTS_U32
    return c


def test_hub_ordered_graph_same_results(hyt, gpu, oracle):
    """HYT_GRAPH_HUB_ORDER renumbers vertices internally by hub score; every
    source and result stays in the caller's ids (single solves and the batch
    engine): SSSP distances identical, PageRank / PPR within the FP64
    tolerance, paths exposing internal ids rejected."""
    g = hyt.rmat(14, 16, 77)
    srcs = hyt.pick_sources(g.row_offsets, 5, 4)
    gf = hyt.CSR(g.row_offsets, g.column_indices, g.weights.astype(np.float32) / 2)
    gn = hyt.CSR(g.row_offsets, g.column_indices)
    for csr in (g, gf, gn):
        with hyt.Graph(csr) as a, hyt.Graph(csr, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER) as b:
            for s in srcs:
                assert np.array_equal(a.sssp(int(s))[0], b.sssp(int(s))[0])
    ref = oracle.pagerank_f64(g.row_offsets, g.column_indices, 0.85, 1e-10, 200)[0]
    with hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_HUB_ORDER) as b:
        r, st = b.pagerank(tolerance=1e-7, max_iterations=200)
        assert np.abs(r.astype(np.float64) - ref).sum() <= 1e-5
        s = int(srcs[0])
        p, _ = b.ppr(s, tolerance=1e-9, max_iterations=300)
        want = oracle.ppr_f64(g.row_offsets, g.column_indices, s, 0.15, 1e-12, 500)[0]
        assert np.abs(p.astype(np.float64) - want).sum() <= 1e-5
        import torch

        out = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
        b.sssp(s, out=out)  # device output: mapped on the device
        with hyt.Graph(g) as a:
            assert np.array_equal(out.cpu().numpy().view(np.uint32), a.sssp(s)[0])
        with pytest.raises(hyt.HytError) as e:
            b.copy_csc()
        assert e.value.code == hyt.capi.HYT_E_UNSUPPORTED
        with pytest.raises(hyt.HytError) as e:
            b.pagerank_contributions(r)
        assert e.value.code == hyt.capi.HYT_E_UNSUPPORTED
        # the batch engine maps ids too: same distances, PPR within tolerance
        with hyt.Graph(g) as a, hyt.Batch([b, a]) as bt:
            outs, res, _ = bt.run([{"graph": 0, "kind": "sssp", "source": s},
                                   {"graph": 1, "kind": "sssp", "source": s},
                                   {"graph": 0, "kind": "ppr", "source": s},
                                   {"graph": 1, "kind": "ppr", "source": s}])
            assert np.array_equal(outs[0], outs[1])
            assert np.array_equal(outs[0], a.sssp(s)[0])
            assert np.abs(outs[2].astype(np.float64) - outs[3]).sum() <= 2e-5


def test_trim_device_memory(hyt, gpu):
    """Cached pool memory goes back to the driver; graphs still build after."""
    g = hyt.rmat(12, 8, 3)
    with hyt.Graph(g):
        pass
    hyt.capi.check(hyt.capi.lib.hyt_trim_device_memory(0))
    with hyt.Graph(g) as a:
        assert a.sssp(int(hyt.pick_sources(g.row_offsets, 1, 1)[0]))[0].shape == (g.num_vertices,)
