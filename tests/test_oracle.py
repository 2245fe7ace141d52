"""The oracle (C restatement of the reference) pinned against the reference's
golden vectors, its known-answer tests and its compiled CPU code."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

from conftest import ROOT  # noqa: F401


def _digest(g):
    h = hashlib.sha256()
    h.update(g.row_offsets.astype("<u8").tobytes())
    h.update(g.column_indices.astype("<u4").tobytes())
    if g.weights is not None:
        h.update(g.weights.astype("<u4").tobytes())
    return h.hexdigest()


def _graph(hyt, m):
    w = (1, 63) if m["weighted"] else (0, 0)
    return hyt.rmat(m["scale"], m["edge_factor"], m["seed"], *w)


def test_generator_matches_golden_digest(hyt, golden):
    for m in golden["meta"]["graphs"]:
        g = _graph(hyt, m)
        assert g.num_edges == m["num_edges"]
        assert _digest(g) == m["csr_sha256"], m["key"]


def test_oracle_generator_matches_golden_and_product(hyt, oracle, golden):
    """The oracle's restatement of the generator (used by the reference arm
    of the bench, which loads no product library) gives the golden digests
    and the product generator's bytes, and the same seeded sources."""
    from types import SimpleNamespace

    for m in golden["meta"]["graphs"]:
        w = (1, 63) if m["weighted"] else (0, 0)
        off, cols, wt = oracle.rmat(m["scale"], m["edge_factor"], m["seed"], *w)
        assert _digest(SimpleNamespace(row_offsets=off, column_indices=cols, weights=wt)) == m["csr_sha256"], m["key"]
    for scale, ef, seed, w in [(13, 16, 9, (1, 63)), (15, 8, 2024, (0, 0)), (17, 16, 20241203, (1, 63)),
                               (12, 4, 3, (5, 9))]:
        off, cols, wt = oracle.rmat(scale, ef, seed, *w)
        g = hyt.rmat(scale, ef, seed, *w)
        assert np.array_equal(off, g.row_offsets) and np.array_equal(cols, g.column_indices)
        assert (wt is None and g.weights is None) or np.array_equal(wt, g.weights)
        for count in (1, 8, 40):
            assert np.array_equal(oracle.pick_sources(off, seed, count), hyt.pick_sources(off, seed, count))


def test_oracle_threads_do_not_change_results():
    """The row-parallel oracle loops give the same bits on one thread and on
    seven (FP64 and FP32 PageRank, the SSSP restatement, Dijkstra)."""
    import os
    import subprocess
    import sys

    code = ("import sys, numpy as np; sys.path.insert(0, %r); from oracle.bindings import Oracle; o = Oracle(); "
            "off, cols, w = o.rmat(15, 16, 4); r64 = o.pagerank_f64(off, cols)[0]; r32 = o.pagerank_f32(off, cols)[0]; "
            "p64 = o.ppr_f64(off, cols, 3)[0]; d = o.sssp(off, cols, w.astype(np.float32), 3)[0]; "
            "dj = o.dijkstra(off, cols, w, 3); "
            "sys.stdout.buffer.write(r64.tobytes() + r32.tobytes() + p64.tobytes() + d.tobytes() + dj.tobytes())"
            ) % str(ROOT)
    outs = []
    for threads in ("1", "7"):
        env = dict(os.environ, ORACLE_THREADS=threads)
        outs.append(subprocess.run([sys.executable, "-c", code], capture_output=True, env=env, check=True).stdout)
    assert outs[0] == outs[1] and len(outs[0]) > 0


def test_dijkstra_agrees_with_the_sssp_restatement(oracle):
    """Two independent oracles of the same labels: Dijkstra (exact integers)
    and the restatement of the reference's synchronous Bellman-Ford."""
    off, cols, w = oracle.rmat(14, 16, 12)
    for s in oracle.pick_sources(off, 12, 3):
        dj = oracle.dijkstra(off, cols, w, int(s))
        bf, _, conv = oracle.sssp(off, cols, w.astype(np.float32), int(s))
        assert conv
        reach = dj != np.iinfo(np.uint64).max
        assert np.array_equal(np.isfinite(bf), reach)
        assert np.array_equal(bf[reach].astype(np.uint64), dj[reach])


def test_oracle_pagerank_f32_bit_identical_to_reference_golden(hyt, oracle, golden):
    for m in golden["meta"]["graphs"]:
        g = _graph(hyt, m)
        r, it, res, conv = oracle.pagerank_f32(g.row_offsets, g.column_indices)
        assert it == m["pr_iterations"] and conv == m["pr_converged"]
        assert np.array_equal(r.view(np.uint32), golden["npz"][f"{m['key']}_pr_bits"])


def test_oracle_sssp_bit_identical_to_reference_golden(hyt, oracle, golden):
    for m in golden["meta"]["graphs"]:
        g = _graph(hyt, m)
        w = g.weights.astype(np.float32) if g.weights is not None else None
        bits = golden["npz"][f"{m['key']}_sssp_bits"]
        for i, s in enumerate(m["sources"]):
            d, rounds, conv = oracle.sssp(g.row_offsets, g.column_indices, w, s)
            assert conv and rounds == m["sssp_rounds"][i]
            assert np.array_equal(d.view(np.uint32), bits[i])


def test_dijkstra_cross_check(hyt, oracle):
    g = hyt.rmat(12, 16, 77)
    for s in hyt.pick_sources(g.row_offsets, 5, 3):
        d, _, _ = oracle.sssp(g.row_offsets, g.column_indices, g.weights.astype(np.float32), int(s))
        dj = oracle.dijkstra(g.row_offsets, g.column_indices, g.weights, int(s))
        reach = dj != np.iinfo(np.uint64).max
        assert np.array_equal(np.isfinite(d), reach)
        assert np.array_equal(d[reach].astype(np.uint64), dj[reach])


def test_hand_known_answers(oracle, golden):
    """The reference's hand-written cases (algorithm_tests.cpp:22-157,
    cuda_algorithm_tests.cu:23-87) reproduced exactly by the oracle."""
    for h in golden["meta"]["hand"]:
        off = np.array(h["row_offsets"], np.uint64)
        cols = np.array(h["column_indices"], np.uint32)
        if "ranks" in h:
            r, it, _, conv = oracle.pagerank_f32(off, cols, 0.85, 1e-6, 200)
            assert conv and it == h["iterations"]
            assert np.array_equal(r, np.array(h["ranks"], np.float32))
        else:
            w = None if h["weights"] is None else np.array(h["weights"], np.float32)
            d, it, conv = oracle.sssp(off, cols, w, h["source"])
            want = np.array([np.inf if x is None else x for x in h["distances"]], np.float32)
            assert conv and it == h["iterations"] and np.array_equal(d, want)
    # the reference's assertions themselves
    by = {h["name"]: h for h in golden["meta"]["hand"]}
    assert np.allclose(by["pr_cycle3"]["ranks"], 1 / 3, atol=1e-5)
    assert abs(sum(by["pr_dangling"]["ranks"]) - 1.0) <= 1e-5
    assert by["sssp_weighted4"]["distances"] == [0.0, 1.0, 3.0, 4.0]
    assert by["sssp_unweighted4"]["distances"] == [0.0, 1.0, 2.0, None]


def test_pagerank_f64_matches_f32_reference_semantics(hyt, oracle):
    g = hyt.rmat(10, 16, 9)
    r32, it32, _, _ = oracle.pagerank_f32(g.row_offsets, g.column_indices, tol=1e-9, max_iter=60)
    r64, it64, _, _ = oracle.pagerank_f64(g.row_offsets, g.column_indices, tol=1e-9, max_iter=60)
    assert abs(r64.sum() - 1.0) < 1e-12
    assert np.abs(r32 - r64).sum() < 1e-4  # float drift of the FP32 restatement


def test_ppr_oracle_hand_cases(oracle):
    # 3-cycle 0->1->2->0 from source 0: x = r * sum_k d^k e_{k mod 3}
    off = np.array([0, 1, 2, 3], np.uint64)
    cols = np.array([1, 2, 0], np.uint32)
    r, _, _, conv = oracle.ppr_f64(off, cols, 0, 0.15, 1e-14, 2000)
    d = 0.85
    want = np.array([1, d, d * d]) * (0.15 / (1 - d ** 3))
    assert conv and np.allclose(r, want, atol=1e-12)
    # star: 0 -> 1..4, leaves dangling (mass returns to the source)
    off = np.array([0, 4, 4, 4, 4, 4], np.uint64)
    cols = np.array([1, 2, 3, 4], np.uint32)
    r, _, _, conv = oracle.ppr_f64(off, cols, 0, 0.15, 1e-14, 2000)
    # fixed point: x0 = 0.15 + 0.85 * (1 - x0) ... leaves share d*x0/4 each
    x0 = 1.0 / (1.0 + 0.85)
    assert conv and abs(r[0] - x0) < 1e-12 and np.allclose(r[1:], 0.85 * x0 / 4, atol=1e-12)
    assert abs(r.sum() - 1.0) < 1e-12


def test_oracle_vs_reference_random(hyt, oracle, reference):
    for seed, (scale, ef) in enumerate([(9, 4), (10, 8), (11, 16)]):
        g = hyt.rmat(scale, ef, 1000 + seed)
        a = oracle.pagerank_f32(g.row_offsets, g.column_indices)
        b = reference.pagerank_cpu(g.row_offsets, g.column_indices)
        assert np.array_equal(a[0].view(np.uint32), b[0].view(np.uint32)) and a[1] == b[1]
        w = g.weights.astype(np.float32)
        for s in hyt.pick_sources(g.row_offsets, seed, 2):
            x = oracle.sssp(g.row_offsets, g.column_indices, w, int(s))
            y = reference.sssp_cpu(g.row_offsets, g.column_indices, w, int(s))
            assert np.array_equal(x[0].view(np.uint32), y[0].view(np.uint32)) and x[1] == y[1]


def test_hytm_cost_model_known_answer(oracle, golden):
    from oracle.bindings import HytmOptions

    k = golden["meta"]["hytm"]
    o = k["options"]
    opts = HytmOptions(o["alpha"], o["beta"], o["gamma"], o["rtt"], o["cpu_throughput"], o["m"], o["mr"], 4, 8, 128)
    c = oracle.hytm_partition(np.array(k["row_offsets"], np.uint64), np.array(k["active"], np.uint8), 0, 2, opts)
    m = k["metrics"]  # vbegin, vend, Av, Ae, Ep, F bytes, C bytes, zc req, zc align, zc total, index
    assert (c.active_vertices, c.active_edges, c.total_edges) == (m[2], m[3], m[4]) == (2, 3, 3)
    assert (c.filter_bytes, c.compaction_bytes, c.zc_requests, c.zc_alignment) == (m[5], m[6], m[7], m[8])
    assert (c.filter_cost, c.compaction_cost, c.zero_copy_cost, c.zc_rtt) == tuple(k["costs"]) == (2.0, 4.0, 2.0, 2.0)
    assert c.engine == k["engine"]


def test_selector_and_combiner_known_answers(oracle, golden):
    for s in golden["meta"]["selector"]:
        assert oracle.select_engine(s["f"], s["c"], s["z"], 0.8, 0.4) == s["engine"]
    for c in golden["meta"]["combiner"]:
        top, teng, tfirst = oracle.task_combine(c["engines"], c["k"])
        assert top.tolist() == c["task_of_partition"]
        assert teng.tolist() == c["task_engine"] and tfirst.tolist() == c["task_first"]


def test_hytm_oracle_vs_reference_random(hyt, oracle, reference):
    from oracle.bindings import HytmOptions

    rng = np.random.default_rng(3)
    g = hyt.rmat(12, 8, 21)
    V = g.num_vertices
    bounds = np.unique(np.concatenate([[0, V], rng.integers(0, V, 14)]))
    parts = np.stack([bounds[:-1], bounds[1:]], 1).astype(np.uint32)
    for frac in (0.0, 0.01, 0.2, 1.0):
        act = (rng.random(V) < frac).astype(np.uint8)
        for rtt, tput in [(1.0, 1.0), (2.0, 14.0), (3e-6, 2.5e10)]:
            metrics, costs, eng = reference.hytm_evaluate(g.row_offsets, g.column_indices, act, parts,
                                                          [0.8, 0.4, 0.625, rtt, tput], [128, 256])
            opts = HytmOptions(0.8, 0.4, 0.625, rtt, tput, 128, 256, 4, 8, 128)
            for i, (vb, ve) in enumerate(parts):
                c = oracle.hytm_partition(g.row_offsets, act, int(vb), int(ve), opts)
                assert (c.active_vertices, c.active_edges, c.total_edges, c.filter_bytes, c.compaction_bytes,
                        c.zc_requests, c.zc_alignment) == tuple(int(x) for x in metrics[i, 2:9])
                assert (c.filter_cost, c.compaction_cost, c.zero_copy_cost, c.zc_rtt) == tuple(costs[i])
                assert c.engine == eng[i]
    rng2 = np.random.default_rng(5)
    for _ in range(50):
        e = rng2.integers(0, 3, rng2.integers(0, 40))
        k = int(rng2.integers(1, 6))
        a = oracle.task_combine(e, k)
        b = reference.task_combine(e, k)
        assert all(np.array_equal(x, y) for x, y in zip(a, b[:3]))


def test_hub_sort_known_answers(oracle, golden):
    """HubSorter cases of the reference's unit tests (unit_tests.cpp:2468-2602),
    frozen from the reference's own output."""
    for c in golden["meta"]["hub_sort"]:
        order, scores, n = oracle.hub_sort(np.array(c["row_offsets"], np.uint64),
                                           np.array(c["column_indices"], np.uint32), c["hub_fraction"])
        assert order.tolist() == c["vertex_order"], c["name"]
        assert scores.tolist() == c["scores"] and n == c["hub_count"], c["name"]
    with pytest.raises(ValueError):
        oracle.hub_sort(np.array([0, 1, 1], np.uint64), np.array([1], np.uint32), 1.5)


def test_reorder_known_answers(oracle, golden):
    """CSRGraph::reorder_vertices cases (unit_tests.cpp:2604-2740)."""
    for c in golden["meta"]["reorder"]:
        w = None if c["weights"] is None else np.array(c["weights"], np.float32)
        off, cols, nw = oracle.reorder(np.array(c["row_offsets"], np.uint64), np.array(c["column_indices"], np.uint32),
                                       w, c["vertex_order"])
        assert off.tolist() == c["new_row_offsets"] and cols.tolist() == c["new_column_indices"], c["name"]
        assert (nw is None and c["new_weights"] is None) or nw.tolist() == c["new_weights"], c["name"]
    off, cols = np.array([0, 1, 2, 3], np.uint64), np.array([1, 2, 0], np.uint32)
    for bad in ([0, 1, 1], [0, 1, 3]):  # duplicate, out of range
        with pytest.raises(ValueError):
            oracle.reorder(off, cols, None, bad)


def test_hub_sort_and_reorder_golden_graphs(hyt, oracle, golden):
    """The oracle reproduces the reference HubSorter's order, scores and hub
    count and the reordered CSR on every golden R-MAT graph."""
    for m in golden["meta"]["graphs"]:
        g = _graph(hyt, m)
        order, scores, n = oracle.hub_sort(g.row_offsets, g.column_indices, m["hub_fraction"])
        assert n == m["hub_count"], m["key"]
        assert hashlib.sha256(order.astype("<u4").tobytes()).hexdigest() == m["hub_order_sha256"], m["key"]
        assert hashlib.sha256(scores.astype("<f8").tobytes()).hexdigest() == m["hub_scores_sha256"], m["key"]
        off, cols, w = oracle.reorder(g.row_offsets, g.column_indices, g.weights, order)
        assert _digest(hyt.CSR(off, cols, w)) == m["reordered_sha256"], m["key"]


def test_hub_sort_oracle_vs_reference_random(hyt, oracle, reference):
    rng = np.random.default_rng(11)
    for scale, ef, seed in [(6, 2, 1), (11, 16, 7), (13, 4, 8)]:
        g = hyt.rmat(scale, ef, seed)
        for frac in (0.0, 0.08, 1.0 / 3.0, 0.5, 1.0, float(rng.random())):
            a = oracle.hub_sort(g.row_offsets, g.column_indices, frac)
            b = reference.hub_sort(g.row_offsets, g.column_indices, frac)
            assert np.array_equal(a[0], b[0]) and a[2] == b[2], (scale, frac)
            assert np.array_equal(a[1].view(np.uint64), b[1].view(np.uint64)), (scale, frac)
        order = rng.permutation(g.num_vertices).astype(np.uint32)
        x = oracle.reorder(g.row_offsets, g.column_indices, g.weights, order)
        y = reference.reorder(g.row_offsets, g.column_indices, g.weights.view(np.float32), order)
        assert all(np.array_equal(p.view(np.uint8), q.view(np.uint8)) for p, q in zip(x, y)), scale


# ---------------------------------------------------------------- loader --
LOADER_CASES = [
    # GraphLoader cases of the reference's unit tests (unit_tests.cpp:374-599)
    ("unweighted", "# simple directed graph\n0 1\n0 2\n1 2\n2 0\n", 4, False),
    ("weighted", "# weighted graph\n0 1 0.5\n0 2 1.25\n1 2 2.5\n", 3, True),
    ("parallel", "0 1\n0 1\n0 2\n", 3, False),
    ("bad_vertex", "0 3\n", 3, False),
    ("missing_weight", "0 1\n", 2, True),
    ("malformed", "this is not an edge\n", 2, False),
]


def test_loader_known_answers(oracle, tmp_path):
    """The expectations of unit_tests.cpp:374-599, on the oracle."""
    got = {}
    for name, text, V, weighted in LOADER_CASES:
        (tmp_path / name).write_text(text)
        try:
            got[name] = oracle.load_edge_list(tmp_path / name, V, weighted)
        except ValueError as e:
            got[name] = str(e)
    off, cols, w = got["unweighted"]
    assert np.diff(off).tolist() == [2, 1, 1, 0] and cols.tolist() == [1, 2, 2, 0] and w is None
    off, cols, w = got["weighted"]
    assert cols.tolist() == [1, 2, 2] and w.tolist() == [0.5, 1.25, 2.5]
    off, cols, w = got["parallel"]
    assert off.tolist() == [0, 3, 3, 3] and cols.tolist() == [1, 1, 2]
    assert got["bad_vertex"] == "GraphLoader::load_edge_list: vertex ID out of range at line 1"
    assert got["missing_weight"] == "GraphLoader::load_edge_list: missing edge weight at line 1"
    assert got["malformed"] == "GraphLoader::load_edge_list: malformed edge at line 1"


def loader_corpus(seed: int, n: int):
    """Seeded edge-list files with the record forms the reference's stream
    extraction treats specially: signs, overflow, exponents, leading zeros,
    comments, blank lines, CRLF, tabs, vertical tabs, trailing data."""
    rng = np.random.default_rng(seed)
    ints = ["0", "1", "7", "+1", "-0", "-1", "007", "18446744073709551615", "18446744073709551616", "1x", "x",
            "", "+", "-", "2.0", "0x1", "4294967296"]
    flts = ["0.5", "1", "-2.5", "1e3", "1E-3", ".5", "5.", ".", "1.5e", "1e+", "1e-50", "1e50", "inf", "nan",
            "+.5e+2", "00.25", "0x1p3", "1.2.3", "3.4028235e38", "3.4028236e38", "1e-45", "7e-46", "-0", "1e5x",
            "", "e5", "+e5", "0.1", "123456789", "1.00000005960464477539062500001"]
    seps = [" ", "\t", "  ", " \t ", "\v", ","]

    def line(weighted):
        if rng.random() < 0.05:
            return str(rng.choice(["", "   ", "\t", "# comment", "  # c", "#", "\r"]))
        parts = [str(rng.choice(ints)) if rng.random() < 0.08 else str(rng.integers(0, 8)) for _ in range(2)]
        if weighted and rng.random() < 0.97:
            parts.append(str(rng.choice(flts)) if rng.random() < 0.5 else f"{rng.random() * 10:.{rng.integers(0, 9)}f}")
        if rng.random() < 0.05:
            parts.append(str(rng.choice(["x", "1", "#"])))
        s = parts[0]
        for p in parts[1:]:
            s += str(rng.choice(seps)) + p
        if rng.random() < 0.2:
            s = str(rng.choice([" ", "\t", "\r"])) + s
        if rng.random() < 0.2:
            s += str(rng.choice([" ", "\t", "\r", "\r\r"]))
        return s

    for _ in range(n):
        weighted = bool(rng.integers(0, 2))
        text = "\n".join(line(weighted) for _ in range(int(rng.integers(1, 6))))
        yield text + ("\n" if rng.random() < 0.5 else ""), 8, weighted


def _load_or_error(loader, path, V, weighted):
    try:
        return loader(path, V, weighted)
    except ValueError as e:
        return str(e).split(": ", 1)[1] if str(e).startswith("ref_") else str(e)


def test_loader_oracle_vs_reference_corpus(oracle, reference, tmp_path):
    """The oracle's record rules equal the reference's GraphLoader (run here
    from its own sources) on 1500 seeded files: same arrays, or the same
    error message and line."""
    path = tmp_path / "f.el"
    for i, (text, V, weighted) in enumerate(loader_corpus(7, 1500)):
        path.write_text(text)
        a = _load_or_error(oracle.load_edge_list, path, V, weighted)
        b = _load_or_error(reference.load_edge_list, path, V, weighted)
        if isinstance(a, str) or isinstance(b, str):
            assert a == b, (i, text)
            continue
        for x, y in zip(a, b):
            assert (x is None and y is None) or np.array_equal(x.view(np.uint8), y.view(np.uint8)), (i, text)


def test_csr_from_edges_oracle(oracle):
    rng = np.random.default_rng(4)
    V, E = 300, 5000
    src = rng.integers(0, V, E).astype(np.uint32)
    dst = rng.integers(0, V, E).astype(np.uint32)
    w = rng.random(E).astype(np.float32)
    off, cols, wo = oracle.csr_from_edges(V, src, dst, w)
    order = np.argsort(src, kind="stable")
    assert np.array_equal(cols, dst[order]) and np.array_equal(wo, w[order])
    assert np.array_equal(off, np.concatenate([[0], np.cumsum(np.bincount(src, minlength=V))]).astype(np.uint64))
    with pytest.raises(ValueError):
        oracle.csr_from_edges(V, np.array([1, V], np.uint32), np.array([0, 0], np.uint32))


# ---------------------------------------------------- contribution scheduling --
def test_contribution_known_answers(oracle):
    """unit_tests.cpp:2751-3005 on the oracle."""
    o, m = oracle.contribution_schedule([0, 1, 2, 3], [0.10, 0.90, 0.30, 0.70])
    assert o.tolist() == [1, 3, 2, 0] and m["input_item_count"] == 4 and m["scheduled_item_count"] == 4
    assert abs(m["scheduling_overhead"] - 2.0) < 1e-12
    assert oracle.contribution_schedule([3, 1, 2, 0], [0.5, 0.5, 0.9, 0.5])[0].tolist() == [2, 0, 1, 3]
    o, m = oracle.contribution_schedule([0, 1, 2, 3], [0.0, 1e-8, 0.25, -1e-8], eps=1e-6)
    assert m["zero_contribution_count"] == 3 and o.tolist() == [2, 1, 0, 3]
    assert oracle.contribution_schedule([0, 1, 2], [0.1, 0.9, 0.3])[1]["reordered_item_count"] == 3
    off = np.array([0, 2, 3, 3], np.uint64)
    cols = np.array([1, 2, 2], np.uint32)
    c = oracle.pagerank_contributions(off, cols, np.array([1, 0, 0], np.float32))
    assert np.allclose(c, [0.95, 0.475, 0.475], atol=1e-5)
    s = oracle.sssp_contributions(np.array([0, 5, np.inf, 10], np.float32), np.array([0, 3, 7, 12], np.float32))
    assert s.tolist() == [0.0, 2.0, 1.0, 0.0]


def test_contribution_oracle_vs_reference(hyt, oracle, reference):
    rng = np.random.default_rng(9)
    g = hyt.rmat(12, 8, 17)
    V = g.num_vertices
    for trial in range(4):
        cur = rng.random(V).astype(np.float32)
        cur /= cur.sum()
        a = oracle.pagerank_contributions(g.row_offsets, g.column_indices, cur, 0.85)
        b = reference.pagerank_contributions(g.row_offsets, g.column_indices, cur, 0.85)
        assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), trial
        c64 = oracle.pagerank_contributions(g.row_offsets, g.column_indices, cur, 0.85, fp64=True)
        assert np.max(np.abs(c64 - b)) < 1e-7
    for trial in range(20):
        n = int(rng.integers(0, 300))
        cur = rng.choice([0.0, 1.0, 2.5, np.inf, np.nan, 7.0], n).astype(np.float32)
        cand = rng.choice([0.0, 1.0, 2.5, np.inf, np.nan, 3.0], n).astype(np.float32)
        for tol in (0.0, 0.5):
            assert np.array_equal(oracle.sssp_contributions(cur, cand, tol), reference.sssp_contributions(cur, cand, tol))
    for trial in range(60):
        n = int(rng.integers(0, 400))
        items = rng.integers(0, max(n, 1) * 2 if trial % 2 else 50, n)
        contrib = rng.choice([0.0, -0.0, 0.5, 0.25, 1e-9, -1e-9, 3.0], n) if trial % 3 else rng.normal(size=n)
        for det in (True, False):
            a = oracle.contribution_schedule(items, contrib, det, 1e-6)
            b = reference.contribution_schedule(items, contrib, det, 1e-6)
            assert a[0].tolist() == b[0].tolist() and a[1] == b[1], (trial, det)
