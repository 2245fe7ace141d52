"""Hub sorting and vertex reordering on the GPU (hyt_hub_sort,
hyt_csr_reorder) against the oracle and the reference's frozen answers.

Order, hub count and reordered arrays are bit-exact; scores are compared bit
for bit too (the kernel reproduces the reference's long-double quotient).
"""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _digest(g):
    h = hashlib.sha256()
    h.update(g.row_offsets.astype("<u8").tobytes())
    h.update(g.column_indices.astype("<u4").tobytes())
    if g.weights is not None:
        h.update(g.weights.astype("<u4").tobytes())
    return h.hexdigest()


def _same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_hub_sort_known_answers(hyt, gpu, golden):
    for c in golden["meta"]["hub_sort"]:
        g = hyt.CSR(np.array(c["row_offsets"], np.uint64), np.array(c["column_indices"], np.uint32))
        order, scores, n = hyt.hub_sort(g, c["hub_fraction"])
        assert order.tolist() == c["vertex_order"], c["name"]
        assert scores.tolist() == c["scores"] and n == c["hub_count"], c["name"]


def test_reorder_known_answers(hyt, gpu, golden):
    for c in golden["meta"]["reorder"]:
        w = None if c["weights"] is None else np.array(c["weights"], np.float32)
        g = hyt.CSR(np.array(c["row_offsets"], np.uint64), np.array(c["column_indices"], np.uint32), w)
        r = hyt.reorder(g, c["vertex_order"])
        assert r.row_offsets.tolist() == c["new_row_offsets"], c["name"]
        assert r.column_indices.tolist() == c["new_column_indices"], c["name"]
        if w is None:
            assert r.weights is None
        else:
            assert r.weights.dtype == np.float32 and r.weights.tolist() == c["new_weights"], c["name"]


def test_golden_graphs(hyt, gpu, golden):
    for m in golden["meta"]["graphs"]:
        g = hyt.rmat(m["scale"], m["edge_factor"], m["seed"], *((1, 63) if m["weighted"] else (0, 0)))
        order, scores, n = hyt.hub_sort(g, m["hub_fraction"])
        assert n == m["hub_count"], m["key"]
        assert hashlib.sha256(order.astype("<u4").tobytes()).hexdigest() == m["hub_order_sha256"], m["key"]
        assert hashlib.sha256(scores.astype("<f8").tobytes()).hexdigest() == m["hub_scores_sha256"], m["key"]
        assert _digest(hyt.reorder(g, order)) == m["reordered_sha256"], m["key"]


@pytest.mark.parametrize("scale,ef,seed", [(14, 16, 3), (17, 8, 4), (20, 16, 5)])
def test_hub_sort_matches_oracle(hyt, gpu, oracle, scale, ef, seed):
    g = hyt.rmat(scale, ef, seed)
    for frac in (0.0, 0.08, 1.0 / 3.0, 1.0):
        order, scores, n = hyt.hub_sort(g, frac)
        o_order, o_scores, o_n = oracle.hub_sort(g.row_offsets, g.column_indices, frac)
        assert n == o_n, (scale, frac)
        assert np.array_equal(order, o_order), (scale, frac)
        assert _same(scores, o_scores), (scale, frac)


@pytest.mark.parametrize("scale,ef,seed", [(12, 16, 6), (18, 8, 7)])
def test_reorder_matches_oracle(hyt, gpu, oracle, scale, ef, seed):
    g = hyt.rmat(scale, ef, seed)
    rng = np.random.default_rng(seed)
    gf = hyt.CSR(g.row_offsets, g.column_indices, g.weights.astype(np.float32) / 7.0)
    for order in (hyt.hub_sort(g)[0], rng.permutation(g.num_vertices).astype(np.uint32)):
        for src in (g, gf):
            r = hyt.reorder(src, order)
            off, cols, w = oracle.reorder(src.row_offsets, src.column_indices, src.weights, order)
            assert _same(r.row_offsets, off) and _same(r.column_indices, cols)
            assert r.weights.dtype == src.weights.dtype and _same(r.weights, w)
        d = hyt.reorder(g, order, device=True)
        back = d.download()
        assert _same(back.row_offsets, off) and _same(back.column_indices, cols)


def test_round_trip_and_sssp_on_reordered_graph(hyt, gpu):
    """Reordering by a permutation and then by its inverse gives back the
    graph; SSSP on the reordered graph gives the same distances, renamed."""
    g = hyt.rmat(22, 16, 9)
    order, _, hubs = hyt.hub_sort(g)
    assert hubs == int(np.ceil(g.num_vertices * 0.08))
    assert np.array_equal(np.sort(order), np.arange(g.num_vertices, dtype=np.uint32))
    r = hyt.reorder(g, order)
    inv = np.empty_like(order)
    inv[order] = np.arange(g.num_vertices, dtype=np.uint32)
    back = hyt.reorder(r, inv)
    assert _same(back.row_offsets, g.row_offsets) and _same(back.column_indices, g.column_indices)
    assert _same(back.weights, g.weights)
    src = int(hyt.pick_sources(g.row_offsets, 5, 1)[0])
    with hyt.Graph(g) as a, hyt.Graph(r) as b:
        da, _ = a.sssp(src)
        db, _ = b.sssp(int(inv[src]))
    assert np.array_equal(db[inv], da)


def test_device_inputs(hyt, gpu):
    """Device-resident CSR in, device-resident CSR out."""
    dev = hyt.rmat(16, 8, 12, device=True)
    host = dev.download()
    order, scores, n = hyt.hub_sort(dev, 0.1)
    h_order, h_scores, h_n = hyt.hub_sort(host, 0.1)
    assert n == h_n and np.array_equal(order, h_order) and _same(scores, h_scores)
    r = hyt.reorder(dev, order, device=True).download()
    rh = hyt.reorder(host, order)
    assert _same(r.row_offsets, rh.row_offsets) and _same(r.column_indices, rh.column_indices)
    assert _same(r.weights, rh.weights)


def test_edge_cases_and_errors(hyt, gpu):
    empty = hyt.CSR(np.zeros(1, np.uint64), np.zeros(0, np.uint32))
    order, scores, n = hyt.hub_sort(empty)
    assert order.size == 0 and scores.size == 0 and n == 0
    r = hyt.reorder(empty, np.zeros(0, np.uint32))
    assert r.row_offsets.tolist() == [0] and r.num_edges == 0
    edgeless = hyt.CSR(np.zeros(5, np.uint64), np.zeros(0, np.uint32))
    order, scores, n = hyt.hub_sort(edgeless)
    assert order.tolist() == [0, 1, 2, 3] and scores.tolist() == [0.0] * 4 and n == 1
    g = hyt.CSR(np.array([0, 1, 2, 3], np.uint64), np.array([1, 2, 0], np.uint32))
    for frac in (-0.1, 1.5, float("nan"), float("inf")):
        with pytest.raises(hyt.HytError) as e:
            hyt.hub_sort(g, frac)
        assert e.value.code == hyt.capi.HYT_E_INVALID
    for bad, what in (([0, 1, 1], "duplicate"), ([0, 1, 3], "out-of-range"), ([0, 1], "exactly one entry")):
        with pytest.raises(hyt.HytError) as e:
            hyt.reorder(g, bad)
        assert e.value.code == hyt.capi.HYT_E_INVALID and what in str(e.value)
    broken = hyt.CSR(np.array([0, 1, 2, 3], np.uint64), np.array([1, 7, 0], np.uint32))
    with pytest.raises(hyt.HytError):
        hyt.hub_sort(broken)


def test_reorder_sparse_and_hub_rows(hyt, gpu, oracle):
    """Tiles that span more than 2048 rows (long runs of empty rows) and a
    row of 100k edges, against the oracle."""
    rng = np.random.default_rng(21)
    V = 60000
    deg = np.where(rng.random(V) < 0.02, rng.integers(1, 6, V), 0).astype(np.uint64)
    deg[123] = 100000
    off = np.zeros(V + 1, np.uint64)
    off[1:] = np.cumsum(deg)
    cols = rng.integers(0, V, int(off[-1])).astype(np.uint32)
    w = rng.integers(1, 64, int(off[-1])).astype(np.uint32)
    g = hyt.CSR(off, cols, w)
    for order in (hyt.hub_sort(g)[0], rng.permutation(V).astype(np.uint32)):
        r = hyt.reorder(g, order)
        o_off, o_cols, o_w = oracle.reorder(off, cols, w, order)
        assert _same(r.row_offsets, o_off) and _same(r.column_indices, o_cols) and _same(r.weights, o_w)


def test_device_buffers_and_stats(hyt, gpu):
    import torch

    g = hyt.rmat(15, 16, 31, device=True)
    order_d = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
    scores_d = torch.empty(g.num_vertices, dtype=torch.float64, device="cuda")
    st = {}
    hyt.hub_sort(g, 0.08, order_out=order_d, scores_out=scores_d, stats=st)
    order_h, scores_h, _ = hyt.hub_sort(g, 0.08)
    assert np.array_equal(order_d.cpu().numpy().view(np.uint32), order_h)
    assert _same(scores_d.cpu().numpy(), scores_h)
    assert st["device_ms"] > 0 and st["kernel_ms"] > 0 and st["kernel_bytes"] >= 4 * g.num_edges
    st2 = {}
    a = hyt.reorder(g, order_d, device=True, stats=st2).download()
    b = hyt.reorder(g, order_h)
    assert _same(a.row_offsets, b.row_offsets) and _same(a.column_indices, b.column_indices)
    assert _same(a.weights, b.weights)
    assert st2["kernel_ms"] > 0 and st2["kernel_bytes"] >= 20 * g.num_edges
