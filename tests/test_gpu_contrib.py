"""Contribution-driven scheduling on the GPU against the oracle (which is
pinned to the reference's own code): PageRank contributions within 1e-12
of the FP64 restatement (and within FP32 rounding of the reference's FP32
values), SSSP contributions and schedules bit for bit."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_schedule_known_answers(hyt, gpu):
    """unit_tests.cpp:2751-2880."""
    o, m = hyt.contribution_schedule([0, 1, 2, 3], [0.10, 0.90, 0.30, 0.70])
    assert o.tolist() == [1, 3, 2, 0] and m["input_item_count"] == 4 and abs(m["scheduling_overhead"] - 2.0) < 1e-12
    assert hyt.contribution_schedule([3, 1, 2, 0], [0.5, 0.5, 0.9, 0.5])[0].tolist() == [2, 0, 1, 3]
    o, m = hyt.contribution_schedule([0, 1, 2, 3], [0.0, 1e-8, 0.25, -1e-8], zero_contribution_epsilon=1e-6)
    assert m["zero_contribution_count"] == 3 and o.tolist() == [2, 1, 0, 3]
    assert hyt.contribution_schedule([0, 1, 2], [0.1, 0.9, 0.3])[1]["reordered_item_count"] == 3
    o, m = hyt.contribution_schedule([], [])
    assert o.size == 0 and m["input_item_count"] == 0
    with pytest.raises(hyt.HytError) as e:
        hyt.contribution_schedule([0, 1], [0.5, np.nan])
    assert e.value.code == hyt.capi.HYT_E_INVALID


@pytest.mark.parametrize("n", [1, 7, 1000, 300000])
def test_schedule_matches_oracle(hyt, gpu, oracle, n):
    rng = np.random.default_rng(n)
    for trial in range(3):
        items = rng.integers(0, n * 2 if trial else max(n // 4, 1), n)
        contrib = rng.choice([0.0, -0.0, 0.5, 0.25, 1e-9, -1e-9, 3.0], n) if trial == 1 else rng.normal(size=n)
        for det in (True, False):
            a = hyt.contribution_schedule(items, contrib, det, 1e-6)
            b = oracle.contribution_schedule(items, contrib, det, 1e-6)
            assert np.array_equal(a[0], b[0]) and a[1] == b[1], (n, trial, det)


def test_sssp_contributions(hyt, gpu, oracle):
    got = hyt.sssp_contributions(np.array([0, 5, np.inf, 10], np.float32), np.array([0, 3, 7, 12], np.float32))
    assert got.tolist() == [0.0, 2.0, 1.0, 0.0]
    rng = np.random.default_rng(3)
    n = 1 << 20
    cur = rng.choice([0.0, 1.0, 2.5, np.inf, np.nan, 7.0, 1e30], n).astype(np.float32) * rng.random(n).astype(np.float32)
    cand = rng.choice([0.0, 1.0, 2.5, np.inf, np.nan, 3.0], n).astype(np.float32) * rng.random(n).astype(np.float32)
    for tol in (0.0, 0.25):
        assert np.array_equal(hyt.sssp_contributions(cur, cand, tol).view(np.uint64),
                              oracle.sssp_contributions(cur, cand, tol).view(np.uint64))
    with pytest.raises(hyt.HytError):
        hyt.sssp_contributions(cur, cand, -1.0)


@pytest.mark.parametrize("scale", [10, 16])
def test_pagerank_contributions(hyt, gpu, oracle, scale):
    g = hyt.rmat(scale, 16, 5 + scale)
    with hyt.Graph(g) as gr:
        # mid-solve ranks: three iterations from uniform
        ranks, _ = gr.pagerank(max_iterations=3, tolerance=1e-30)
        got = gr.pagerank_contributions(ranks, 0.85)
    want64 = oracle.pagerank_contributions(g.row_offsets, g.column_indices, ranks, 0.85, fp64=True)
    want32 = oracle.pagerank_contributions(g.row_offsets, g.column_indices, ranks, 0.85, fp64=False)
    scale_ = max(float(np.abs(want64).max()), 1e-30)
    assert np.max(np.abs(got - want64)) <= 1e-12 * scale_ + 1e-18
    assert np.max(np.abs(got - want32)) <= 5e-6 * float(ranks.max())  # the reference's FP32 sums (long rows)


def test_unit_pagerank_contributions(hyt, gpu):
    """unit_tests.cpp:2903-2939: 0 -> {1, 2}, 1 -> 2, ranks {1, 0, 0}."""
    g = hyt.CSR(np.array([0, 2, 3, 3], np.uint64), np.array([1, 2, 2], np.uint32))
    with hyt.Graph(g) as gr:
        c = gr.pagerank_contributions(np.array([1, 0, 0], np.float32), 0.85)
    assert np.allclose(c, [0.95, 0.475, 0.475], atol=1e-5)


def test_partition_contributions(hyt, gpu):
    rng = np.random.default_rng(1)
    c = rng.random(100000)
    bounds = np.array([0, 10, 10, 5000, 99999, 100000], np.uint64)
    got = hyt.partition_contributions(c, bounds)
    want = [c[int(a):int(b)].sum() for a, b in zip(bounds[:-1], bounds[1:])]
    assert np.allclose(got, want, rtol=1e-13, atol=0)
    with pytest.raises(hyt.HytError):
        hyt.partition_contributions(c, np.array([0, 200000], np.uint64))
