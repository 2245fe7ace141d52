"""Model of the SSSP pull sweep's row skipping, run on the CPU.

The CUDA pull sweep (hytgraph_b200/csrc/sssp.cu, sssp_pull_kernel) skips
every row whose label is at most extend(fmin, min_w): fmin is the lowest
label in the round's frontier (found by sssp_round_close_kernel), min_w the
graph's smallest weight with the sign of -0.0 cleared.  This model runs the
same round structure in Python -- push rounds over the frontier, in-place
pull sweeps over the CSC when the frontier's out-edges exceed E / 4, rows
and frontier vertices visited in a shuffled order in place of the GPU's
unordered tiles and warps -- and checks that skipping leaves the distances
equal to the oracle's (Dijkstra for integer weights, the reference's float
Bellman-Ford for float weights) while relaxing fewer edges.
"""
import numpy as np
import pytest

INF = float("inf")


def _csc(off, cols, w):
    V = off.shape[0] - 1
    src = np.repeat(np.arange(V, dtype=np.int64), np.diff(off).astype(np.int64))
    order = np.argsort(cols, kind="stable")
    in_off = np.zeros(V + 1, np.int64)
    np.cumsum(np.bincount(cols, minlength=V), out=in_off[1:])
    return in_off, src[order], w[order]


def _solve(off, cols, w, source, add, min_w, skip, seed):
    """Label-correcting rounds with the product's push / pull rule; returns
    (labels, relaxed edges, pull sweeps)."""
    V, E = off.shape[0] - 1, cols.shape[0]
    in_off, in_src, in_w = _csc(off, cols, w)
    off_l, cols_l, w_l = off.tolist(), cols.tolist(), w.tolist()
    in_off_l, in_src_l, in_w_l = in_off.tolist(), in_src.tolist(), in_w.tolist()
    rng = np.random.default_rng(seed)
    d = [INF] * V
    d[source] = add(0.0, 0.0)
    front = {source}
    relaxed = pulls = 0
    while front:
        nxt = set()
        if sum(off_l[u + 1] - off_l[u] for u in front) * 4 > E:
            pulls += 1
            bound = add(min(d[u] for u in front), min_w)
            for v in rng.permutation(V).tolist():
                if skip and d[v] <= bound:
                    continue  # no in-edge can lower d[v] this round
                best = d[v]
                for i in range(in_off_l[v], in_off_l[v + 1]):
                    relaxed += 1
                    du = d[in_src_l[i]]
                    if du != INF:
                        best = min(best, add(du, in_w_l[i]))
                if best < d[v]:
                    d[v] = best
                    nxt.add(v)
        else:
            for u in rng.permutation(sorted(front)).tolist():
                for i in range(off_l[u], off_l[u + 1]):
                    relaxed += 1
                    c = add(d[u], w_l[i])
                    v = cols_l[i]
                    if c < d[v]:
                        d[v] = c
                        nxt.add(v)
        front = nxt
    return d, relaxed, pulls


def _add_u32(a, b):
    return min(a + b, 0xFFFFFFFE)  # the product's saturating integer extend


def _add_f32(a, b):
    return float(np.float32(a) + np.float32(b))


@pytest.mark.parametrize("wmin,wmax", [(0, 4), (1, 63), (3, 9)])
def test_skipping_keeps_integer_distances(oracle, wmin, wmax):
    off, cols, w = oracle.rmat(10, 8, 20 + wmin, weight_min=wmin, weight_max=wmax)
    min_w = int(w.min())
    for s in oracle.pick_sources(off, 5, 3):
        want = oracle.dijkstra(off, cols, w, int(s))
        want = [INF if x == np.iinfo(np.uint64).max or x >= 0xFFFFFFFF else int(x) for x in want]
        got, relaxed, pulls = _solve(off, cols, w.astype(np.int64), int(s), _add_u32, min_w, True, 1)
        ref, relaxed_all, pulls_all = _solve(off, cols, w.astype(np.int64), int(s), _add_u32, min_w, False, 1)
        assert got == ref == want, int(s)
        assert pulls >= 1 and pulls_all >= 1
        assert relaxed < relaxed_all


def test_skipping_keeps_float_distances_with_negative_zero(oracle):
    off, cols, _ = oracle.rmat(10, 8, 7)
    rng = np.random.default_rng(3)
    wf = (rng.random(cols.shape[0]) * 10).astype(np.float32)
    wf[::7] = np.float32(-0.0)  # passes validation (>= 0) and counts as weight 0
    wf[3::11] = np.float32(0.0)
    bits = wf.view(np.uint32) & np.uint32(0x7FFFFFFF)  # the product's min_w: sign of -0.0 cleared
    min_w = float(bits.min().view(np.float32))
    assert min_w == 0.0
    for s in oracle.pick_sources(off, 9, 2):
        ref, _, _ = oracle.sssp(off, cols, wf, int(s))
        want = [float(x) for x in ref]
        got, relaxed, pulls = _solve(off, cols, wf.astype(np.float64), int(s), _add_f32, min_w, True, 2)
        base, relaxed_all, _ = _solve(off, cols, wf.astype(np.float64), int(s), _add_f32, min_w, False, 2)
        assert got == base == want, int(s)
        assert pulls >= 1 and relaxed <= relaxed_all


def test_a_wrong_bound_is_caught(oracle):
    """The check has teeth: a bound one unit too loose (min_w + 1 on a graph
    whose smallest weight occurs) skips rows that could still improve."""
    off, cols, w = oracle.rmat(10, 8, 21, weight_min=0, weight_max=2)
    bad = 0
    for s in oracle.pick_sources(off, 5, 4):
        want = oracle.dijkstra(off, cols, w, int(s))
        want = [INF if x >= 0xFFFFFFFF else int(x) for x in want]
        got, _, _ = _solve(off, cols, w.astype(np.int64), int(s), _add_u32, int(w.min()) + 1, True, 1)
        bad += got != want
    assert bad > 0
