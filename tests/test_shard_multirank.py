"""Sharded solves (hytgraph_b200.shard.ShardedGraph) at world sizes 2 and 3
on CPU processes (gloo): the exchange, the shared stop rule and the final
gather, with the CPU stand-in kernels of shard_standin.py in place of the
GPU ones.  Every process must return the same result, equal to the oracle's
(PageRank / personalized PageRank: L1 <= 1e-5 against FP64; SSSP: bit for
bit)."""
from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]
L1_TOL = 1e-5


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _graph(seed: int, V: int = 1500, max_deg: int = 24):
    """Random graph with a hub (vertex 7: in- and out-degree ~V/2), some
    dangling vertices and uint32 weights."""
    rng = np.random.default_rng(seed)
    deg = rng.integers(0, max_deg, V)
    deg[rng.choice(V, V // 20, replace=False)] = 0
    deg[7] = V // 2
    off = np.concatenate([[0], np.cumsum(deg)]).astype(np.uint64)
    cols = rng.integers(0, V, int(off[-1])).astype(np.uint32)
    cols[rng.random(cols.shape[0]) < 0.3] = 7
    for v in range(V):  # sorted rows (duplicates kept)
        a, b = int(off[v]), int(off[v + 1])
        cols[a:b] = np.sort(cols[a:b])
    w = rng.integers(1, 64, cols.shape[0]).astype(np.uint32)
    return off, cols, w


def _solve(part: int, parts: int, seed: int, sources):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from shard_standin import NumpyShardKernels

    from hytgraph_b200.shard import ShardedGraph

    off, cols, w = _graph(seed)
    sg = ShardedGraph(kernels=NumpyShardKernels(off, cols, w, part, parts))
    r, st = sg.pagerank()
    out = {"pr": (r, st)}
    out["ppr"] = [sg.ppr(int(s)) for s in sources]
    out["sssp"] = [sg.sssp(int(s)) for s in sources]
    return out


def _rank_main(rank: int, world: int, port: int, seed: int, sources, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        out[rank] = _solve(rank, world, seed, sources)
    finally:
        dist.destroy_process_group()


def _run(world: int, seed: int, sources):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank_main, args=(r, world, port, seed, sources, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        return dict(out)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_solves_match_the_oracle(world, oracle):
    seed, sources = 5, [0, 7, 1234]
    off, cols, w = _graph(seed)
    res = _run(world, seed, sources)
    assert sorted(res) == list(range(world))
    single = _solve(0, 1, seed, sources)  # one shard, no process group

    ref, it_ref, _, conv_ref = oracle.pagerank_f64(off, cols)
    ranges = set()
    for rank in range(world):
        r, st = res[rank]["pr"]
        assert np.array_equal(r.view(np.uint32), res[0]["pr"][0].view(np.uint32))  # same on every process
        assert float(np.abs(r.astype(np.float64) - ref).sum()) <= L1_TOL
        assert st["iterations"] == res[0]["pr"][1]["iterations"]
        assert abs(st["iterations"] - it_ref) <= 1 and st["converged"] == conv_ref
        assert st["parts"] == world and st["part"] == rank
        V = off.shape[0] - 1  # one contribution vector per iteration + the final ranks
        assert st["exchanged_bytes"] == 4 * V * (st["iterations"] + 1)
        ranges.add((st["vertex_begin"], st["vertex_end"]))
    # the ranges tile [0, V)
    b = sorted(ranges)
    assert b[0][0] == 0 and b[-1][1] == off.shape[0] - 1
    assert all(b[i][1] == b[i + 1][0] for i in range(len(b) - 1))
    r1, st1 = single["pr"]
    assert float(np.abs(r1.astype(np.float64) - res[0]["pr"][0]).sum()) <= 1e-6
    assert st1["iterations"] == res[0]["pr"][1]["iterations"]

    w32 = w.astype(np.float32)
    for i, s in enumerate(sources):
        pref, _, _, _ = oracle.ppr_f64(off, cols, s)
        want, _, _ = oracle.sssp(off, cols, w32, s)
        fin = np.isfinite(want)
        want = np.where(fin, np.where(fin, want, 0).astype(np.uint64), 0xFFFFFFFF).astype(np.uint32)
        for rank in range(world):
            r, _ = res[rank]["ppr"][i]
            assert float(np.abs(r.astype(np.float64) - pref).sum()) <= L1_TOL
            d, st = res[rank]["sssp"][i]
            assert np.array_equal(d, want), (rank, s)
            assert st["converged"] == 1
        assert np.array_equal(single["sssp"][i][0], want)


def test_sharded_bounds_split_work_evenly():
    sys.path.insert(0, str(ROOT / "tests"))
    from shard_standin import PULL, PUSH, NumpyShardKernels

    off, cols, w = _graph(9, V=4000)
    for parts in (1, 2, 5, 8):
        k = NumpyShardKernels(off, cols, w, 0, parts)
        for kind, o in ((PULL, k.in_off), (PUSH, k.off)):
            b = k.bounds(kind)
            assert b[0] == 0 and b[-1] == k.num_vertices and b == sorted(b)
            cost = [int(o[b[p + 1]]) + b[p + 1] - int(o[b[p]]) - b[p] for p in range(parts)]
            total = int(o[-1]) + k.num_vertices
            # a part exceeds its share by at most one row (the hub)
            row = int(np.diff(o.astype(np.int64)).max()) + 1
            assert max(cost) <= total / parts + row, (parts, kind, cost)


def test_sharded_argument_errors():
    sys.path.insert(0, str(ROOT / "tests"))
    from shard_standin import NumpyShardKernels

    import hytgraph_b200 as hyt

    off, cols, w = _graph(3, V=200)
    sg = hyt.ShardedGraph(kernels=NumpyShardKernels(off, cols, w, 0, 1))
    for kw in ({"tolerance": 0.0}, {"tolerance": float("nan")}, {"max_iterations": 0}):
        with pytest.raises(hyt.HytError) as e:
            sg.pagerank(**kw)
        assert e.value.code == hyt.capi.HYT_E_INVALID
    with pytest.raises(hyt.HytError):
        sg.ppr(0, restart=0.0)
    r, st = sg.pagerank(tolerance=1e-30, max_iterations=3)
    assert st["iterations"] == 3 and st["converged"] == 0
    d, st = sg.sssp(0, max_rounds=1)
    assert st["iterations"] == 1
    with pytest.raises(ValueError):
        hyt.ShardedGraph()


def _group_main(rank: int, world: int, port: int, seed: int, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "tests"))
    from shard_standin import NumpyShardKernels

    from hytgraph_b200.shard import ShardedGraph

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        groups = [dist.new_group([0, 1]), dist.new_group([2, 3])]  # every rank creates every group
        group = groups[rank // 2]
        off, cols, w = _graph(seed)
        part, parts = dist.get_rank(group), dist.get_world_size(group)
        sg = ShardedGraph(group=group, kernels=NumpyShardKernels(off, cols, w, part, parts))
        r, st = sg.pagerank()
        d, _ = sg.sssp(7)
        out[rank] = (r, st["part"], st["parts"], d)
    finally:
        dist.destroy_process_group()


def test_sharded_solves_inside_subgroups(oracle):
    """Four processes as two independent two-shard solves (process groups
    {0, 1} and {2, 3}): slice owners are addressed by their global ranks."""
    seed = 11
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = _free_port()
        procs = [ctx.Process(target=_group_main, args=(r, 4, port, seed, out)) for r in range(4)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        res = dict(out)
    off, cols, w = _graph(seed)
    ref, _, _, _ = oracle.pagerank_f64(off, cols)
    want, _, _ = oracle.sssp(off, cols, w.astype(np.float32), 7)
    fin = np.isfinite(want)
    want = np.where(fin, np.where(fin, want, 0).astype(np.uint64), 0xFFFFFFFF).astype(np.uint32)
    assert [(res[r][1], res[r][2]) for r in range(4)] == [(0, 2), (1, 2), (0, 2), (1, 2)]
    for r in range(4):
        assert np.array_equal(res[r][0].view(np.uint32), res[0][0].view(np.uint32))
        assert float(np.abs(res[r][0].astype(np.float64) - ref).sum()) <= L1_TOL
        assert np.array_equal(res[r][3], want)
