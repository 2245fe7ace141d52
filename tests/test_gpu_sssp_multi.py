"""hyt_sssp_multi: up to 8 SSSP sources in one shared solve.  Each source's
labels must equal hyt_sssp's bit for bit (SSSP is exact), for unit, uint32
and float weights, in input and hub vertex order, with push rounds and pull
sweeps, duplicate sources and fewer than 8 lanes."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cases(hyt):
    g = hyt.rmat(17, 16, 41)
    yield "u32", g
    yield "none", hyt.CSR(g.row_offsets, g.column_indices, None)
    yield "f32", hyt.CSR(g.row_offsets, g.column_indices, g.weights.astype(np.float32) / 3)
    yield "u32-s20", hyt.rmat(20, 16, 5)


@pytest.mark.parametrize("flags_name", ["ALL", "HUB"])
def test_sssp_multi_matches_single_source(hyt, gpu, flags_name):
    flags = hyt.capi.HYT_GRAPH_ALL | (hyt.capi.HYT_GRAPH_HUB_ORDER if flags_name == "HUB" else 0)
    for name, g in _cases(hyt):
        srcs = [int(s) for s in hyt.pick_sources(g.row_offsets, 99, 8)]
        with hyt.Graph(g, flags=flags) as dg:
            want = [dg.sssp(s)[0] for s in srcs]
            for k in (8, 3, 1):
                got, st = dg.sssp_multi(srcs[:k])
                assert st["converged"] == 1, (name, k)
                for lane in range(k):
                    assert np.array_equal(got[lane], want[lane]), (name, k, lane)
            # a pull sweep counts every edge: the 8-source solve of the
            # larger graphs takes at least one
            if name == "u32-s20":
                got, st = dg.sssp_multi(srcs)
                assert st["edges_processed"] >= g.num_edges


def test_sssp_multi_duplicates_device_output_and_errors(hyt, gpu):
    import torch

    g = hyt.rmat(15, 8, 3)
    s = [int(x) for x in hyt.pick_sources(g.row_offsets, 4, 2)]
    srcs = [s[0], s[1], s[0], s[0]]
    with hyt.Graph(g) as dg:
        want = {x: dg.sssp(x)[0] for x in set(srcs)}
        out = torch.empty((4, g.num_vertices), dtype=torch.int32, device="cuda")
        dg.sssp_multi(srcs, out=out)
        got = out.cpu().numpy().view(np.uint32)
        for lane, x in enumerate(srcs):
            assert np.array_equal(got[lane], want[x])
        for bad in ([], list(range(9)), [g.num_vertices]):
            with pytest.raises(hyt.HytError) as e:
                dg.sssp_multi(bad)
            assert e.value.code == hyt.capi.HYT_E_INVALID


def test_sssp_multi_staged_pull_matches(hyt, gpu):
    """With HYT_STAGED=1 (256-unit tiles) the pull sweeps stage ids by bulk
    copies instead of reading them in place; the labels are the same fixed
    point, equal to the default build's for all 8 lanes."""
    import os
    import subprocess
    import sys

    from conftest import ROOT

    code = ("import sys; sys.path.insert(0, %r); import hytgraph_b200 as hyt; "
            "g = hyt.rmat(20, 16, 5); src = [int(s) for s in hyt.pick_sources(g.row_offsets, 99, 8)]; "
            "dg = hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER); "
            "d, st = dg.sssp_multi(src); assert st['edges_processed'] >= g.num_edges, st; "
            "sys.stdout.buffer.write(d.tobytes())") % str(ROOT)
    outs = []
    for staged in ("1", "0"):
        r = subprocess.run([sys.executable, "-c", code], capture_output=True,
                           env=dict(os.environ, HYT_STAGED=staged), timeout=600)
        assert r.returncode == 0, r.stderr.decode()[-2000:]
        outs.append(r.stdout)
    assert outs[0] == outs[1] and len(outs[0]) > 0
