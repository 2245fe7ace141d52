"""Packed personalized PageRank (hyt_ppr_multi): every query within the
FP64 oracle's tolerance, the same bits alone and packed, sources and
results in the caller's ids on hub-ordered graphs."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale", [12, 16])
def test_ppr_multi_matches_oracle(hyt, gpu, oracle, scale):
    g = hyt.rmat(scale, 16, 40 + scale)
    srcs = hyt.pick_sources(g.row_offsets, 7, 8)
    with hyt.Graph(g) as gr:
        got, st = gr.ppr_multi(srcs, tolerance=1e-7, max_iterations=300)
    for l, s in enumerate(srcs):
        want = oracle.ppr_f64(g.row_offsets, g.column_indices, int(s), 0.15, 1e-12, 600)[0]
        assert np.abs(got[l].astype(np.float64) - want).sum() <= 1e-5, (scale, l)
        assert st[l]["converged"] == 1 and st[l]["iterations"] > 0


def test_ppr_multi_same_alone_and_packed(hyt, gpu):
    g = hyt.rmat(15, 16, 3)
    srcs = hyt.pick_sources(g.row_offsets, 11, 8)
    with hyt.Graph(g) as gr:
        packed, pst = gr.ppr_multi(srcs)
        for l in (0, 3, 7):
            alone, ast = gr.ppr_multi(srcs[l:l + 1])
            assert np.array_equal(alone[0].view(np.uint32), packed[l].view(np.uint32)), l
            assert ast[0]["iterations"] == pst[l]["iterations"]
        three, _ = gr.ppr_multi(srcs[[5, 1, 6]])
        assert np.array_equal(three[1].view(np.uint32), packed[1].view(np.uint32))
        # close to the single-source solver (both converged to 1e-6)
        one, _ = gr.ppr(int(srcs[2]))
        assert np.abs(one.astype(np.float64) - packed[2]).sum() <= 2e-5


def test_ppr_multi_hub_order_and_device_out(hyt, gpu):
    import torch

    g = hyt.rmat(14, 16, 9)
    srcs = hyt.pick_sources(g.row_offsets, 2, 5)
    with hyt.Graph(g) as a, hyt.Graph(g, flags=hyt.capi.HYT_GRAPH_ALL | hyt.capi.HYT_GRAPH_HUB_ORDER) as b:
        ra, _ = a.ppr_multi(srcs)
        out = torch.empty((5, g.num_vertices), dtype=torch.float32, device="cuda")
        b.ppr_multi(srcs, out=out)
        rb = out.cpu().numpy()
    for l in range(5):
        assert np.abs(ra[l].astype(np.float64) - rb[l]).sum() <= 2e-5


def test_ppr_multi_rejects_bad_calls(hyt, gpu):
    g = hyt.rmat(10, 8, 1)
    with hyt.Graph(g) as gr:
        for bad in ([], list(range(9))):
            with pytest.raises(hyt.HytError) as e:
                gr.ppr_multi(np.array(bad, np.uint32))
            assert e.value.code == hyt.capi.HYT_E_INVALID
        with pytest.raises(hyt.HytError):
            gr.ppr_multi([g.num_vertices])
        with pytest.raises(hyt.HytError):
            gr.ppr_multi([0], restart=0.0)
