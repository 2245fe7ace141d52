"""hyt_sssp_noalloc: the SSSP entry point for callers that cannot allocate
device memory -- for example an application whose own caching allocator has
already reserved the GPU's free memory, a latency-critical loop that cannot
afford cudaMalloc's implicit device synchronisation, or a plugin host that
forbids its components to allocate.  The caller owns the CSR and the output
array; the solver's state lives in a fixed device array inside the library.

This file is collected last so that a run stopping at its first failure has
already run every other test; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_csr(hyt, off, cols, w, torch):
    """Device copies of host CSR arrays and the hyt_csr describing them."""
    d_off = torch.from_numpy(np.ascontiguousarray(off).view(np.int64)).cuda()
    d_cols = torch.from_numpy(np.ascontiguousarray(cols).view(np.int32)).cuda()
    d_w = None if w is None else torch.from_numpy(np.ascontiguousarray(w).view(np.int32)).cuda()
    c = hyt.capi.hyt_csr()
    c.num_vertices, c.num_edges = off.shape[0] - 1, cols.shape[0]
    c.row_offsets, c.column_indices = d_off.data_ptr(), d_cols.data_ptr()
    c.weights = 0 if w is None else d_w.data_ptr()
    if w is None:
        c.weight_kind = hyt.capi.HYT_WEIGHTS_NONE
    else:
        c.weight_kind = hyt.capi.HYT_WEIGHTS_F32 if w.dtype == np.float32 else hyt.capi.HYT_WEIGHTS_U32
    return c, (d_off, d_cols, d_w)


def _noalloc(hyt, csr, source, out):
    st = hyt.capi.hyt_run_stats()
    rc = hyt.capi.lib.hyt_sssp_noalloc(C.byref(csr), source, out.data_ptr(), None, C.byref(st))
    return rc, st


def _memory(torch):
    torch.cuda.synchronize()
    return torch.cuda.mem_get_info()[0], torch.cuda.memory_reserved()


@pytest.mark.parametrize("weights", ["u32", "none", "f32"])
def test_noalloc_matches_the_allocating_entry_point(hyt, gpu, weights):
    """Two calls in a row (and a repeat of the first) agree bit for bit with
    hyt_sssp, the allocating entry point (SSSP distances are exact), and no
    call after the first changes the device's free memory or torch's
    reserved memory."""
    import torch

    g = hyt.rmat(16, 16, 777)
    w = {"u32": g.weights, "none": None, "f32": g.weights.astype(np.float32) / 4}[weights]
    sources = [int(s) for s in hyt.pick_sources(g.row_offsets, 31, 2)]
    with hyt.Graph(hyt.CSR(g.row_offsets, g.column_indices, w)) as dg:
        want = [dg.sssp(s)[0] for s in sources]
    csr, keep = _device_csr(hyt, g.row_offsets, g.column_indices, w, torch)
    outs = [torch.full((g.num_vertices,), 7, dtype=torch.int32, device="cuda") for _ in range(3)]
    rc, _ = _noalloc(hyt, csr, sources[0], outs[0])  # first call: the library looks up its array
    assert rc == hyt.capi.HYT_OK, hyt.capi.last_error()
    before = _memory(torch)
    for s, ref, out in zip(sources + sources[:1], want + want[:1], outs):
        out.fill_(7)
        rc, st = _noalloc(hyt, csr, s, out)
        assert rc == hyt.capi.HYT_OK, hyt.capi.last_error()
        assert st.converged == 1 and st.iterations > 0
        assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
    assert _memory(torch) == before, "hyt_sssp_noalloc allocated device memory"
    del keep


def test_noalloc_rejects_graphs_beyond_its_capacity(hyt, gpu):
    import torch

    V = hyt.capi.HYT_NOALLOC_MAX_VERTICES
    off = torch.zeros(V + 2, dtype=torch.int64, device="cuda")  # V + 1 vertices, no edges
    c = hyt.capi.hyt_csr()
    c.num_vertices, c.num_edges = V + 1, 0
    c.row_offsets, c.column_indices, c.weights = off.data_ptr(), 0, 0
    c.weight_kind = hyt.capi.HYT_WEIGHTS_NONE
    out = torch.empty(V + 1, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(hyt, c, 0, out)
    assert rc == hyt.capi.HYT_E_INVALID
    assert "capacity" in hyt.capi.last_error()
    # host buffers are refused: the caller must pass device memory
    g = hyt.rmat(8, 4, 1)
    host = g.to_c()
    out_small = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
    rc, _ = _noalloc(hyt, host, 0, out_small)
    assert rc == hyt.capi.HYT_E_INVALID and "device memory" in hyt.capi.last_error()


def test_noalloc_rejects_malformed_csr(hyt, gpu):
    """Malformed offsets, an out-of-range column and a negative float weight
    are caught on the device before any solver kernel indexes with them."""
    import torch

    g = hyt.rmat(10, 8, 5)
    out = torch.empty(g.num_vertices, dtype=torch.int32, device="cuda")
    bad_off = g.row_offsets.copy()
    bad_off[5], bad_off[6] = bad_off[6] + 1, bad_off[5]  # a decreasing pair
    bad_cols = g.column_indices.copy()
    bad_cols[g.num_edges // 2] = g.num_vertices  # destination out of range
    bad_w = g.weights.astype(np.float32)
    bad_w[3] = -1.0
    cases = [(bad_off, g.column_indices, g.weights, "row offsets"),
             (g.row_offsets, bad_cols, g.weights, "invalid destination"),
             (g.row_offsets, g.column_indices, bad_w, "non-negative")]
    for off, cols, w, msg in cases:
        csr, keep = _device_csr(hyt, off, cols, w, torch)
        rc, _ = _noalloc(hyt, csr, 0, out)
        assert rc == hyt.capi.HYT_E_INVALID, msg
        assert msg in hyt.capi.last_error()
        del keep
    # a valid call right after the rejections still matches hyt_sssp
    csr, keep = _device_csr(hyt, g.row_offsets, g.column_indices, g.weights, torch)
    src = int(hyt.pick_sources(g.row_offsets, 3, 1)[0])
    rc, _ = _noalloc(hyt, csr, src, out)
    assert rc == hyt.capi.HYT_OK, hyt.capi.last_error()
    with hyt.Graph(g) as dg:
        assert np.array_equal(out.cpu().numpy().view(np.uint32), dg.sssp(src)[0])
