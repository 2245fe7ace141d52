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


def _device_csr(hyt, g, torch, weighted=True):
    off = torch.from_numpy(g.row_offsets.view(np.int64)).cuda()
    cols = torch.from_numpy(g.column_indices.view(np.int32)).cuda()
    w = torch.from_numpy(g.weights.view(np.int32)).cuda() if weighted else None
    c = hyt.capi.hyt_csr()
    c.num_vertices, c.num_edges = g.num_vertices, g.num_edges
    c.row_offsets, c.column_indices = off.data_ptr(), cols.data_ptr()
    c.weights = w.data_ptr() if weighted else 0
    c.weight_kind = hyt.capi.HYT_WEIGHTS_U32 if weighted else hyt.capi.HYT_WEIGHTS_NONE
    return c, (off, cols, w)


def _noalloc(hyt, csr, source, out):
    st = hyt.capi.hyt_run_stats()
    rc = hyt.capi.lib.hyt_sssp_noalloc(C.byref(csr), source, out.data_ptr(), None, C.byref(st))
    return rc, st


def test_noalloc_matches_the_allocating_entry_point(hyt, gpu):
    """Two calls in a row (and a repeat of the first) agree bit for bit with
    hyt_sssp, the allocating entry point; SSSP distances are exact."""
    import torch

    g = hyt.rmat(16, 16, 777)
    sources = [int(s) for s in hyt.pick_sources(g.row_offsets, 31, 2)]
    with hyt.Graph(g) as dg:
        want = [dg.sssp(s)[0] for s in sources]
    for weighted in (True, False):
        csr, keep = _device_csr(hyt, g, torch, weighted)
        if not weighted:
            with hyt.Graph(hyt.CSR(g.row_offsets, g.column_indices, None)) as dg:
                want = [dg.sssp(s)[0] for s in sources]
        for s, ref in zip(sources + sources[:1], want + want[:1]):
            out = torch.full((g.num_vertices,), 7, dtype=torch.int32, device="cuda")
            rc, st = _noalloc(hyt, csr, s, out)
            assert rc == hyt.capi.HYT_OK, hyt.capi.last_error()
            assert st.converged == 1 and st.iterations > 0
            assert np.array_equal(out.cpu().numpy().view(np.uint32), ref)
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
