"""C ABI: the library loads, exports every symbol include/hyt/capi.h
declares, fails cleanly without a GPU, and the host generator matches an
independent numpy restatement of its definition."""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

from conftest import ROOT

GOLDEN = np.uint64(0x9E3779B97F4A7C15)


def _declared(header):
    text = (ROOT / "include" / "hyt" / header).read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(hyt_\w+)\s*\(", text, re.M)))


def test_every_declared_symbol_is_exported(hyt):
    names = _declared("capi.h")
    assert len(names) >= 12
    for n in names:
        assert hasattr(hyt.capi.lib, n), n
    assert set(hyt.capi.EXPORTED) <= set(names)


def test_abi_version_and_errors_without_device(hyt):
    lib = hyt.capi.lib
    assert lib.hyt_abi_version() == 1
    n = hyt.device_count()
    assert n >= 0
    if n == 0:
        g = hyt.rmat(6, 4, 1)
        with pytest.raises(hyt.HytError) as e:
            hyt.Graph(g)
        assert e.value.code == hyt.capi.HYT_E_NO_DEVICE
        assert "no CUDA device" in hyt.capi.last_error()
        with pytest.raises(hyt.HytError) as e:
            hyt.measure_peaks()
        assert e.value.code == hyt.capi.HYT_E_NO_DEVICE


def test_invalid_generator_params(hyt):
    with pytest.raises(hyt.HytError) as e:
        hyt.rmat(0, 4, 1)
    assert e.value.code == hyt.capi.HYT_E_INVALID
    with pytest.raises(hyt.HytError):
        hyt.rmat(8, 4, 1, a=0.9, b=0.2, c=0.1)
    with pytest.raises(hyt.HytError):
        hyt.rmat(8, 0, 1)


def _mix64(z):
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def _numpy_rmat(scale, ef, seed, a=0.57, b=0.19, c=0.19, wmin=1, wmax=63):
    """Independent restatement of the generator's definition."""
    n = ef << scale
    i = np.arange(n, dtype=np.uint64)
    thr = [min(int(x * 4294967296.0), 0xFFFFFFFF) for x in (a, a + b, a + b + c)]
    src = np.zeros(n, np.uint64)
    dst = np.zeros(n, np.uint64)
    with np.errstate(over="ignore"):
        for lvl in range(scale):
            if lvl % 2 == 0:
                word = _mix64(np.uint64(seed) + GOLDEN * (np.uint64(16) * i + np.uint64(lvl >> 1)))
            r = (word >> np.uint64(32)) if lvl % 2 else (word & np.uint64(0xFFFFFFFF))
            bit = np.uint64(1 << (scale - 1 - lvl))
            q_b = (r >= thr[0]) & (r < thr[1])
            q_c = (r >= thr[1]) & (r < thr[2])
            q_d = r >= thr[2]
            dst |= np.where(q_b | q_d, bit, np.uint64(0))
            src |= np.where(q_c | q_d, bit, np.uint64(0))
    keep = src != dst
    keys = np.unique((src[keep] << np.uint64(32)) | dst[keep])
    V = 1 << scale
    s = (keys >> np.uint64(32)).astype(np.int64)
    off = np.searchsorted(s, np.arange(V + 1), side="left").astype(np.uint64)
    cols = (keys & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    wseed = _mix64(np.uint64(seed) ^ np.uint64(0x5EEDF00DCAFEBABE))
    w = (np.uint64(wmin) + _mix64(keys ^ wseed) % np.uint64(wmax - wmin + 1)).astype(np.uint32)
    return off, cols, w


@pytest.mark.parametrize("scale,ef,seed", [(6, 4, 1), (9, 16, 12345), (12, 8, 99)])
def test_host_generator_matches_numpy_restatement(hyt, scale, ef, seed):
    g = hyt.rmat(scale, ef, seed)
    off, cols, w = _numpy_rmat(scale, ef, seed)
    assert np.array_equal(g.row_offsets, off)
    assert np.array_equal(g.column_indices, cols)
    assert np.array_equal(g.weights, w)


def test_generator_properties(hyt):
    g = hyt.rmat(14, 16, 4242)
    V = g.num_vertices
    off, cols = g.row_offsets, g.column_indices
    src = np.repeat(np.arange(V, dtype=np.uint64), np.diff(off).astype(np.int64))
    keys = (src << np.uint64(32)) | cols.astype(np.uint64)
    assert np.all(keys[1:] > keys[:-1])                                  # sorted, no duplicates
    assert np.all(src != cols)                                           # no self-loops
    assert g.weights.min() >= 1 and g.weights.max() <= 63
    assert 0.85 * 16 * V < g.num_edges < 16 * V
    u = hyt.rmat(10, 4, 1, 0, 0)
    assert u.weights is None
    assert hyt.rmat(14, 16, 4242).column_indices.tobytes() == cols.tobytes()  # deterministic


def test_pick_sources(hyt):
    g = hyt.rmat(10, 8, 3)
    s = hyt.pick_sources(g.row_offsets, 11, 8)
    assert len(set(s.tolist())) == 8
    assert np.all(np.diff(g.row_offsets)[s] > 0)
    assert np.array_equal(s, hyt.pick_sources(g.row_offsets, 11, 8))
    off = np.array([0, 0, 1, 1], np.uint64)  # only vertex 1 has an edge
    assert hyt.pick_sources(off, 1, 3).tolist() == [1, 1, 1]
    with pytest.raises(hyt.HytError):
        hyt.pick_sources(np.zeros(4, np.uint64), 1, 1)


def test_host_library_exports(hyt):
    lib = C.CDLL(str(ROOT / "hytgraph_b200" / "lib" / "libhytgraph.so"))
    import subprocess

    out = subprocess.run(["nm", "-DC", "--defined-only", str(ROOT / "hytgraph_b200" / "lib" / "libhytgraph.so")],
                         capture_output=True, text=True, check=True).stdout
    for sym in ["hytgraph::algorithms::pagerank_gpu", "hytgraph::algorithms::sssp_gpu",
                "hytgraph::transfer::HyTMCostModel::select_engine", "hytgraph::scheduling::TaskCombiner::combine",
                "hytgraph::transfer::ExpTMCompaction::compact", "hytgraph::transfer::ImpTMZeroCopy::prepare",
                "hytgraph::transfer::ExpTMFilter::plan", "hytgraph::graph::LogicalPartitioner::partition"]:
        assert sym in out, sym
    assert lib is not None


def test_csr_rejects_wrong_dtypes(hyt):
    off = np.array([0, 1, 2], np.uint64)
    cols = np.array([1, 0], np.uint32)
    with pytest.raises(TypeError):
        hyt.CSR(off, cols, np.array([1, 1])).to_c()            # int64 weights
    with pytest.raises(TypeError):
        hyt.CSR(off.astype(np.int64), cols).to_c()
    assert hyt.CSR(off, cols, np.array([1, 1], np.uint32)).to_c().weight_kind == hyt.capi.HYT_WEIGHTS_U32
    assert hyt.CSR(off, cols, np.array([1, 1], np.float32)).to_c().weight_kind == hyt.capi.HYT_WEIGHTS_F32
