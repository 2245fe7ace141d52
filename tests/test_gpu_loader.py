"""Edge-list loading (hyt_load_edge_list), CSR construction on the GPU
(hyt_csr_from_edges) and the binary CSR file (hyt_csr_save / hyt_csr_load),
against the oracle and the reference's GraphLoader expectations.

Arrays are compared bit for bit; errors by status code and message.
"""
from __future__ import annotations

import numpy as np
import pytest

from test_oracle import LOADER_CASES, loader_corpus

pytestmark = pytest.mark.gpu


def _same(a, b):
    if a is None or b is None:
        return a is None and b is None
    return a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def _ours(hyt, path, V, weighted, device=False):
    try:
        g = hyt.load_edge_list(path, V, weighted, device=device)
        return g.download() if device else g
    except hyt.HytError as e:
        assert e.code == hyt.capi.HYT_E_INVALID, e
        return str(e).split("] ", 1)[1]


def _oracle(oracle, path, V, weighted):
    try:
        return oracle.load_edge_list(path, V, weighted)
    except ValueError as e:
        return str(e)


def _match(ours, want):
    if isinstance(ours, str) or isinstance(want, str):
        return ours == want
    return _same(ours.row_offsets, want[0]) and _same(ours.column_indices, want[1]) and _same(ours.weights, want[2])


def test_loader_known_answers(hyt, gpu, tmp_path):
    """unit_tests.cpp:374-599 through hyt_load_edge_list."""
    got = {}
    for name, text, V, weighted in LOADER_CASES:
        (tmp_path / name).write_text(text)
        got[name] = _ours(hyt, tmp_path / name, V, weighted)
    g = got["unweighted"]
    assert np.diff(g.row_offsets).tolist() == [2, 1, 1, 0] and g.column_indices.tolist() == [1, 2, 2, 0]
    assert g.weights is None
    g = got["weighted"]
    assert g.weights.dtype == np.float32 and g.weights.tolist() == [0.5, 1.25, 2.5]
    g = got["parallel"]
    assert g.row_offsets.tolist() == [0, 3, 3, 3] and g.column_indices.tolist() == [1, 1, 2]
    assert got["bad_vertex"] == "GraphLoader::load_edge_list: vertex ID out of range at line 1"
    assert got["missing_weight"] == "GraphLoader::load_edge_list: missing edge weight at line 1"
    assert got["malformed"] == "GraphLoader::load_edge_list: malformed edge at line 1"
    with pytest.raises(hyt.HytError) as e:
        hyt.load_edge_list(tmp_path / "does_not_exist", 4)
    assert e.value.code == hyt.capi.HYT_E_IO and "unable to open file" in str(e.value)


def test_loader_corpus_matches_oracle(hyt, gpu, oracle, tmp_path):
    path = tmp_path / "f.el"
    for i, (text, V, weighted) in enumerate(loader_corpus(11, 400)):
        path.write_text(text)
        want = _oracle(oracle, path, V, weighted)
        assert _match(_ours(hyt, path, V, weighted, device=bool(i % 2)), want), (i, text)


def _edge_text(src, dst, w=None, comments_every=0):
    lines = []
    for i in range(src.shape[0]):
        if comments_every and i % comments_every == 0:
            lines.append("# block %d" % i)
        lines.append(f"{src[i]} {dst[i]}" if w is None else f"{src[i]}\t{dst[i]} {w[i]!r}")
    return "\n".join(lines) + "\n"


def test_loader_large_multichunk(hyt, gpu, oracle, tmp_path):
    """A shuffled scale-16 edge list (about 30 MB, a million GPU parser
    threads) with float weights, and an error near its end reported at the
    right line."""
    g = hyt.rmat(16, 16, 5)
    src = np.repeat(np.arange(g.num_vertices, dtype=np.uint32), np.diff(g.row_offsets).astype(np.int64))
    rng = np.random.default_rng(2)
    perm = rng.permutation(g.num_edges)
    s, d = src[perm], g.column_indices[perm]
    w = (rng.random(g.num_edges) * 100).astype(np.float32)
    path = tmp_path / "big.el"
    path.write_text(_edge_text(s, d, [float(x) for x in w], comments_every=997))
    assert path.stat().st_size > 16 << 20
    st = {}
    ours = hyt.load_edge_list(path, g.num_vertices, True, stats=st)
    want = oracle.load_edge_list(path, g.num_vertices, True)
    assert _match(ours, want) and st["num_edges"] == g.num_edges and st["file_bytes"] == path.stat().st_size
    dev = hyt.load_edge_list(path, g.num_vertices, True, device=True).download()
    assert _match(dev, want)
    lines = path.read_text().split("\n")
    lines[-5] = "12 x"
    path.write_text("\n".join(lines))
    assert _ours(hyt, path, g.num_vertices, True) == _oracle(oracle, path, g.num_vertices, True)
    assert f"at line {len(lines) - 4}" in _ours(hyt, path, g.num_vertices, True)


def test_csr_from_edges(hyt, gpu, oracle):
    import torch

    rng = np.random.default_rng(8)
    for V, E in ((1, 0), (5, 40), (1000, 200000), (1 << 18, 3 << 20)):
        src = rng.integers(0, V, E).astype(np.uint32)
        dst = rng.integers(0, V, E).astype(np.uint32)
        for w in (None, rng.integers(0, 1 << 31, E).astype(np.uint32), rng.random(E).astype(np.float32)):
            want = oracle.csr_from_edges(V, src, dst, w)
            got = hyt.csr_from_edges(src, dst, V, weights=w)
            assert _match(got, want), (V, E, None if w is None else w.dtype)
    ts, td = torch.from_numpy(src.view(np.int32)).cuda(), torch.from_numpy(dst.view(np.int32)).cuda()
    st = {}
    got = hyt.csr_from_edges(ts, td, V, device=True, stats=st).download()
    assert _match(got, oracle.csr_from_edges(V, src, dst)) and st["kernel_ms"] > 0
    with pytest.raises(hyt.HytError) as e:
        hyt.csr_from_edges(np.array([0, 3, 1], np.uint32), np.array([1, 1, 9], np.uint32), 4)
    assert e.value.code == hyt.capi.HYT_E_INVALID and "edge 2" in str(e.value)


@pytest.mark.parametrize("kind", ["none", "u32", "f32"])
def test_binary_round_trip(hyt, gpu, tmp_path, kind):
    g = hyt.rmat(14, 16, 3)
    w = {"none": None, "u32": g.weights, "f32": g.weights.astype(np.float32) / 3}[kind]
    host = hyt.CSR(g.row_offsets, g.column_indices, w)
    p = tmp_path / f"g_{kind}.csr"
    hyt.save_csr(host, p)
    for device in (False, True):
        st = {}
        r = hyt.load_csr(p, device=device, stats=st)
        r = r.download() if device else r
        assert _same(r.row_offsets, host.row_offsets) and _same(r.column_indices, host.column_indices)
        assert _same(r.weights, w)
        assert st["file_bytes"] == p.stat().st_size
    # saved from device arrays: the same bytes
    d = hyt.rmat(14, 16, 3, device=True)
    if kind == "u32":
        p2 = tmp_path / "from_device.csr"
        hyt.save_csr(d, p2)
        assert p2.read_bytes() == p.read_bytes()
    d.free()


def test_binary_detects_damage(hyt, gpu, tmp_path):
    g = hyt.rmat(12, 8, 1)
    p = tmp_path / "g.csr"
    hyt.save_csr(g, p)
    raw = bytearray(p.read_bytes())

    def expect(data, words, device):
        q = tmp_path / "bad.csr"
        q.write_bytes(bytes(data))
        with pytest.raises(hyt.HytError) as e:
            hyt.load_csr(q, device=device)
        assert e.value.code == hyt.capi.HYT_E_INVALID and words in str(e.value), str(e.value)

    for device in (False, True):
        flipped = bytearray(raw)
        flipped[64 + 8 * 100 + 3] ^= 0x10  # a row offset
        expect(flipped, "checksum mismatch", device)
        flipped = bytearray(raw)
        flipped[-9] ^= 0x01  # a weight (the last 4 bytes may be padding)
        expect(flipped, "checksum mismatch", device)
        expect(raw[:-8], "truncated", device)
        expect(b"NOTACSR!" + raw[8:], "bad magic", device)
        hdr = bytearray(raw)
        hdr[16] ^= 0x01  # V, caught by the header check
        expect(hdr, "corrupt hytgraph CSR header", device)
        expect(raw[:40], "shorter than its header", device)
    with pytest.raises(hyt.HytError) as e:
        hyt.load_csr(tmp_path / "missing.csr")
    assert e.value.code == hyt.capi.HYT_E_IO
    bad = hyt.CSR(np.array([0, 2, 1], np.uint64), np.array([0, 1], np.uint32))
    with pytest.raises(hyt.HytError) as e:
        hyt.save_csr(bad, tmp_path / "never.csr")
    assert e.value.code == hyt.capi.HYT_E_INVALID and not (tmp_path / "never.csr").exists()


def test_binary_large_device_round_trip(hyt, gpu, tmp_path):
    """Scale 20 (16.5M edges, several pinned-ring pieces): save from the
    device, load to the device, identical arrays and a working graph."""
    d = hyt.rmat(20, 16, 9, device=True)
    p = tmp_path / "s20.csr"
    hyt.save_csr(d, p)
    st = {}
    r = hyt.load_csr(p, device=True, stats=st)
    a, b = d.download(), r.download()
    assert _same(a.row_offsets, b.row_offsets) and _same(a.column_indices, b.column_indices)
    assert _same(a.weights, b.weights)
    assert st["threads"] > 1
    src = int(hyt.pick_sources(a.row_offsets, 1, 1)[0])
    with hyt.Graph(d) as g1, hyt.Graph(r) as g2:
        assert np.array_equal(g1.sssp(src)[0], g2.sssp(src)[0])
    d.free()
    r.free()
