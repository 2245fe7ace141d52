"""Regenerates the golden fixtures in this folder from the REFERENCE's own
compiled CPU code (oracle/_ref/libhytref.so, built by
`make -C oracle REF=<reference checkout>` from the reference sources).

    python tests/golden/make_golden.py

Fixtures:
  rmat_reference.npz -- for several seeded R-MAT graphs (scales 8-12): a
      SHA-256 of the generated CSR bytes, the reference's pagerank_cpu ranks
      (float32 bits) / iterations / residual, and sssp_cpu distances (float32
      bits) / iterations from seeded sources.
  known_answers.json -- the reference's hand-written known-answer cases
      (tests/algorithm_tests.cpp:22-157, tests/cuda_algorithm_tests.cu:23-87,
      tests/unit_tests.cpp:2058-2204, 2268-2466) evaluated by the reference,
      the hub-sort and reorder cases (unit_tests.cpp:2468-2740), and per
      R-MAT graph the reference HubSorter's order / scores digests and hub
      count at hub_fraction 0.08 plus the digest of the CSR reordered by it.
"""
from __future__ import annotations

import hashlib
import json
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import hytgraph_b200 as hyt  # noqa: E402  (host-side generator only)
from oracle.bindings import Reference  # noqa: E402

OUT = Path(__file__).resolve().parent

# (scale, edge_factor, seed, weighted)
GRAPHS = [(8, 16, 1, True), (9, 8, 2, True), (10, 16, 3, True), (11, 4, 4, False), (12, 16, 5, True)]
N_SOURCES = 3


def csr_digest(g) -> str:
    h = hashlib.sha256()
    h.update(g.row_offsets.astype("<u8").tobytes())
    h.update(g.column_indices.astype("<u4").tobytes())
    if g.weights is not None:
        h.update(g.weights.astype("<u4").tobytes())
    return h.hexdigest()


def main() -> None:
    ref = Reference()
    arrays = {}
    meta = []
    for scale, ef, seed, weighted in GRAPHS:
        g = hyt.rmat(scale, ef, seed, *( (1, 63) if weighted else (0, 0) ))
        key = f"s{scale}_ef{ef}_seed{seed}"
        ranks, it, res, conv = ref.pagerank_cpu(g.row_offsets, g.column_indices)
        arrays[f"{key}_pr_bits"] = ranks.view(np.uint32)
        srcs = hyt.pick_sources(g.row_offsets, seed + 100, N_SOURCES)
        w = g.weights.astype(np.float32) if g.weights is not None else None
        dists, rounds = [], []
        for s in srcs:
            d, r, c = ref.sssp_cpu(g.row_offsets, g.column_indices, w, int(s))
            assert c
            dists.append(d.view(np.uint32))
            rounds.append(r)
        arrays[f"{key}_sssp_bits"] = np.stack(dists)
        order, scores, hubs = ref.hub_sort(g.row_offsets, g.column_indices, 0.08)
        # u32 weights travel through the reference's float array bit for bit
        r_off, r_cols, r_w = ref.reorder(g.row_offsets, g.column_indices,
                                         None if g.weights is None else g.weights.view(np.float32), order)
        reordered = hyt.CSR(r_off, r_cols, None if r_w is None else r_w.view(np.uint32))
        meta.append({"key": key, "scale": scale, "edge_factor": ef, "seed": seed, "weighted": weighted,
                     "num_vertices": g.num_vertices, "num_edges": g.num_edges, "csr_sha256": csr_digest(g),
                     "pr_iterations": it, "pr_residual": float(res), "pr_converged": conv,
                     "sources": [int(s) for s in srcs], "source_seed": seed + 100, "sssp_rounds": rounds,
                     "hub_fraction": 0.08, "hub_count": int(hubs),
                     "hub_order_sha256": hashlib.sha256(order.astype("<u4").tobytes()).hexdigest(),
                     "hub_scores_sha256": hashlib.sha256(scores.astype("<f8").tobytes()).hexdigest(),
                     "reordered_sha256": csr_digest(reordered)})
    np.savez_compressed(OUT / "rmat_reference.npz", **arrays)

    # Hand-written graphs from the reference's tests, evaluated by the reference.
    hand = []
    cases = [
        ("pr_cycle3", [0, 1, 2, 3], [1, 2, 0], None, None),
        ("pr_dangling", [0, 1, 2, 2], [1, 0], None, None),
        ("pr_cuda3", [0, 2, 3, 4], [1, 2, 2, 0], None, None),
        ("sssp_weighted4", [0, 2, 4, 5, 5], [1, 2, 2, 3, 3], [1.0, 4.0, 2.0, 6.0, 1.0], 0),
        ("sssp_unweighted4", [0, 1, 2, 2, 2], [1, 2], None, 0),
    ]
    for name, off, cols, w, src in cases:
        off_a = np.array(off, np.uint64)
        cols_a = np.array(cols, np.uint32)
        entry = {"name": name, "row_offsets": off, "column_indices": cols, "weights": w}
        if src is None:
            r, it, res, conv = ref.pagerank_cpu(off_a, cols_a, 0.85, 1e-6, 200)
            entry.update(ranks=[float(x) for x in r], iterations=it, converged=conv)
        else:
            d, it, conv = ref.sssp_cpu(off_a, cols_a, None if w is None else np.array(w, np.float32), src)
            entry.update(source=src, distances=[None if not np.isfinite(x) else float(x) for x in d],
                         iterations=it, converged=conv)
        hand.append(entry)
    # HyTM cost model known answer (unit_tests.cpp:2058-2158) and selector
    # boundaries (unit_tests.cpp:2159-2204), evaluated by the reference.
    off = np.array([0, 2, 3, 4, 4], np.uint64)
    cols = np.array([1, 2, 2, 0], np.uint32)
    act = np.array([1, 1, 0, 0], np.uint8)
    metrics, costs, eng = ref.hytm_evaluate(off, cols, act, np.array([[0, 2]], np.uint32),
                                            [0.8, 0.4, 0.625, 2.0, 14.0], [128, 256])
    hytm = {"row_offsets": off.tolist(), "column_indices": cols.tolist(), "active": act.tolist(),
            "partition": [0, 2], "options": {"alpha": 0.8, "beta": 0.4, "gamma": 0.625, "rtt": 2.0,
                                             "cpu_throughput": 14.0, "m": 128, "mr": 256},
            "metrics": metrics[0].tolist(), "costs": costs[0].tolist(), "engine": int(eng[0])}
    selector = []
    for f, c, z in [(10.0, 7.0, 20.0), (10.0, 8.0, 20.0), (10.0, 20.0, 10.0), (20.0, 8.0, 20.0)]:
        selector.append({"f": f, "c": c, "z": z, "engine": ref.select_engine(f, c, z, 0.8, 0.4)})
    combiner = []
    for engines, k in [([0, 0, 0, 0, 0, 0], 4), ([0, 1, 0, 0, 2, 0], 4), ([1, 2, 1, 2], 4), ([], 4),
                       ([0, 0, 1, 0, 0, 0, 0, 0, 2, 2, 0], 2)]:
        top, teng, tfirst, m = ref.task_combine(engines, k)
        combiner.append({"engines": engines, "k": k, "task_of_partition": top.tolist(),
                         "task_engine": teng.tolist(), "task_first": tfirst.tolist(), "metrics": m.tolist()})
    # Hub sorting (unit_tests.cpp:2468-2602, 2709-2740) and reordering
    # (unit_tests.cpp:2604-2707), evaluated by the reference.
    hub = []
    for name, off, cols, frac in [("scores3", [0, 2, 3, 4], [1, 2, 2, 0], 2.0 / 3.0),
                                  ("hubs_first5", [0, 3, 4, 5, 6, 7], [1, 2, 3, 0, 0, 0, 0], 0.4),
                                  ("permutation6", [0, 2, 3, 4, 5, 6, 6], [1, 2, 2, 3, 0, 0], 0.08),
                                  ("edgeless4", [0, 0, 0, 0, 0], [], 0.08)]:
        o, sc, n = ref.hub_sort(np.array(off, np.uint64), np.array(cols, np.uint32), frac)
        hub.append({"name": name, "row_offsets": off, "column_indices": cols, "hub_fraction": frac,
                    "vertex_order": o.tolist(), "scores": sc.tolist(), "hub_count": int(n)})
    reorder = []
    for name, off, cols, w, order in [("reorder3", [0, 2, 3, 4], [1, 2, 2, 0], None, [2, 0, 1]),
                                      ("reorder3_weights", [0, 2, 3, 4], [1, 2, 2, 0], [1.0, 2.0, 3.0, 4.0],
                                       [2, 0, 1]),
                                      ("hub_reorder5", [0, 3, 4, 5, 6, 7], [1, 2, 3, 0, 0, 0, 0], None,
                                       [0, 1, 2, 3, 4])]:
        ro, rc, rw = ref.reorder(np.array(off, np.uint64), np.array(cols, np.uint32),
                                 None if w is None else np.array(w, np.float32), np.array(order, np.uint32))
        reorder.append({"name": name, "row_offsets": off, "column_indices": cols, "weights": w,
                        "vertex_order": order, "new_row_offsets": ro.tolist(), "new_column_indices": rc.tolist(),
                        "new_weights": None if rw is None else rw.tolist()})
    with open(OUT / "known_answers.json", "w") as f:
        json.dump({"graphs": meta, "hand": hand, "hytm": hytm, "selector": selector, "combiner": combiner,
                   "hub_sort": hub, "reorder": reorder}, f, indent=1)
    print("wrote", OUT / "rmat_reference.npz", OUT / "known_answers.json")


if __name__ == "__main__":
    main()
