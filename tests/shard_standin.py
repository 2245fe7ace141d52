"""CPU stand-in for hytgraph_b200.shard.CudaShardKernels (test
infrastructure): the same vector contract on CPU torch tensors, computed
with numpy, so the sharded exchange (bounds, broadcasts, reductions, stop
rules) runs on gloo processes without a GPU.  Results are checked against
the oracle, never shipped."""
from __future__ import annotations

import numpy as np
import torch

PULL, PUSH = 1, 2
BIAS = np.uint32(0x80000000)
INF = np.uint32(0xFFFFFFFF)


class NumpyShardKernels:
    def __init__(self, off, cols, weights, part: int, parts: int):
        self.off = np.asarray(off, np.uint64)
        self.cols = np.asarray(cols, np.uint32)
        self.w = None if weights is None else np.asarray(weights, np.uint32)
        self.part, self.parts = part, parts
        V = self.off.shape[0] - 1
        self.num_vertices = V
        src = np.repeat(np.arange(V, dtype=np.uint32), np.diff(self.off).astype(np.int64))
        order = np.argsort(self.cols, kind="stable")
        self.in_src = src[order]
        self.in_w = None if self.w is None else self.w[order]
        self.in_dst = self.cols[order]
        self.in_off = np.concatenate([[0], np.cumsum(np.bincount(self.cols, minlength=V))]).astype(np.uint64)
        self.out_deg = np.diff(self.off).astype(np.uint32)
        self.prev = None

    def bounds(self, kind: int) -> list:
        V = self.num_vertices
        off = self.in_off if kind == PULL else self.off
        cost = off.astype(np.int64) + np.arange(V + 1)
        total = int(cost[-1])
        b = [0]
        for p in range(1, self.parts):
            target = (total * p + self.parts - 1) // self.parts
            b.append(max(int(np.searchsorted(cost, target, "left")), b[-1]))
        b.append(V)
        return b

    def empty(self, n: int, dtype):
        return torch.empty(n, dtype=dtype)

    def _range(self, kind):
        b = self.bounds(kind)
        return b[self.part], b[self.part + 1]

    def pagerank_init(self, v) -> None:
        V = self.num_vertices
        r0 = np.zeros(V, np.float32)
        if v.personalized:
            r0[v.source] = 1.0
        else:
            r0[:] = np.float32(1.0) / np.float32(V)
        od = self.out_deg
        c0 = np.where(od > 0, r0 / np.maximum(od, 1).astype(np.float32), np.float32(0)).astype(np.float32)
        v.rank[0].copy_(torch.from_numpy(r0))
        v.contrib[0].copy_(torch.from_numpy(c0))
        lo, hi = self._range(PULL)
        dang = float(r0[lo:hi][od[lo:hi] == 0].astype(np.float64).sum())
        v.sums.copy_(torch.tensor([0.0, dang], dtype=torch.float64))

    def pagerank_step(self, v, iteration: int, dangling: float) -> None:
        V = self.num_vertices
        d = np.float32(v.damping)
        cur = v.rank[iteration & 1].numpy()
        ccur = v.contrib[iteration & 1].numpy()
        nxt = v.rank[(iteration + 1) & 1].numpy()
        cnxt = v.contrib[(iteration + 1) & 1].numpy()
        lo, hi = self._range(PULL)
        res = dang = 0.0
        if hi > lo:
            e0, e1 = int(self.in_off[lo]), int(self.in_off[hi])
            vals = ccur[self.in_src[e0:e1]].astype(np.float64)
            csum = np.concatenate([[0.0], np.cumsum(vals)])
            rel = (self.in_off[lo:hi + 1] - np.uint64(e0)).astype(np.int64)
            sums = (csum[rel[1:]] - csum[rel[:-1]]).astype(np.float32)
            if v.personalized:
                nx = (d * sums).astype(np.float32)
                tele = np.float32((1.0 - float(d)) + float(d) * dangling)
                if lo <= v.source < hi:
                    nx[v.source - lo] = np.float32(tele + nx[v.source - lo])
            else:
                base = (np.float32(1.0) - d) / np.float32(V)
                dshare = np.float32(base + np.float32(float(d) * dangling / V))
                nx = (dshare + d * sums).astype(np.float32)
            od = self.out_deg[lo:hi]
            res = float(np.abs(nx.astype(np.float64) - cur[lo:hi].astype(np.float64)).sum())
            dang = float(nx[od == 0].astype(np.float64).sum())
            nxt[lo:hi] = nx
            cnxt[lo:hi] = np.where(od > 0, nx / np.maximum(od, 1).astype(np.float32), np.float32(0))
        v.sums.copy_(torch.tensor([res, dang], dtype=torch.float64))

    def emit(self, values, out=None) -> np.ndarray:
        if out is None:
            return values.numpy().copy()
        out[:] = values.numpy()
        return out

    def sssp_init(self, keys, source: int) -> None:
        V = self.num_vertices
        k = np.full(V + 1, INF ^ BIAS, np.uint32)
        k[source] = np.uint32(0) ^ BIAS
        k[V] = 0
        keys.copy_(torch.from_numpy(k.view(np.int32)))
        lo, hi = self._range(PUSH)
        self.prev = np.full(hi - lo, INF, np.uint32)

    def sssp_collect(self, keys, frontier) -> None:
        V = self.num_vertices
        lo, hi = self._range(PUSH)
        lab = keys.numpy().view(np.uint32)[:V] ^ BIAS
        own = lab[lo:hi].copy()
        act = np.nonzero(own < self.prev)[0]
        self.prev[act] = own[act]
        self._active = (lo + act, own[act])
        fe = int(self.out_deg[lo + act].astype(np.int64).sum())
        frontier.copy_(torch.tensor([fe], dtype=torch.int64))

    def sssp_relax(self, keys, frontier) -> None:
        V, E = self.num_vertices, int(self.cols.shape[0])
        k = keys.numpy().view(np.uint32)  # shares the tensor's memory
        lab = k[:V] ^ BIAS
        verts, labels = self._active
        if int(frontier[0]) * 4 > E:  # pull sweep over this shard's rows of the PULL bounds
            plo, phi = self._range(PULL)
            e0, e1 = int(self.in_off[plo]), int(self.in_off[phi])
            src = self.in_src[e0:e1]
            w = np.ones(e1 - e0, np.uint64) if self.in_w is None else self.in_w[e0:e1].astype(np.uint64)
            du = lab[src].astype(np.uint64)
            cand = np.where(du == INF, np.uint64(INF), np.minimum(du + w, np.uint64(0xFFFFFFFE))).astype(np.uint32)
            np.minimum.at(lab, self.in_dst[e0:e1], cand)
        else:
            for v, d in zip(verts, labels):
                e0, e1 = int(self.off[v]), int(self.off[v + 1])
                w = np.ones(e1 - e0, np.uint64) if self.w is None else self.w[e0:e1].astype(np.uint64)
                nd = np.minimum(np.uint64(d) + w, np.uint64(0xFFFFFFFE)).astype(np.uint32)
                np.minimum.at(lab, self.cols[e0:e1], nd)
        k[:V] = lab ^ BIAS
        k[V] = 0 if verts.size else 1

    def sssp_labels(self, keys, out=None) -> np.ndarray:
        lab = keys.numpy().view(np.uint32)[: self.num_vertices] ^ BIAS
        if out is None:
            return lab
        out[:] = lab
        return out
