// Per-warp staging pipeline of the pull kernels (PageRank iterations and
// SSSP pull sweeps over an in-HBM CSC).  A warp walks its pull tasks
// (graph.cuh descriptors) as units -- a tile, or a kUnitEdges-edge piece of
// a long-row chunk -- and stages each unit's source ids into shared memory
// with one bulk copy (cp.async.bulk, completion on an mbarrier), one unit
// ahead of the unit it is working on.  Ids then cost no registers and no
// load latency on the warp's critical path; the warp's registers go to the
// dependent gathers instead.
//
// Sources are this GPU's own memory only (no multicast).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bulk.cuh"
#include "graph.cuh"

namespace hyt::stage {

constexpr uint32_t kUnitEdges = 512;  // edges of one staged unit (a tile, or a piece of a chunk)
constexpr uint32_t kSlotWords = 520;  // unit + 16-byte alignment at both ends, in 4-byte words
constexpr int kStageSlots = 2;        // staging slots per warp (double buffering)
// A tile's edges: the rows starting inside a tile span < tile_cost merge
// units, and its last short row adds < tile_cost more, so < 2 * tile_cost.
static_assert(2 * kTileCostMax - 1 + 6 <= kSlotWords, "a tile's edges must fit one staging slot");
static_assert(kLongChunk % kUnitEdges == 0, "chunks split into whole units");

// Dynamic shared memory of the staged kernels: per-warp mbarriers and slots,
// then the hot-source table.
constexpr size_t kStageHead = size_t(kPRThreads / 32) * kStageSlots * sizeof(uint64_t);
constexpr size_t kStageBytes = kStageHead + size_t(kPRThreads / 32) * kStageSlots * kSlotWords * 4;

inline size_t staged_shared_bytes(uint32_t num_hot) { return kStageBytes + size_t(num_hot) * 4; }

#ifdef __CUDACC__

// This warp's barriers and slots in the kernel's dynamic shared memory
// (kStageBytes from its start); lane 0 initialises the barriers.
struct WarpStage {
    uint64_t *bars;
    uint32_t *slots;
};
__device__ __forceinline__ WarpStage warp_stage(unsigned char *smem, int warp, int lane) {
    WarpStage w;
    w.bars = reinterpret_cast<uint64_t *>(smem) + warp * kStageSlots;
    w.slots = reinterpret_cast<uint32_t *>(smem + kStageHead) + size_t(warp) * kStageSlots * kSlotWords;
    if (lane == 0)
        for (int i = 0; i < kStageSlots; ++i) bulk::mbar_init(w.bars + i);
    bulk::fence_barrier_init();
    __syncwarp();
    return w;
}

// Edge range [lo, hi) of unit j of task d.
struct Unit {
    uint64_t lo, hi;
};
__device__ __forceinline__ Unit unit_of(uint4 d, uint32_t j) {
    const uint64_t e0 = task_first_edge(d), n = task_edges(d);
    const uint64_t lo = e0 + uint64_t(j) * kUnitEdges;
    return Unit{lo, (lo + kUnitEdges < e0 + n) ? lo + kUnitEdges : e0 + n};
}
__device__ __forceinline__ uint32_t units_of(uint4 d) {
    return task_is_chunk(d) ? (task_edges(d) + kUnitEdges - 1) / kUnitEdges : 1u;
}

// Lane 0 announces and issues the bulk copy of unit u's ids (16-byte
// aligned: the span rounded out to whole 4-id groups, which the 16 bytes of
// tail padding behind every id array keep in bounds) into `slot`.
__device__ __forceinline__ void stage_unit(const uint32_t *in_src, Unit u, uint32_t *slot, uint64_t *bar, uint64_t pol,
                                           int lane) {
    if (lane == 0) {
        const uint64_t a0 = u.lo & ~uint64_t(3), a1 = (u.hi + 3) & ~uint64_t(3);
        const uint32_t bytes = static_cast<uint32_t>(a1 - a0) * 4u;
        bulk::mbar_arrive_expect_tx(bar, bytes);
        if (bytes) bulk::copy_g2s(slot, in_src + a0, bytes, bar, pol);
    }
}

// Drives one warp through its tasks (first, first + stride, ... < total):
// stages unit after unit into the warp's slots, one copy ahead, and calls
// consume(d, task, j, units, slot words, first staged edge) for each unit
// once its ids have landed.  false: a wait ran out (the copy still in
// flight has been waited for, within the same budget).
template <class Consume>
__device__ __forceinline__ bool stage_pipeline(const uint4 *tasks, const uint32_t *in_src, uint64_t first,
                                               uint64_t stride, uint64_t total, uint32_t *slots, uint64_t *bars,
                                               int lane, Consume &&consume) {
    if (first >= total) return true;
    const uint64_t pol = bulk::policy_evict_first();
    uint4 d = tasks[first];
    uint64_t t = first, nt = first + stride;
    uint4 dn = nt < total ? tasks[nt] : make_uint4(0, 0, 0, 0);
    uint32_t j = 0, phase = 0;
    int s = 0;
    stage_unit(in_src, unit_of(d, 0), slots, bars, pol, lane);
    for (;;) {
        const uint32_t nu = units_of(d);
        bool more = true;
        uint4 d2 = d;
        uint64_t t2 = t;
        uint32_t j2 = j + 1;
        if (j2 >= nu) {
            more = nt < total;
            d2 = dn;
            t2 = nt;
            j2 = 0;
            if (more) {
                nt += stride;
                dn = nt < total ? tasks[nt] : make_uint4(0, 0, 0, 0);
            }
        }
        if (more) stage_unit(in_src, unit_of(d2, j2), slots + (s ^ 1) * kSlotWords, bars + (s ^ 1), pol, lane);
        if (!bulk::mbar_wait(bars + s, (phase >> s) & 1u)) {
            if (more) bulk::mbar_wait(bars + (s ^ 1), (phase >> (s ^ 1)) & 1u);
            return false;
        }
        phase ^= 1u << s;
        const Unit u = unit_of(d, j);
        consume(d, t, j, nu, slots + s * kSlotWords, u.lo & ~uint64_t(3));
        bulk::fence_proxy_async_smem();  // this slot's generic accesses before its next bulk copy
        __syncwarp();
        if (!more) return true;
        d = d2;
        t = t2;
        j = j2;
        s ^= 1;
    }
}

#endif  // __CUDACC__

}  // namespace hyt::stage
