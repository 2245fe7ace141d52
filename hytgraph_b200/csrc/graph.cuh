// Device-resident graph behind the opaque hyt_graph handle.
//
// HBM layout (E < 2^32 edges per graph on this path):
//   push side (CSR, frontier SSSP):   row_offsets u64[V+1], cols u32[E],
//                                     weights u32[E] (u32 or f32 bits)
//   pull side (CSC, PageRank):        in_offsets u64[V+1], in_sources u32[E]
//   per vertex:                       out_degree u32[V]
//   PageRank work list:               tile_start u32[T+1] (short-row tiles),
//                                     long rows + their chunk tasks
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace hyt {

// PageRank pull work decomposition.  Rows are cut into tiles along the
// merge path (1 unit per row + 1 per in-edge): a tile spans tile_cost units,
// so its rows hold fewer than tile_cost edges except for its last row.  A
// last row with in-degree >= tile_cost is a "long row": it is excluded from
// the tile and split into kLongChunk-edge chunks.  One warp processes one
// task (tile or chunk), so a tile's staged contributions fit in a per-warp
// shared-memory slice of 2 * tile_cost floats.
constexpr uint32_t kTileCostDefault = 512;   // merge-path units per tile (tunable: HYT_PR_TILE)
constexpr uint32_t kTileCostMax = 512;       // register-path tiles; bulk-staged tasks need <= kStageTileMax
constexpr uint32_t kStageTileMax = 256;      // a tile's edges (< 2 * tile_cost) fit one staging slot
constexpr uint32_t kLongChunk = 4096;
constexpr uint32_t kHotSourcesDefault = 8192;   // shared-memory source cache (tunable: HYT_PR_HOT)
constexpr uint32_t kHotSourcesMax = 32768;
constexpr uint32_t kPRSmemMax = 226 * 1024;     // dynamic shared memory per CTA (227 KB opt-in - static)
constexpr uint32_t kHotTag = 0x80000000u;       // in_sources tag: source is hot slot (low bits)

// Pull task descriptors (pull_tasks[i], chunks first, then tiles: the task
// numbering of the pull kernels), 16 bytes each so a warp fetches its next
// task with one load:
//   x = first edge (low 32 bits)
//   y = first edge bits 32..39 | edge count << 8 (< 2^23) | 1 << 31 for a chunk
//   z, w = first row and end row of a tile (the end excludes a chunked long
//          last row); long-row index and chunk number of a chunk
__host__ __device__ __forceinline__ uint64_t task_first_edge(uint4 d) {
    return uint64_t(d.x) | (uint64_t(d.y & 0xFFu) << 32);
}
__host__ __device__ __forceinline__ uint32_t task_edges(uint4 d) { return (d.y >> 8) & 0x7FFFFFu; }
__host__ __device__ __forceinline__ bool task_is_chunk(uint4 d) { return (d.y >> 31) != 0; }

#ifndef HYT_PULL_PREFETCH
#define HYT_PULL_PREFETCH 1
#endif
#ifdef __CUDACC__
// Warms L2 with the edge arrays a0 (and a1 when not NULL) of pull task d:
// lane l touches the 128-byte lines at edges l*32, l*32 + 1024, ... of the
// task, so the next task's streaming loads find their lines in L2.
__device__ __forceinline__ void prefetch_task(uint4 d, const uint32_t *a0, const uint32_t *a1, int lane) {
    if constexpr (HYT_PULL_PREFETCH) {
        const uint64_t e0 = task_first_edge(d), n = task_edges(d);
        for (uint64_t x = uint64_t(lane) * 32; x < n; x += 32 * 32) {
            asm volatile("prefetch.global.L2 [%0];" ::"l"(a0 + e0 + x));
            if (a1) asm volatile("prefetch.global.L2 [%0];" ::"l"(a1 + e0 + x));
        }
    }
}
#endif

struct LongRow {
    uint32_t row;
    uint32_t first_chunk;  // index of its first partial-sum slot
    uint32_t num_chunks;
    uint32_t pad;
};

// An instantiated CUDA graph holding a solver's conditional while-loop,
// kept with the graph object and reused by later solves while the loop's
// shape (`key`: kernels, launch shapes, argument pointers) is unchanged.
// Its conditional handle is set to 1 at every launch.
struct LoopGraph {
    std::vector<unsigned char> key;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphConditionalHandle cond = 0;

    LoopGraph() = default;
    LoopGraph(const LoopGraph &) = delete;
    LoopGraph &operator=(const LoopGraph &) = delete;
    ~LoopGraph() { reset(); }
    void reset() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        key.clear();
    }
    bool matches(const void *k, size_t n) const {
        return exec && key.size() == n && std::memcmp(key.data(), k, n) == 0;
    }
    void set_key(const void *k, size_t n) {
        key.assign(static_cast<const unsigned char *>(k), static_cast<const unsigned char *>(k) + n);
    }
};

struct GraphImpl {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    uint64_t V = 0, E = 0;
    uint32_t weight_kind = HYT_WEIGHTS_NONE;
    uint32_t flags = 0;
    bool weights_ok = true;  // F32 weights all finite and >= 0
    uint32_t default_delta = 0;  // SSSP near/far bucket width (2x mean u32 weight)

    // push side
    GraphArray<uint64_t> row_offsets;
    GraphArray<uint32_t> cols;
    GraphArray<uint32_t> weights;
    GraphArray<uint32_t> out_degree;
    // HYT_GRAPH_HUB_ORDER: perm[new] = caller id, inv[caller id] = new
    // (empty otherwise)
    GraphArray<uint32_t> perm, inv;
    std::vector<uint32_t> h_inv;  // host copy of inv, filled by graph_vertex_map (engines mapping many sources)

    // pull side
    GraphArray<uint64_t> in_offsets;
    GraphArray<uint32_t> in_sources;
    GraphArray<uint32_t> in_weights;   // [E] weights in CSC order (PUSH|PULL weighted graphs; SSSP pull rounds)
    GraphArray<uint32_t> tile_start;   // [num_tiles + 1]
    GraphArray<LongRow> long_rows;     // [num_long]
    GraphArray<uint2> chunk_tasks;     // [num_chunks] = (long row index, chunk)
    GraphArray<uint4> pull_tasks;      // [num_chunks + num_tiles] descriptors (task_first_edge, ...)
    uint64_t num_tiles = 0, num_long = 0, num_chunks = 0;
    uint32_t tile_cost = kTileCostDefault;  // a row is long when its in-degree >= tile_cost
    // Hot sources: the num_hot vertices of largest out-degree.  Their
    // occurrences in in_sources carry kHotTag | slot, and each PageRank CTA
    // keeps their contributions in shared memory for the iteration.
    GraphArray<uint32_t> hot_vertex;   // [num_hot], by slot
    uint32_t num_hot = 0;
    uint64_t hot_edges = 0;             // in-edges whose source is hot

    // host-side facts
    uint64_t max_in_degree = 0, max_out_degree = 0, dangling = 0;
    double build_ms = 0.0;

    // Solver workspaces, grown on demand and reused across calls.
    GraphArray<float> rank[2];
    GraphArray<float> contrib[2];
    GraphArray<float> partial;        // long-row chunk partial sums (s, c)
    GraphArray<uint32_t> ticket;      // long-row arrival counters
    GraphArray<unsigned char> pr_state;
    uint32_t pr_state_iters = 0;

    GraphArray<uint32_t> dist;
    GraphArray<uint32_t> stamp;
    GraphArray<uint32_t> queue[2];
    GraphArray<uint32_t> far[2];
    GraphArray<uint2> hub_tasks;
    GraphArray<unsigned char> sssp_state;
    GraphArray<uint32_t> ppr_wide;         // packed PPR: rows of 32+ in-edges below the long-row threshold
    uint64_t ppr_wide_n = 0;
    bool ppr_wide_ready = false;
    uint32_t min_in_weight = 0;            // smallest CSC weight (bit pattern, sign of -0.0 cleared)
    bool min_in_weight_ready = false;
    GraphArray<uint32_t> ms_dist;          // multi-source labels [V][8]
    GraphArray<unsigned char> ms_state;
    PinnedArray<uint64_t> host_scratch;  // small pinned readback area
    LoopGraph sssp_loop;                 // instantiated SSSP round loop (reused while its shape holds)

    size_t device_bytes() const;
};

// PageRank CTA shape: kPRThreads threads; dynamic shared memory = hot cache
// + one staging slice (2 * tile_cost + 8 floats) per warp.
constexpr int kPRThreads = 1024;
inline size_t pr_shared_bytes(uint32_t num_hot, uint32_t tile_cost) {
    return (size_t(num_hot) + size_t(kPRThreads / 32) * (2 * size_t(tile_cost) + 8)) * sizeof(float);
}

// Builds the device graph from a CSR (host or device pointers).
void graph_build(GraphImpl &g, const hyt_csr &csr, uint32_t flags);

// Copies the CSC with hot tags removed into caller buffers (host or device).
void graph_copy_csc(const GraphImpl &g, uint64_t *in_offsets, uint32_t *in_sources);
// Builds the graph; with HYT_GRAPH_HUB_ORDER in flags, in hub order.
void graph_create(GraphImpl &g, const hyt_csr &csr, uint32_t flags);
// The internal id of a caller's vertex (identity without a hub order):
// from the host copy of the map when graph_vertex_map has made one, else
// one 4-byte read of the device map on stream s.
uint32_t graph_vertex(const GraphImpl &g, uint32_t v, cudaStream_t s);
// Makes the host copy of a hub-ordered graph's vertex map (once), for
// callers that map many sources; no-op without a hub order.
void graph_vertex_map(GraphImpl &g);
// Writes V 4-byte per-vertex values (internal order, device) to dst (host
// or device) in the caller's vertex order.
void graph_emit(const GraphImpl &g, void *dst, const void *src, cudaStream_t s);
// Fails with HYT_E_UNSUPPORTED for a hub-ordered graph.
void graph_require_caller_order(const GraphImpl &g, const char *what);

}  // namespace hyt

struct hyt_graph {
    hyt::GraphImpl impl;
};
