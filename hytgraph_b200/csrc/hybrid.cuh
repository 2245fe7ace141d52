// Partition-driven solvers for graphs whose edges live in pinned host memory.
//
// The solvers keep vertex data (offsets, degrees, ranks, labels, frontiers)
// in HBM and ask a *source* for the edges of each partition right before
// they are read.  The source (hybrid.cu) decides, per partition and per
// iteration, whether those edges are already resident, copied whole into a
// staging slot (ExpTM-Filter), gathered by host threads and shipped packed
// (ExpTM-Compaction), or read in place from mapped host memory by the kernel
// (ImpTM-Zero-Copy).  Every pointer a source hands back is indexed by GLOBAL
// edge id: a staging slot holding edges [e0, e1) is returned as slot - e0.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "graph.cuh"

namespace hyt {

// ---------------------------------------------------------------- pull ----
// A piece: a vertex range of one partition whose in-edges are contiguous;
// partitions larger than a staging slot are split into several pieces.
struct PullPart {
    uint64_t chunk_begin, chunk_end;  // long-row chunk tasks of the piece
    uint64_t tile_begin, tile_end;    // tiles of the piece
};

class PullSource {
public:
    virtual ~PullSource() = default;
    virtual size_t parts() const = 0;  // pieces, in vertex order
    virtual PullPart part(size_t p) const = 0;
    virtual void begin_iteration(cudaStream_t compute) = 0;
    // Makes partition p's source ids readable by work enqueued on `compute`
    // from now on; returns their global-edge-indexed base pointer.
    virtual const uint32_t *acquire(size_t p, cudaStream_t compute) = 0;
    // Work reading partition p has been enqueued on `compute`.
    virtual void release(size_t p, cudaStream_t compute) = 0;
};

// PageRank / personalized PageRank over a graph whose CSC sources come from
// `src` (g holds in_offsets, out_degree, tiles and long rows, not the
// sources).  Same semantics and stop rule as pagerank_run / ppr_run.
void pagerank_partitioned(GraphImpl &g, PullSource &src, bool personalized, uint32_t source, float damping,
                          float tolerance, uint32_t max_iter, cudaStream_t s, float *ranks_out, hyt_run_stats *stats);

// ---------------------------------------------------------------- push ----
// kLocDirect: edges at cols/weights (for the vertices of [vlo, vhi): a
// partition larger than a staging slot is staged piece by piece, one piece
// per wave); kLocCompacted: expanded from the packed payload; kLocSkip: not
// expanded in this wave (another wave covers it).
enum : uint32_t { kLocDirect = 0, kLocCompacted = 1, kLocSkip = 2 };

struct EdgeLoc {
    const uint32_t *cols;     // global-edge-indexed (device slot - e0, or host)
    const uint32_t *weights;  // same addressing
    uint32_t mode;            // kLocDirect, kLocCompacted or kLocSkip
    uint32_t vlo, vhi;        // kLocDirect: only vertices in [vlo, vhi) are expanded
    uint32_t pad;
};

// Frontier statistics of one partition in one round (HyTM metrics inputs).
struct PartMetrics {
    unsigned long long active_vertices, active_edges, zc_requests, zc_alignment;
};

// Packed rows of the compacted partitions' frontier vertices on the device:
// row i belongs to vertex verts[i] and owns edges [index[i], index[i+1]).
struct CompactPayload {
    const uint32_t *verts;
    const uint64_t *index;
    const uint32_t *cols;
    const uint32_t *weights;
    uint64_t rows;
};

// A round is expanded in waves: wave w's loc table marks the partitions
// whose edges that wave reaches (kLocDirect); the others are kLocSkip in
// it.  Compacted partitions are kLocCompacted in every wave.
struct RoundPlan {
    std::vector<std::vector<EdgeLoc>> waves;
    bool compacted = false;
};

class PushSource {
public:
    virtual ~PushSource() = default;
    virtual uint32_t part_shift() const = 0;
    virtual size_t parts() const = 0;
    // Decides each partition's engine for this round from its frontier
    // metrics and lays out the waves.
    virtual void plan_round(const std::vector<PartMetrics> &m, RoundPlan &plan) = 0;
    // Before / after the kernels of wave w are enqueued on `s`: the source
    // makes the wave's staged edges ready (and prefetches the next wave).
    virtual void enter_wave(size_t w, cudaStream_t s) = 0;
    virtual void leave_wave(size_t w, cudaStream_t s) = 0;
    // Gathers the rows of the listed frontier vertices (host array) and
    // ships them; the payload is valid for work enqueued on `s`.
    virtual CompactPayload compact(const uint32_t *verts, uint64_t n, cudaStream_t s) = 0;
    virtual void end_round(cudaStream_t s) = 0;
};

// SSSP over a graph whose CSR edges come from `src` (g holds row_offsets and
// the label/frontier workspaces).  Distances equal sssp_run's bit for bit.
void sssp_partitioned(GraphImpl &g, PushSource &src, uint32_t source, uint32_t max_rounds, cudaStream_t s,
                      uint32_t *dist_out, hyt_run_stats *stats);

// Work tiles / long rows of the pull side from g.in_offsets (graph.cu).
void build_pull_tiles(GraphImpl &g, cudaStream_t s);

}  // namespace hyt
