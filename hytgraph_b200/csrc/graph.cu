// Device graph construction: upload + validation, out-degrees, the CSC
// transpose and the PageRank pull work tiles.  Runs once per graph.
//
// The reference builds its incoming CSR on the host, single-threaded, on
// every pagerank_gpu / sssp_gpu call (cuda/pagerank.cu:33-74,
// cuda/sssp.cu:34-79).  Here the transpose is a stable radix sort on the
// GPU, so sources stay ascending inside every in-row exactly as the
// reference's counting pass leaves them.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.cuh"
#include "graph.cuh"
#include "prims.cuh"
#include "scratch.cuh"
#include "solvers.cuh"
#include "stage.cuh"

namespace hyt {
namespace {

enum : uint32_t { kBadOffsets = 1u, kBadColumn = 2u, kBadWeight = 4u, kBadTerminal = 8u };

__global__ void validate_offsets_kernel(const uint64_t *off, uint64_t V, uint64_t E, uint32_t *err) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) {
        if (off[v + 1] < off[v]) atomicOr(err, kBadOffsets);
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (off[0] != 0) atomicOr(err, kBadOffsets);
        if (off[V] != E) atomicOr(err, kBadTerminal);
    }
}

__global__ void validate_edges_kernel(const uint32_t *cols, const uint32_t *w, uint32_t wkind, uint64_t V,
                                      uint64_t E, uint32_t *err, unsigned long long *weight_sum) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    uint32_t bad = 0;
    unsigned long long wsum = 0;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < E; e += stride) {
        if (cols[e] >= V) bad |= kBadColumn;
        if (wkind == HYT_WEIGHTS_F32) {
            const float x = __uint_as_float(w[e]);
            if (!(x >= 0.0f) || isinf(x)) bad |= kBadWeight;  // NaN fails x >= 0
        } else if (wkind == HYT_WEIGHTS_U32) {
            wsum += w[e];
        }
    }
    if (bad) atomicOr(err, bad);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) wsum += __shfl_xor_sync(0xffffffffu, wsum, o);
    if ((threadIdx.x & 31) == 0 && wsum) atomicAdd(weight_sum, wsum);
}

__global__ void out_degree_kernel(const uint64_t *off, uint64_t V, uint32_t *deg, unsigned long long *dangling) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    uint32_t nd = 0;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) {
        const uint32_t d = static_cast<uint32_t>(off[v + 1] - off[v]);
        deg[v] = d;
        nd += (d == 0);
    }
    if (nd) atomicAdd(dangling, (unsigned long long)nd);
}

// Writes the source vertex of every CSR edge.  A CTA owns 256 consecutive
// rows; their edges are spread over all threads via an in-CTA prefix of the
// degrees, so rows of any length are load-balanced inside the CTA.
// Source row of every edge, in two balanced passes (no block walks a hub
// row alone): each non-empty row writes its id at its first edge, then an
// inclusive max-scan over the edges carries it to the rest of the row
// (row ids are non-decreasing along the edge array).
__global__ void mark_row_starts_kernel(const uint64_t *off, uint64_t V, uint32_t *src) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) {
        const uint64_t b = off[v];
        if (off[v + 1] > b) src[b] = static_cast<uint32_t>(v);
    }
}

void expand_sources(const uint64_t *off, uint64_t V, uint64_t E, uint32_t *src, cudaStream_t s) {
    if (E == 0) return;
    Scratch<uint32_t> marks(E, s);
    HYT_CUDA(cudaMemsetAsync(marks.get(), 0, E * sizeof(uint32_t), s));
    mark_row_starts_kernel<<<grid_for(V, 256), 256, 0, s>>>(off, V, marks.get());
    HYT_CUDA(cudaGetLastError());
    prims::inclusive_max_scan_u32(marks.get(), src, E, s);
}  // marks is freed in stream order, after the scan

// Row offsets of a sorted key array: off[v] = first position with key >= v.
__global__ void offsets_from_sorted_kernel(const uint32_t *keys, uint64_t E, uint64_t V, uint64_t *off) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e <= E; e += stride) {
        const int64_t prev = (e == 0) ? -1 : static_cast<int64_t>(keys[e - 1]);
        const int64_t cur = (e == E) ? static_cast<int64_t>(V) : static_cast<int64_t>(keys[e]);
        for (int64_t v = prev + 1; v <= cur; ++v) off[v] = e;
    }
}

// tile_start[k] = first row whose merge-path coordinate (row + in_offset)
// reaches k * tile.
__global__ void tile_bounds_kernel(const uint64_t *in_off, uint64_t V, uint64_t E, uint64_t num_tiles, uint32_t tile,
                                   uint32_t *tile_start) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v <= V; v += stride) {
        const int64_t p_prev = (v == 0) ? -1 : static_cast<int64_t>((v - 1) + in_off[v - 1]);
        const int64_t p_cur = static_cast<int64_t>(v + in_off[v]);
        int64_t k_lo = (p_prev < 0) ? 0 : p_prev / tile + 1;
        int64_t k_hi = (v == V) ? static_cast<int64_t>(num_tiles) : p_cur / tile;
        for (int64_t k = k_lo; k <= k_hi; ++k) tile_start[k] = static_cast<uint32_t>(v);
    }
}

__global__ void in_degree_kernel(const uint64_t *in_off, uint64_t V, uint32_t long_degree, uint32_t *deg,
                                 uint8_t *is_long) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) {
        const uint32_t d = static_cast<uint32_t>(in_off[v + 1] - in_off[v]);
        deg[v] = d;
        is_long[v] = d >= long_degree;
    }
}

__global__ void iota_kernel(uint32_t *out, uint64_t n) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) out[i] = static_cast<uint32_t>(i);
}

__global__ void hot_slot_kernel(const uint32_t *hot, uint32_t n, uint32_t *slot) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) slot[hot[i]] = i;
}

// Replaces hot sources in the CSC by kHotTag | slot; counts them.
__global__ void tag_hot_kernel(uint32_t *in_src, uint64_t E, const uint32_t *slot, unsigned long long *count) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    unsigned long long c = 0;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < E; e += stride) {
        const uint32_t s = slot[in_src[e]];
        if (s != 0xFFFFFFFFu) {
            in_src[e] = kHotTag | s;
            ++c;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

__global__ void gather_u32_kernel(const uint32_t *src, const uint32_t *idx, uint64_t n, uint32_t *out) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) out[i] = src[idx[i]];
}

int bits_for(uint64_t max_value) {
    int b = 1;
    while (b < 64 && (max_value >> b) != 0) ++b;
    return b;
}

__global__ void untag_sources_kernel(const uint32_t *in_src, uint64_t n, const uint32_t *hot_vertex, uint32_t *out) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) {
        const uint32_t u = in_src[i];
        out[i] = (u & kHotTag) ? hot_vertex[u & ~kHotTag] : u;
    }
}

}  // namespace

namespace {

__global__ void invert_kernel(const uint32_t *__restrict__ perm, uint64_t V, uint32_t *__restrict__ inv) {
    for (uint64_t n = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; n < V; n += uint64_t(gridDim.x) * blockDim.x)
        inv[perm[n]] = static_cast<uint32_t>(n);
}

// out[i] = hi[i] << 32 | lo[i].
__global__ void pack_pairs_kernel(const uint32_t *__restrict__ hi, const uint32_t *__restrict__ lo, uint64_t n,
                                  uint64_t *__restrict__ out) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        out[i] = (uint64_t(hi[i]) << 32) | lo[i];
}

// hi[i] = in[i] >> 32, lo[i] = in[i] & 0xFFFFFFFF.
__global__ void unpack_pairs_kernel(const uint64_t *__restrict__ in, uint64_t n, uint32_t *__restrict__ hi,
                                    uint32_t *__restrict__ lo) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t v = in[i];
        hi[i] = static_cast<uint32_t>(v >> 32);
        lo[i] = static_cast<uint32_t>(v);
    }
}

// dst[v] = src[inv[v]]: values back in the caller's vertex order.
__global__ void emit_kernel(const uint32_t *__restrict__ src, const uint32_t *__restrict__ inv, uint64_t V,
                            uint32_t *__restrict__ dst) {
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += uint64_t(gridDim.x) * blockDim.x)
        dst[v] = src[inv[v]];
}

}  // namespace

void graph_create(GraphImpl &g, const hyt_csr &csr, uint32_t flags) {
    if (!(flags & HYT_GRAPH_HUB_ORDER)) {
        graph_build(g, csr, flags);
        return;
    }
    const uint64_t V = csr.num_vertices;
    if (V == 0) fail(HYT_E_INVALID, "graph requires at least one vertex");
    if (V > 0xFFFFFFFFull) fail(HYT_E_INVALID, "vertex ids are uint32: num_vertices must be < 2^32");
    // the reference's HubSorter with every vertex ranked, then the CSR
    // renumbered (both on the GPU, from one device copy of a host CSR)
    const uint64_t E = csr.num_edges;
    const bool weighted = csr.weight_kind != HYT_WEIGHTS_NONE && E;
    GraphArray<uint64_t> d_off;
    GraphArray<uint32_t> d_cols, d_w;
    hyt_csr dev = csr;
    if (csr.row_offsets && !is_device_pointer(csr.row_offsets)) {
        d_off.allocate(V + 1);
        copy_to_device(d_off.get(), csr.row_offsets, (V + 1) * 8, g.stream);
        dev.row_offsets = d_off.get();
    }
    if (E && csr.column_indices && !is_device_pointer(csr.column_indices)) {
        d_cols.allocate(E);
        copy_to_device(d_cols.get(), csr.column_indices, E * 4, g.stream);
        dev.column_indices = d_cols.get();
    }
    // the weights are first needed by the reorder: their upload runs on the
    // graph's stream while the hub sort (its own stream) ranks the vertices
    if (weighted && csr.weights && !is_device_pointer(csr.weights)) {
        d_w.allocate(E);
        HYT_CUDA(cudaMemcpyAsync(d_w.get(), csr.weights, E * 4, cudaMemcpyHostToDevice, g.stream));
        dev.weights = d_w.get();
    }
    GraphArray<uint32_t> perm(V);
    try {
        hub_sort(dev, 1.0, perm.get(), nullptr, nullptr, nullptr);
    } catch (...) {
        cudaStreamSynchronize(g.stream);  // the weights copy lands before its buffer is freed
        throw;
    }
    HYT_CUDA(cudaStreamSynchronize(g.stream));
    hyt_csr_buffers b{};
    csr_reorder(dev, perm.get(), true, &b, nullptr, true);
    d_off.release();
    d_cols.release();
    d_w.release();
    struct Free {
        hyt_csr_buffers *b;
        ~Free() { free_pooled_buffers(b); }
    } release{&b};
    hyt_csr r = csr;
    r.row_offsets = b.row_offsets;
    r.column_indices = b.column_indices;
    r.weights = b.weights;
    graph_build(g, r, flags & ~uint32_t(HYT_GRAPH_HUB_ORDER));
    g.inv.allocate(V);
    invert_kernel<<<grid_for(V, 256), 256, 0, g.stream>>>(perm.get(), V, g.inv.get());
    HYT_CUDA(cudaGetLastError());
    HYT_CUDA(cudaStreamSynchronize(g.stream));
    g.perm = std::move(perm);
}

uint32_t graph_vertex(const GraphImpl &g, uint32_t v, cudaStream_t s) {
    if (!g.inv.get()) return v;
    if (!g.h_inv.empty()) return g.h_inv[v];
    // one entry of the device map: a single-source solve pays one small
    // read instead of a copy of the whole map at graph creation
    uint32_t local = 0;
    uint32_t *h = g.host_scratch.ptr ? reinterpret_cast<uint32_t *>(g.host_scratch.ptr) : &local;
    HYT_CUDA(cudaMemcpyAsync(h, g.inv.get() + v, sizeof(uint32_t), cudaMemcpyDeviceToHost, s ? s : g.stream));
    HYT_CUDA(cudaStreamSynchronize(s ? s : g.stream));
    return *h;
}

void graph_vertex_map(GraphImpl &g) {
    if (!g.inv.get() || !g.h_inv.empty()) return;
    HYT_CUDA(cudaSetDevice(g.device));
    std::vector<uint32_t> m(g.V);
    HYT_CUDA(cudaMemcpyAsync(m.data(), g.inv.get(), g.V * 4, cudaMemcpyDeviceToHost, g.stream));
    HYT_CUDA(cudaStreamSynchronize(g.stream));
    g.h_inv = std::move(m);
}

void graph_emit(const GraphImpl &g, void *dst, const void *src, cudaStream_t s) {
    const uint64_t V = g.V;
    if (!g.inv.get()) {
        copy_from_device(dst, src, V * 4, s);
        return;
    }
    if (is_device_pointer(dst)) {
        emit_kernel<<<grid_for(V, 256), 256, 0, s>>>(static_cast<const uint32_t *>(src), g.inv.get(), V,
                                                     static_cast<uint32_t *>(dst));
        HYT_CUDA(cudaGetLastError());
        return;
    }
    Scratch<uint32_t> tmp(V, s);
    emit_kernel<<<grid_for(V, 256), 256, 0, s>>>(static_cast<const uint32_t *>(src), g.inv.get(), V, tmp.get());
    HYT_CUDA(cudaGetLastError());
    copy_from_device(dst, tmp.get(), V * 4, s);
    HYT_CUDA(cudaStreamSynchronize(s));
}

void graph_require_caller_order(const GraphImpl &g, const char *what) {
    if (g.perm.get()) fail(HYT_E_UNSUPPORTED, std::string(what) + " does not take graphs built with HYT_GRAPH_HUB_ORDER");
}

void graph_copy_csc(const GraphImpl &g, uint64_t *in_offsets, uint32_t *in_sources) {
    graph_require_caller_order(g, "hyt_graph_copy_csc");
    if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PULL");
    cudaStream_t s = g.stream;
    HYT_CUDA(cudaMemcpyAsync(in_offsets, g.in_offsets.get(), (g.V + 1) * 8, cudaMemcpyDefault, s));
    if (g.num_hot == 0) {
        HYT_CUDA(cudaMemcpyAsync(in_sources, g.in_sources.get(), g.E * 4, cudaMemcpyDefault, s));
    } else {
        const uint64_t chunk = std::min<uint64_t>(g.E, uint64_t(1) << 26);
        DeviceArray<uint32_t> tmp(std::max<uint64_t>(chunk, 1));
        for (uint64_t e0 = 0; e0 < g.E; e0 += chunk) {
            const uint64_t n = std::min(chunk, g.E - e0);
            untag_sources_kernel<<<grid_for(n, 256), 256, 0, s>>>(g.in_sources.get() + e0, n, g.hot_vertex.get(),
                                                                  tmp.get());
            HYT_CUDA(cudaGetLastError());
            HYT_CUDA(cudaMemcpyAsync(in_sources + e0, tmp.get(), n * 4, cudaMemcpyDefault, s));
            HYT_CUDA(cudaStreamSynchronize(s));  // tmp is reused by the next chunk
        }
    }
    HYT_CUDA(cudaStreamSynchronize(s));
}

size_t GraphImpl::device_bytes() const {
    size_t b = row_offsets.bytes() + cols.bytes() + weights.bytes() + out_degree.bytes() + in_offsets.bytes() +
               in_sources.bytes() + in_weights.bytes() + tile_start.bytes() + long_rows.bytes() + chunk_tasks.bytes() +
         pull_tasks.bytes();
    for (int i = 0; i < 2; ++i) b += rank[i].bytes() + contrib[i].bytes() + queue[i].bytes() + far[i].bytes();
    b += partial.bytes() + ticket.bytes() + pr_state.bytes() + dist.bytes() + stamp.bytes() + hub_tasks.bytes() +
         sssp_state.bytes() + ms_dist.bytes() + ms_state.bytes() + ppr_wide.bytes();
    return b;
}

// Descriptor of pull task i (graph.cuh): chunks [0, num_chunks), then tiles.
__global__ void pull_task_kernel(const uint64_t *in_off, const uint32_t *tile_start, const LongRow *long_rows,
                                 const uint2 *chunk_tasks, uint64_t num_chunks, uint64_t num_tiles, uint32_t tile_cost,
                                 uint4 *out) {
    const uint64_t n = num_chunks + num_tiles, stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) {
        uint64_t e0 = 0, len = 0;
        uint32_t a = 0, b = 0, chunk = 0;
        if (i < num_chunks) {
            const uint2 t = chunk_tasks[i];
            const LongRow L = long_rows[t.x];
            const uint64_t rb = in_off[L.row], re = in_off[L.row + 1];
            e0 = rb + uint64_t(t.y) * kLongChunk;
            len = ((e0 + kLongChunk < re) ? e0 + kLongChunk : re) - e0;
            a = t.x;
            b = t.y;
            chunk = 1;
        } else {
            const uint64_t k = i - num_chunks;
            const uint32_t r0 = tile_start[k], r1 = tile_start[k + 1];
            a = b = r0;
            e0 = in_off[r0];
            if (r0 != r1) {
                const uint64_t last_b = in_off[r1 - 1], last_e = in_off[r1];
                const uint32_t rl = (last_e - last_b >= tile_cost) ? r1 - 1 : r1;  // a long last row is chunked
                len = ((rl == r1) ? last_e : last_b) - e0;
                b = rl;
            }
        }
        out[i] = make_uint4(static_cast<uint32_t>(e0),
                            static_cast<uint32_t>((e0 >> 32) & 0xFFu) | static_cast<uint32_t>(len << 8) | (chunk << 31),
                            a, b);
    }
}

// Work tiles and long-row chunks of the pull side, from g.in_offsets on the
// device (g.V, g.E, g.tile_cost set).  Shared by graph_build and the
// out-of-HBM engine.
void build_pull_tiles(GraphImpl &g, cudaStream_t s) {
    const uint64_t V = g.V, E = g.E;
    // Work tiles along the merge path.
    g.num_tiles = (V + E) / g.tile_cost + 1;
    g.tile_start.allocate(g.num_tiles + 1);
    tile_bounds_kernel<<<grid_for(V + 1, 256), 256, 0, s>>>(g.in_offsets.get(), V, E, g.num_tiles, g.tile_cost,
                                                             g.tile_start.get());
    HYT_CUDA(cudaGetLastError());

    // Long rows (in-degree >= tile_cost) and their chunk tasks.
    Scratch<uint32_t> in_deg(V, s);
    Scratch<uint8_t> is_long(V, s);
    in_degree_kernel<<<grid_for(V, 256), 256, 0, s>>>(g.in_offsets.get(), V, g.tile_cost, in_deg.get(),
                                                       is_long.get());
    HYT_CUDA(cudaGetLastError());
    g.max_in_degree = prims::reduce_max_u32(in_deg.get(), V, s);
    Scratch<uint32_t> long_ids(V, s);
    g.num_long = prims::select_flagged_index(is_long.get(), long_ids.get(), V, s);
    std::vector<LongRow> lr(g.num_long);
    std::vector<uint2> tasks;
    if (g.num_long) {
        Scratch<uint32_t> long_deg(g.num_long, s);
        gather_u32_kernel<<<grid_for(g.num_long, 256), 256, 0, s>>>(in_deg.get(), long_ids.get(), g.num_long,
                                                                     long_deg.get());
        HYT_CUDA(cudaGetLastError());
        std::vector<uint32_t> ids(g.num_long), degs(g.num_long);
        HYT_CUDA(cudaMemcpyAsync(ids.data(), long_ids.get(), g.num_long * 4, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaMemcpyAsync(degs.data(), long_deg.get(), g.num_long * 4, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        uint32_t next = 0;
        for (uint64_t i = 0; i < g.num_long; ++i) {
            const uint32_t nc = (degs[i] + kLongChunk - 1) / kLongChunk;
            lr[i] = LongRow{ids[i], next, nc, 0};
            for (uint32_t c = 0; c < nc; ++c) tasks.push_back(make_uint2(static_cast<uint32_t>(i), c));
            next += nc;
        }
    }
    g.num_chunks = tasks.size();
    g.long_rows.allocate(std::max<uint64_t>(g.num_long, 1));
    g.chunk_tasks.allocate(std::max<uint64_t>(g.num_chunks, 1));
    if (g.num_long)
        HYT_CUDA(cudaMemcpyAsync(g.long_rows.get(), lr.data(), lr.size() * sizeof(LongRow),
                                 cudaMemcpyHostToDevice, s));
    if (g.num_chunks)
        HYT_CUDA(cudaMemcpyAsync(g.chunk_tasks.get(), tasks.data(), tasks.size() * sizeof(uint2),
                                 cudaMemcpyHostToDevice, s));
    // One descriptor per task (first edges below 2^40).
    const uint64_t ntasks = g.num_chunks + g.num_tiles;
    g.pull_tasks.allocate(ntasks);
    pull_task_kernel<<<grid_for(ntasks, 256), 256, 0, s>>>(g.in_offsets.get(), g.tile_start.get(), g.long_rows.get(),
                                                            g.chunk_tasks.get(), g.num_chunks, g.num_tiles, g.tile_cost,
                                                            g.pull_tasks.get());
    HYT_CUDA(cudaGetLastError());
    HYT_CUDA(cudaStreamSynchronize(s));
}

void graph_build(GraphImpl &g, const hyt_csr &csr, uint32_t flags) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (V == 0) fail(HYT_E_INVALID, "graph requires at least one vertex");
    if (V > 0xFFFFFFFFull) fail(HYT_E_INVALID, "vertex ids are uint32: num_vertices must be < 2^32");
    if (E > 0xFFFFFFFEull) fail(HYT_E_UNSUPPORTED, "in-HBM graphs hold fewer than 2^32 edges");
    if (!csr.row_offsets) fail(HYT_E_INVALID, "row_offsets is NULL");
    if (E > 0 && !csr.column_indices) fail(HYT_E_INVALID, "column_indices is NULL");
    if (csr.weight_kind > HYT_WEIGHTS_F32) fail(HYT_E_INVALID, "unknown weight_kind");
    if (csr.weight_kind != HYT_WEIGHTS_NONE && E > 0 && !csr.weights)
        fail(HYT_E_INVALID, "weights is NULL for a weighted graph");
    if (flags == 0) flags = HYT_GRAPH_ALL;
    // PageRank decomposition knobs (same work, different tiling): tile cost
    // in {64..512} and hot-source cache size, bounded by shared memory.  The
    // staged kernels (HYT_STAGED=1) need tiles that fit one staging slot.
    g.tile_cost = stage::staged_requested() ? kStageTileMax : kTileCostDefault;
    if (const char *t = std::getenv("HYT_PR_TILE")) {
        const unsigned long v = std::strtoul(t, nullptr, 10);
        if (v >= 64 && v <= kTileCostMax) g.tile_cost = static_cast<uint32_t>(v);
    }
    uint32_t hot_request = kHotSourcesDefault;
    if (const char *t = std::getenv("HYT_PR_HOT")) hot_request = static_cast<uint32_t>(std::strtoul(t, nullptr, 10));
    hot_request = std::min(hot_request, kHotSourcesMax);
    while (hot_request && pr_shared_bytes(hot_request, g.tile_cost) > kPRSmemMax) hot_request /= 2;
    if ((flags & HYT_GRAPH_PULL) && V > (kHotTag >> 0) - 1)
        fail(HYT_E_UNSUPPORTED, "pull graphs hold fewer than 2^31 vertices (bit 31 tags cached sources)");

    cudaStream_t s = g.stream;
    EventTimer timer;
    timer.start(s);

    g.V = V;
    g.E = E;
    g.flags = flags;
    g.weight_kind = csr.weight_kind;

    g.row_offsets.allocate(V + 1);
    copy_to_device(g.row_offsets.get(), csr.row_offsets, (V + 1) * sizeof(uint64_t), s);
    g.cols.allocate(E ? E : 1);
    if (E) copy_to_device(g.cols.get(), csr.column_indices, E * sizeof(uint32_t), s);
    const bool keep_weights = (flags & HYT_GRAPH_PUSH) && csr.weight_kind != HYT_WEIGHTS_NONE;
    if (keep_weights) {
        g.weights.allocate(E ? E : 1);
        if (E) copy_to_device(g.weights.get(), csr.weights, E * sizeof(uint32_t), s);
    }

    // Validation: malformed offsets or out-of-range ids would turn into
    // out-of-bounds device accesses later, so they are rejected here.
    Scratch<uint32_t> err(1, s);
    Scratch<unsigned long long> counter(1, s);
    HYT_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(uint32_t), s));
    HYT_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(unsigned long long), s));
    validate_offsets_kernel<<<grid_for(V, 256), 256, 0, s>>>(g.row_offsets.get(), V, E, err.get());
    HYT_CUDA(cudaGetLastError());
    uint32_t h_err = 0;
    HYT_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(h_err), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (h_err & kBadOffsets) fail(HYT_E_INVALID, "row offsets must start at 0 and be non-decreasing");
    if (h_err & kBadTerminal) fail(HYT_E_INVALID, "terminal row offset must equal the number of edges");
    if (E) {
        Scratch<unsigned long long> wsum(1, s);
        HYT_CUDA(cudaMemsetAsync(wsum.get(), 0, sizeof(unsigned long long), s));
        validate_edges_kernel<<<grid_for(E, 256), 256, 0, s>>>(g.cols.get(), keep_weights ? g.weights.get() : nullptr,
                                                                keep_weights ? csr.weight_kind : 0u, V, E, err.get(),
                                                                wsum.get());
        HYT_CUDA(cudaGetLastError());
        unsigned long long h_wsum = 0;
        HYT_CUDA(cudaMemcpyAsync(&h_err, err.get(), sizeof(h_err), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaMemcpyAsync(&h_wsum, wsum.get(), sizeof(h_wsum), cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        if (h_err & kBadColumn) fail(HYT_E_INVALID, "column index contains an invalid destination vertex ID");
        // Negative / non-finite float weights are legal for PageRank; SSSP
        // rejects them when it is called (reference: sssp.cpp:117-124).
        g.weights_ok = (h_err & kBadWeight) == 0;
        if (keep_weights && csr.weight_kind == HYT_WEIGHTS_U32) {
            const double mean = static_cast<double>(h_wsum) / static_cast<double>(E);
            g.default_delta = static_cast<uint32_t>(std::min(4.0e9, std::max(1.0, 2.0 * mean)));
        }
    }

    g.out_degree.allocate(V);
    out_degree_kernel<<<grid_for(V, 256), 256, 0, s>>>(g.row_offsets.get(), V, g.out_degree.get(), counter.get());
    HYT_CUDA(cudaGetLastError());
    unsigned long long h_dangling = 0;
    HYT_CUDA(cudaMemcpyAsync(&h_dangling, counter.get(), sizeof(h_dangling), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    g.dangling = h_dangling;
    g.max_out_degree = prims::reduce_max_u32(g.out_degree.get(), V, s);

    if (flags & HYT_GRAPH_PULL) {
        // CSC transpose: stable sort of (destination, source) by destination.
        // Graphs that keep both sides with weights also get the weights in
        // CSC order (SSSP pull rounds): sort edge ids instead, then gather.
        Scratch<uint32_t> keys(E ? E : 1, s);
        g.in_sources.allocate(E ? E : 1);
        const bool csc_weights = (flags & HYT_GRAPH_PUSH) && keep_weights && g.weights.get();
        if (E) {
            HYT_CUDA(cudaMemcpyAsync(keys.get(), g.cols.get(), E * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
            if (csc_weights) {
                // (source, weight) packed into one 64-bit value travels with
                // its destination key: every pass streams, no gathers
                Scratch<uint64_t> sw(E, s);
                {
                    Scratch<uint32_t> src(E, s);
                    expand_sources(g.row_offsets.get(), V, E, src.get(), s);
                    pack_pairs_kernel<<<grid_for(E, 256), 256, 0, s>>>(src.get(), g.weights.get(), E, sw.get());
                    HYT_CUDA(cudaGetLastError());
                }
                prims::sort_pairs_u32_u64(keys.get(), sw.get(), E, bits_for(V - 1), s);
                g.in_weights.allocate(E);
                unpack_pairs_kernel<<<grid_for(E, 256), 256, 0, s>>>(sw.get(), E, g.in_sources.get(),
                                                                      g.in_weights.get());
                HYT_CUDA(cudaGetLastError());
                HYT_CUDA(cudaStreamSynchronize(s));
            } else {
                expand_sources(g.row_offsets.get(), V, E, g.in_sources.get(), s);
                prims::sort_pairs_u32(keys.get(), g.in_sources.get(), E, bits_for(V - 1), s);
            }
        }
        g.in_offsets.allocate(V + 1);
        offsets_from_sorted_kernel<<<grid_for(E + 1, 256), 256, 0, s>>>(keys.get(), E, V, g.in_offsets.get());
        HYT_CUDA(cudaGetLastError());
        keys.release();

        // Hot sources: largest out-degree first (ties by vertex id).
        g.num_hot = static_cast<uint32_t>(std::min<uint64_t>(hot_request, V));
        if (E && g.num_hot) {
            Scratch<uint32_t> deg(V, s), ids(V, s), slot(V, s);
            HYT_CUDA(cudaMemcpyAsync(deg.get(), g.out_degree.get(), V * 4, cudaMemcpyDeviceToDevice, s));
            iota_kernel<<<grid_for(V, 256), 256, 0, s>>>(ids.get(), V);
            HYT_CUDA(cudaGetLastError());
            prims::sort_pairs_desc_u32(deg.get(), ids.get(), V, s);
            g.hot_vertex.allocate(g.num_hot);
            HYT_CUDA(cudaMemcpyAsync(g.hot_vertex.get(), ids.get(), g.num_hot * 4ull, cudaMemcpyDeviceToDevice, s));
            HYT_CUDA(cudaMemsetAsync(slot.get(), 0xFF, V * 4, s));
            hot_slot_kernel<<<(g.num_hot + 255) / 256, 256, 0, s>>>(g.hot_vertex.get(), g.num_hot, slot.get());
            HYT_CUDA(cudaMemsetAsync(counter.get(), 0, sizeof(unsigned long long), s));
            tag_hot_kernel<<<grid_for(E, 256), 256, 0, s>>>(g.in_sources.get(), E, slot.get(), counter.get());
            HYT_CUDA(cudaGetLastError());
            unsigned long long h_hot = 0;
            HYT_CUDA(cudaMemcpyAsync(&h_hot, counter.get(), sizeof(h_hot), cudaMemcpyDeviceToHost, s));
            HYT_CUDA(cudaStreamSynchronize(s));
            g.hot_edges = h_hot;
        } else {
            g.num_hot = 0;
        }

        build_pull_tiles(g, s);
    }

    if (!(flags & HYT_GRAPH_PUSH)) {
        // Pull-only graphs keep the CSC; the CSR edges are not needed.
        g.cols.release();
        g.weights.release();
    }
    timer.stop(s);
    g.build_ms = timer.ms();
}

}  // namespace hyt
