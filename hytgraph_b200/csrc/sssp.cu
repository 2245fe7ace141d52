// Single-source shortest paths: frontier push over the CSR with atomicMin.
//
// The reference solver (src/algorithms/sssp.cpp:109-234, cuda/sssp.cu:
// 100-154) is a synchronous Bellman-Ford that pulls over all in-edges every
// round.  Any label-correcting schedule reaches the same fixed point
//     d[s] = 0,  d[v] = min_{u->v} (d[u] + w(u,v))
// because every relaxation only lowers a label to a value that some path
// attains; so distances are bit-identical to the reference.  Integer (u32)
// weights relax with exact integer adds; float weights relax with the same
// IEEE add the reference uses, compared as ordered bit patterns (valid for
// non-negative floats).
//
// Per round only the frontier (vertices whose label dropped in the previous
// round) is expanded.  A CTA stages 256 frontier vertices (row offset,
// degree, label) in shared memory, prefix-sums their degrees, and all its
// threads walk the combined edge list, so rows of any length are balanced
// inside the CTA.  Rows of >= kHubDegree edges are cut into kHubChunk-edge
// tasks for a second, grid-wide kernel.  A vertex joins the next frontier
// once per round (round stamp), appended with one warp-aggregated atomic.
// All round state lives on the device; inside a CUDA graph the rounds run
// as a conditional while-loop with no host round trip.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "graph.cuh"
#include "solvers.cuh"

namespace cg = cooperative_groups;

namespace hyt {
namespace {

constexpr int kSSThreads = 256;
constexpr uint32_t kHubDegree = 4096;
constexpr uint32_t kHubChunk = 4096;

struct SSHeader {
    uint32_t round;     // rounds completed
    uint32_t done;
    uint32_t converged;
    uint32_t qsize[2];  // frontier sizes, indexed by round parity
    uint32_t hub_count;
    uint32_t max_rounds;
    uint32_t pad;
    unsigned long long relaxations;     // edges relaxed
    unsigned long long frontier_total;  // frontier vertices expanded
};

struct SSArgs {
    const uint64_t *row_off;
    const uint32_t *cols;
    const uint32_t *weights;
    uint32_t *dist;
    uint32_t *stamp;
    uint32_t *queue[2];
    uint2 *hubs;
    SSHeader *hdr;
    uint32_t V;
    uint32_t source;
    uint32_t inf;
    uint32_t use_cond;
    cudaGraphConditionalHandle cond;
};

template <int WK>
__device__ __forceinline__ uint32_t edge_weight(const uint32_t *w, uint64_t e) {
    if constexpr (WK == HYT_WEIGHTS_NONE) {
        return 1u;
    } else {
        return dev::ld_stream(w + e);
    }
}

template <int WK>
__device__ __forceinline__ uint32_t extend(uint32_t d, uint32_t w) {
    if constexpr (WK == HYT_WEIGHTS_F32) {
        return __float_as_uint(__fadd_rn(__uint_as_float(d), __uint_as_float(w)));
    } else {
        const uint64_t s = uint64_t(d) + w;
        return s >= 0xFFFFFFFFull ? 0xFFFFFFFEu : static_cast<uint32_t>(s);
    }
}

__device__ __forceinline__ void relax(uint32_t *dist, uint32_t *stamp, uint32_t u, uint32_t nd,
                                      uint32_t next_stamp, uint32_t *qnext, uint32_t *qnext_size) {
    if (nd < __ldcg(dist + u)) {
        const uint32_t old = atomicMin(dist + u, nd);
        if (nd < old && atomicExch(stamp + u, next_stamp) != next_stamp) {
            cg::coalesced_group g = cg::coalesced_threads();
            uint32_t base = 0;
            if (g.thread_rank() == 0) base = atomicAdd(qnext_size, g.size());
            base = g.shfl(base, 0);
            qnext[base + g.thread_rank()] = u;
        }
    }
}

template <int WK>
__global__ void __launch_bounds__(kSSThreads) sssp_expand_kernel(const SSArgs *__restrict__ args) {
    __shared__ uint32_t s_scan[kSSThreads + 1];
    __shared__ uint64_t s_off[kSSThreads];
    __shared__ uint32_t s_d[kSSThreads];
    __shared__ uint32_t s_wsum[kSSThreads / 32];

    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done) return;
    const uint32_t r = *(volatile uint32_t *)&a.hdr->round;
    const uint32_t qn = *(volatile uint32_t *)((r & 1) ? &a.hdr->qsize[1] : &a.hdr->qsize[0]);
    const uint32_t *q = (r & 1) ? a.queue[1] : a.queue[0];
    uint32_t *qnext = (r & 1) ? a.queue[0] : a.queue[1];
    uint32_t *qnext_size = (r & 1) ? &a.hdr->qsize[0] : &a.hdr->qsize[1];
    const uint32_t next_stamp = r + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    unsigned long long relaxed = 0;

    for (uint32_t chunk = blockIdx.x; uint64_t(chunk) * kSSThreads < qn; chunk += gridDim.x) {
        const uint32_t i = chunk * kSSThreads + tid;
        uint32_t deg = 0, d = a.inf;
        uint64_t off = 0;
        if (i < qn) {
            const uint32_t v = q[i];
            off = a.row_off[v];
            const uint64_t full = a.row_off[v + 1] - off;
            d = __ldcg(a.dist + v);
            if (full >= kHubDegree) {
                const uint32_t nch = static_cast<uint32_t>((full + kHubChunk - 1) / kHubChunk);
                const uint32_t base = atomicAdd(&a.hdr->hub_count, nch);
                for (uint32_t c = 0; c < nch; ++c) a.hubs[base + c] = make_uint2(v, c);
                relaxed += full;
            } else {
                deg = static_cast<uint32_t>(full);
            }
        }
        // block-wide exclusive prefix of the staged degrees
        uint32_t x = deg;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t w = (lane < kSSThreads / 32) ? s_wsum[lane] : 0u;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < kSSThreads / 32) s_wsum[lane] = w;
        }
        __syncthreads();
        const uint32_t excl = x - deg + (warp > 0 ? s_wsum[warp - 1] : 0u);
        s_scan[tid] = excl;
        s_off[tid] = off;
        s_d[tid] = d;
        if (tid == kSSThreads - 1) s_scan[kSSThreads] = excl + deg;
        __syncthreads();
        const uint32_t total = s_scan[kSSThreads];
        if (tid == 0) relaxed += total;
        for (uint32_t j = tid; j < total; j += kSSThreads) {
            int lo = 0, hi = kSSThreads - 1;  // last staged vertex whose prefix <= j
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (s_scan[mid] <= j) lo = mid; else hi = mid - 1;
            }
            const uint64_t e = s_off[lo] + (j - s_scan[lo]);
            const uint32_t u = dev::ld_stream(a.cols + e);
            const uint32_t w = edge_weight<WK>(a.weights, e);
            relax(a.dist, a.stamp, u, extend<WK>(s_d[lo], w), next_stamp, qnext, qnext_size);
        }
        __syncthreads();
    }
    if (relaxed) atomicAdd(&a.hdr->relaxations, relaxed);
}

template <int WK>
__global__ void __launch_bounds__(kSSThreads) sssp_hub_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    if (*(volatile uint32_t *)&a.hdr->done) return;
    const uint32_t r = *(volatile uint32_t *)&a.hdr->round;
    const uint32_t n = *(volatile uint32_t *)&a.hdr->hub_count;
    uint32_t *qnext = (r & 1) ? a.queue[0] : a.queue[1];
    uint32_t *qnext_size = (r & 1) ? &a.hdr->qsize[0] : &a.hdr->qsize[1];
    const uint32_t next_stamp = r + 1;
    for (uint32_t t = blockIdx.x; t < n; t += gridDim.x) {
        const uint2 h = a.hubs[t];
        const uint64_t rb = a.row_off[h.x], re = a.row_off[h.x + 1];
        const uint64_t b = rb + uint64_t(h.y) * kHubChunk;
        const uint64_t e = (b + kHubChunk < re) ? b + kHubChunk : re;
        const uint32_t d = __ldcg(a.dist + h.x);
        for (uint64_t x = b + threadIdx.x; x < e; x += kSSThreads) {
            const uint32_t u = dev::ld_stream(a.cols + x);
            relax(a.dist, a.stamp, u, extend<WK>(d, edge_weight<WK>(a.weights, x)), next_stamp, qnext, qnext_size);
        }
    }
}

__global__ void sssp_round_end_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    SSHeader *h = a.hdr;
    if (h->done) return;
    const uint32_t r = h->round;
    const uint32_t n_next = h->qsize[(r + 1) & 1];
    h->frontier_total += h->qsize[r & 1];
    h->qsize[r & 1] = 0;
    h->hub_count = 0;
    h->round = r + 1;
    if (n_next == 0 || r + 1 >= h->max_rounds) {
        h->done = 1;
        h->converged = (n_next == 0) ? 1u : 0u;
        if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
    }
}

__global__ void sssp_init_kernel(const SSArgs *__restrict__ args) {
    const SSArgs a = *args;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < a.V; v += stride) {
        const bool s = (v == a.source);
        a.dist[v] = s ? 0u : a.inf;
        a.stamp[v] = s ? 0u : 0xFFFFFFFFu;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.queue[0][0] = a.source;
}

template <int WK>
struct SSKernels {
    static int grid() {
        static int g = 0;
        if (g == 0) {
            int per_sm = 0;
            HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sssp_expand_kernel<WK>, kSSThreads, 0));
            g = sm_count() * std::max(per_sm, 1);
        }
        return g;
    }
};

template <int WK>
void sssp_solve(GraphImpl &g, uint32_t source, uint32_t max_rounds, uint32_t flags, cudaStream_t s,
                uint32_t *dist_out, hyt_run_stats *stats) {
    const uint64_t V = g.V;
    if (g.dist.count < V) g.dist.allocate(V);
    if (g.stamp.count < V) g.stamp.allocate(V);
    for (int i = 0; i < 2; ++i)
        if (g.queue[i].count < V) g.queue[i].allocate(V);
    const uint64_t hub_cap = 2 * (g.E / kHubChunk) + 2;
    if (g.hub_tasks.count < hub_cap) g.hub_tasks.allocate(hub_cap);
    const size_t sb = 512 + sizeof(SSHeader);
    if (g.sssp_state.count < sb) g.sssp_state.allocate(sb);
    SSArgs *d_args = reinterpret_cast<SSArgs *>(g.sssp_state.get());
    SSHeader *hdr = reinterpret_cast<SSHeader *>(g.sssp_state.get() + 256);

    SSArgs a{};
    a.row_off = g.row_offsets.get();
    a.cols = g.cols.get();
    a.weights = g.weights.get();
    a.dist = g.dist.get();
    a.stamp = g.stamp.get();
    a.queue[0] = g.queue[0].get();
    a.queue[1] = g.queue[1].get();
    a.hubs = g.hub_tasks.get();
    a.hdr = hdr;
    a.V = static_cast<uint32_t>(V);
    a.source = source;
    a.inf = (WK == HYT_WEIGHTS_F32) ? 0x7F800000u : HYT_DIST_INF_U32;

    SSHeader h0{};
    h0.qsize[0] = 1;
    h0.max_rounds = max_rounds;

    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH) && !(flags & HYT_RUN_PROFILE);
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
        HYT_CUDA(cudaGraphCreate(&graph, 0));
        HYT_CUDA(cudaGraphConditionalHandleCreate(&a.cond, graph, 1, cudaGraphCondAssignDefault));
        a.use_cond = 1;
    }
    const int grid = SSKernels<WK>::grid();

    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(a), cudaMemcpyHostToDevice, s));
    HYT_CUDA(cudaMemcpyAsync(hdr, &h0, sizeof(h0), cudaMemcpyHostToDevice, s));
    sssp_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    uint32_t launches = 1, hot = 0;
    double kernel_ms = 0.0;

    if (use_graph) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = a.cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        HYT_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        void *kargs[] = {&d_args};
        cudaKernelNodeParams kp = {};
        kp.kernelParams = kargs;
        kp.blockDim = dim3(kSSThreads);
        kp.gridDim = dim3(grid);
        kp.func = reinterpret_cast<void *>(sssp_expand_kernel<WK>);
        cudaGraphNode_t n1, n2, n3;
        HYT_CUDA(cudaGraphAddKernelNode(&n1, body, nullptr, 0, &kp));
        kp.func = reinterpret_cast<void *>(sssp_hub_kernel<WK>);
        HYT_CUDA(cudaGraphAddKernelNode(&n2, body, &n1, 1, &kp));
        kp.func = reinterpret_cast<void *>(sssp_round_end_kernel);
        kp.gridDim = dim3(1);
        kp.blockDim = dim3(1);
        HYT_CUDA(cudaGraphAddKernelNode(&n3, body, &n2, 1, &kp));
        HYT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        HYT_CUDA(cudaGraphLaunch(exec, s));
    } else {
        EventTimer kt;
        for (uint32_t r = 0; r < max_rounds; ++r) {
            if (flags & HYT_RUN_PROFILE) kt.start(s);
            sssp_expand_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args);
            sssp_hub_kernel<WK><<<grid, kSSThreads, 0, s>>>(d_args);
            if (flags & HYT_RUN_PROFILE) kt.stop(s);
            sssp_round_end_kernel<<<1, 1, 0, s>>>(d_args);
            HYT_CUDA(cudaGetLastError());
            launches += 3;
            hot += 2;
            uint32_t done = 0;
            HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
            HYT_CUDA(cudaStreamSynchronize(s));
            if (flags & HYT_RUN_PROFILE) kernel_ms += kt.ms();
            if (done) break;
        }
    }
    SSHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    total.stop(s);
    const double total_ms = total.ms();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (use_graph) launches += 3 * h.round;
    if (dist_out) copy_from_device(dist_out, g.dist.get(), V * sizeof(uint32_t), s);
    if (stats) {
        stats->iterations = h.round;
        stats->converged = h.converged;
        stats->residual = 0.0;
        stats->device_ms = total_ms;
        stats->kernel_ms = kernel_ms;
        stats->kernel_launches = hot;
        stats->total_launches = launches;
        stats->edges_processed = h.relaxations;
        stats->vertices_processed = h.frontier_total;
        // per frontier vertex: 8 B offset pair (read twice) + 4 B label +
        // 4 B queue entry; per edge: 4 B column + 4 B weight + 4 B label.
        stats->algorithmic_bytes = 16ull * h.frontier_total + 12ull * h.relaxations;
    }
}

}  // namespace

void sssp_run(GraphImpl &g, const hyt_sssp_params &p, uint32_t *dist_out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PUSH)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PUSH");
    if (p.source >= g.V) fail(HYT_E_INVALID, "SSSP source vertex is out of range");
    if (!g.weights_ok) fail(HYT_E_INVALID, "SSSP requires finite non-negative edge weights");
    cudaStream_t s = p.stream ? static_cast<cudaStream_t>(p.stream) : g.stream;
    // Each round lowers at least one label; with non-negative weights the
    // label-correcting frontier empties within V rounds.
    const uint32_t max_rounds = p.max_rounds ? p.max_rounds : static_cast<uint32_t>(std::min<uint64_t>(g.V + 1, 0xFFFFFFF0ull));
    switch (g.weight_kind) {
        case HYT_WEIGHTS_NONE: sssp_solve<HYT_WEIGHTS_NONE>(g, p.source, max_rounds, p.flags, s, dist_out, stats); break;
        case HYT_WEIGHTS_U32: sssp_solve<HYT_WEIGHTS_U32>(g, p.source, max_rounds, p.flags, s, dist_out, stats); break;
        case HYT_WEIGHTS_F32: sssp_solve<HYT_WEIGHTS_F32>(g, p.source, max_rounds, p.flags, s, dist_out, stats); break;
        default: fail(HYT_E_INTERNAL, "unknown weight kind");
    }
}

}  // namespace hyt
