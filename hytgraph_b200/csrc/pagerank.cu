// PageRank and personalized PageRank: synchronous (Jacobi) pull over the CSC.
//
// Semantics follow the reference CPU solver (src/algorithms/pagerank.cpp:
// 89-163): x_0 = 1/n; each step
//     x'[v] = (1-d)/n + d * dangling / n + d * sum_{u->v} x[u] / deg(u)
// with dangling = sum of x over out-degree-0 vertices, residual = L1 change,
// stop when residual <= tolerance or after max_iterations.  Per-edge
// contributions x[u]/deg(u) are formed once per vertex in the producing
// step (the reference divides per edge, same float quotient).  In-row sums
// are compensated (TwoSum/Kahan) in FP32; residual and dangling mass are
// reduced in FP64.
//
// One persistent kernel per iteration.  CTAs pull tasks from a counter:
//   chunk tasks  -- 8192-edge slices of rows with in-degree >= 4096; each
//                   CTA writes a compensated partial, the last arriving CTA
//                   of a row merges the partials in chunk order;
//   tile tasks   -- merge-path tiles of consecutive rows; the tile's
//                   in-sources are read with 128-bit streaming loads, the
//                   contributions gathered into shared memory, then reduced
//                   thread-per-row (in-degree < 32) or warp-per-row.
// Results are deterministic: every sum has a fixed association order.
// The last CTA to finish an iteration evaluates the stop rule and, inside a
// CUDA graph, ends the conditional while-loop.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "common.cuh"
#include "graph.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

constexpr int kPRThreads = 256;
constexpr uint32_t kWarpRowDegree = 32;
constexpr uint32_t kMaxWarpRows = kStageCap / kWarpRowDegree + 1;

struct PRHeader {
    uint32_t iter;       // iterations completed
    uint32_t done;
    uint32_t converged;
    uint32_t pad;
    double last_residual;
};

// Device-resident arguments (a cached CUDA graph reads them every launch).
struct PRArgs {
    const uint64_t *in_off;
    const uint32_t *in_src;
    const uint32_t *out_deg;
    const uint32_t *tile_start;
    const LongRow *long_rows;
    const uint2 *chunk_tasks;
    float *rank[2];
    float *contrib[2];
    float2 *partial;
    uint32_t *ticket;
    PRHeader *hdr;
    uint32_t *task_counter;  // [max_iter]
    uint32_t *finished;      // [max_iter]
    double *residual;        // [max_iter]
    double *dangling;        // [max_iter + 1]
    uint64_t num_tiles;
    uint32_t num_chunks;
    uint32_t V;
    float damping;
    float base;         // PR: (1-d)/n
    float tolerance;
    uint32_t max_iter;
    uint32_t source;    // PPR
    uint32_t personalized;
    cudaGraphConditionalHandle cond;
    uint32_t use_cond;
};

struct PRState {
    // per-iteration scalars
    float damping, base, teleport_scale;
    float dshare;  // PR: d * dangling / n
    float tele;    // PPR: (1-d) + d * dangling
    uint32_t source;
    bool personalized;
};

__device__ __forceinline__ void finalize_row(const PRArgs &a, const PRState &ps, uint32_t r, float sum,
                                             const float *cur, float *nxt, float *cnxt, double &res, double &dang) {
    float nx;
    if (ps.personalized) {
        nx = __fmul_rn(ps.damping, sum);
        if (r == ps.source) nx = __fadd_rn(ps.tele, nx);
    } else {
        nx = __fadd_rn(ps.dshare, __fmul_rn(ps.damping, sum));
    }
    const float old = cur[r];
    res += fabs(static_cast<double>(nx) - static_cast<double>(old));
    nxt[r] = nx;
    const uint32_t od = a.out_deg[r];
    cnxt[r] = od ? __fdiv_rn(nx, static_cast<float>(od)) : 0.0f;
    if (od == 0) dang += static_cast<double>(nx);
}

// Compensated block reduction; result valid in thread 0.
__device__ __forceinline__ dev::CSum block_csum(dev::CSum v, float2 *scratch) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = dev::warp_reduce(v);
    __syncthreads();
    if (lane == 0) scratch[warp] = make_float2(v.s, v.c);
    __syncthreads();
    dev::CSum t;
    if (threadIdx.x == 0) {
        const int nw = blockDim.x >> 5;
        for (int w = 0; w < nw; ++w) {
            dev::CSum x;
            x.s = scratch[w].x;
            x.c = scratch[w].y;
            t.merge(x);
        }
    }
    return t;
}

__global__ void __launch_bounds__(kPRThreads) pr_iterate_kernel(const PRArgs *__restrict__ args) {
    __shared__ __align__(16) float s_vals[kStageCap + 8];
    __shared__ uint32_t s_warp_rows[kMaxWarpRows];
    __shared__ uint32_t s_nwarp_rows;
    __shared__ uint32_t s_task;
    __shared__ float2 s_red2[kPRThreads / 32];
    __shared__ double s_red[32];

    const PRArgs a = *args;
    const uint32_t it = *(volatile uint32_t *)&a.hdr->iter;
    if (*(volatile uint32_t *)&a.hdr->done) return;

    const float *cur = (it & 1) ? a.rank[1] : a.rank[0];
    float *nxt = (it & 1) ? a.rank[0] : a.rank[1];
    const float *ccur = (it & 1) ? a.contrib[1] : a.contrib[0];
    float *cnxt = (it & 1) ? a.contrib[0] : a.contrib[1];

    PRState ps;
    ps.damping = a.damping;
    ps.source = a.source;
    ps.personalized = a.personalized != 0;
    const double dmass = a.dangling[it];
    ps.dshare = __fadd_rn(a.base, static_cast<float>(static_cast<double>(a.damping) * dmass / static_cast<double>(a.V)));
    ps.tele = static_cast<float>((1.0 - static_cast<double>(a.damping)) + static_cast<double>(a.damping) * dmass);

    const uint64_t pol = dev::policy_evict_last();
    const uint64_t total_tasks = a.num_chunks + a.num_tiles;
    double res = 0.0, dang = 0.0;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarps = kPRThreads / 32;

    for (;;) {
        if (tid == 0) s_task = atomicAdd(&a.task_counter[it], 1u);
        __syncthreads();
        const uint32_t task = s_task;
        __syncthreads();
        if (task >= total_tasks) break;

        if (task < a.num_chunks) {
            // ---- slice of a long row ------------------------------------
            const uint2 t = a.chunk_tasks[task];
            const LongRow L = a.long_rows[t.x];
            const uint64_t rb = a.in_off[L.row], re = a.in_off[L.row + 1];
            const uint64_t b = rb + uint64_t(t.y) * kLongChunk;
            const uint64_t e = (b + kLongChunk < re) ? b + kLongChunk : re;
            dev::CSum acc;
            const uint64_t b4 = b & ~3ull;
            const uint64_t nvec = (e - b4 + 3) >> 2;
            const uint4 *src4 = reinterpret_cast<const uint4 *>(a.in_src + b4);
            for (uint64_t i = tid; i < nvec; i += kPRThreads) {
                const uint4 q = dev::ld_stream4(src4 + i);
                const uint64_t x = b4 + 4 * i;
                const float v0 = (x + 0 >= b && x + 0 < e) ? dev::ld_keep(ccur + q.x, pol) : 0.f;
                const float v1 = (x + 1 >= b && x + 1 < e) ? dev::ld_keep(ccur + q.y, pol) : 0.f;
                const float v2 = (x + 2 >= b && x + 2 < e) ? dev::ld_keep(ccur + q.z, pol) : 0.f;
                const float v3 = (x + 3 >= b && x + 3 < e) ? dev::ld_keep(ccur + q.w, pol) : 0.f;
                acc.add(v0);
                acc.add(v1);
                acc.add(v2);
                acc.add(v3);
            }
            const dev::CSum tot = block_csum(acc, s_red2);
            if (tid == 0) {
                a.partial[L.first_chunk + t.y] = make_float2(tot.s, tot.c);
                __threadfence();
                const uint32_t tk = atomicAdd(&a.ticket[t.x], 1u) + 1u;
                if (tk % L.num_chunks == 0) {
                    __threadfence();
                    dev::CSum row;
                    for (uint32_t j = 0; j < L.num_chunks; ++j) {
                        const float2 p = __ldcg(a.partial + L.first_chunk + j);
                        dev::CSum x;
                        x.s = p.x;
                        x.c = p.y;
                        row.merge(x);
                    }
                    finalize_row(a, ps, L.row, row.value(), cur, nxt, cnxt, res, dang);
                }
            }
            __syncthreads();
        } else {
            // ---- merge-path tile of consecutive rows --------------------
            const uint64_t k = task - a.num_chunks;
            const uint32_t r0 = a.tile_start[k];
            const uint32_t r1 = a.tile_start[k + 1];
            if (r0 == r1) continue;
            uint32_t rl = r1;  // rows [r0, rl) are staged; a long last row is chunked
            const uint64_t last_b = a.in_off[r1 - 1], last_e = a.in_off[r1];
            if (last_e - last_b >= kLongDegree) rl = r1 - 1;
            const uint64_t e0 = a.in_off[r0];
            const uint64_t e1 = (rl == r1) ? last_e : last_b;
            const uint64_t a0 = e0 & ~3ull;
            const uint32_t nvec = static_cast<uint32_t>((e1 - a0 + 3) >> 2);
            const uint4 *src4 = reinterpret_cast<const uint4 *>(a.in_src + a0);
            float4 *sv4 = reinterpret_cast<float4 *>(s_vals);
            if (tid == 0) s_nwarp_rows = 0;
            for (uint32_t i = tid; i < nvec; i += kPRThreads) {
                const uint4 q = dev::ld_stream4(src4 + i);
                const uint64_t x = a0 + 4ull * i;
                float4 v;
                v.x = (x + 0 >= e0 && x + 0 < e1) ? dev::ld_keep(ccur + q.x, pol) : 0.f;
                v.y = (x + 1 >= e0 && x + 1 < e1) ? dev::ld_keep(ccur + q.y, pol) : 0.f;
                v.z = (x + 2 >= e0 && x + 2 < e1) ? dev::ld_keep(ccur + q.z, pol) : 0.f;
                v.w = (x + 3 >= e0 && x + 3 < e1) ? dev::ld_keep(ccur + q.w, pol) : 0.f;
                sv4[i] = v;
            }
            __syncthreads();
            // rows with in-degree < 32: one thread each
            for (uint32_t r = r0 + tid; r < rl; r += kPRThreads) {
                const uint64_t b = a.in_off[r], e = a.in_off[r + 1];
                if (e - b < kWarpRowDegree) {
                    dev::CSum acc;
                    for (uint64_t x = b; x < e; ++x) acc.add(s_vals[x - a0]);
                    finalize_row(a, ps, r, acc.value(), cur, nxt, cnxt, res, dang);
                } else {
                    const uint32_t slot = atomicAdd(&s_nwarp_rows, 1u);
                    s_warp_rows[slot] = r;
                }
            }
            __syncthreads();
            // rows with in-degree >= 32: one warp each
            const uint32_t nwr = s_nwarp_rows;
            for (uint32_t j = warp; j < nwr; j += nwarps) {
                const uint32_t r = s_warp_rows[j];
                const uint64_t b = a.in_off[r], e = a.in_off[r + 1];
                dev::CSum acc;
                for (uint64_t x = b + lane; x < e; x += 32) acc.add(s_vals[x - a0]);
                acc = dev::warp_reduce(acc);
                if (lane == 0) finalize_row(a, ps, r, acc.value(), cur, nxt, cnxt, res, dang);
            }
            __syncthreads();
        }
    }

    const double bres = dev::block_sum(res, s_red);
    __syncthreads();
    const double bdang = dev::block_sum(dang, s_red);
    if (tid == 0) {
        atomicAdd(&a.residual[it], bres);
        atomicAdd(&a.dangling[it + 1], bdang);
        __threadfence();
        const uint32_t t = atomicAdd(&a.finished[it], 1u);
        if (t == gridDim.x - 1) {
            __threadfence();
            const double r = atomicAdd(&a.residual[it], 0.0);
            const uint32_t n_it = it + 1;
            const bool conv = r <= static_cast<double>(a.tolerance);
            a.hdr->last_residual = r;
            a.hdr->iter = n_it;
            if (conv || n_it >= a.max_iter) {
                a.hdr->done = 1;
                a.hdr->converged = conv ? 1u : 0u;
                if (a.use_cond) cudaGraphSetConditional(a.cond, 0);
            }
        }
    }
}

__global__ void pr_init_kernel(const PRArgs *__restrict__ args) {
    __shared__ double s_red[32];
    const PRArgs a = *args;
    const uint32_t V = a.V;
    const float r0_uniform = __fdiv_rn(1.0f, static_cast<float>(V));
    double dang = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
        const float r0 = a.personalized ? (v == a.source ? 1.0f : 0.0f) : r0_uniform;
        a.rank[0][v] = r0;
        const uint32_t od = a.out_deg[v];
        a.contrib[0][v] = od ? __fdiv_rn(r0, static_cast<float>(od)) : 0.0f;
        if (od == 0) dang += r0;
    }
    const double b = dev::block_sum(dang, s_red);
    if (threadIdx.x == 0 && b != 0.0) atomicAdd(&a.dangling[0], b);
}

size_t state_bytes(uint32_t max_iter) {
    return sizeof(PRHeader) + size_t(max_iter) * (2 * sizeof(uint32_t) + sizeof(double)) +
           size_t(max_iter + 1) * sizeof(double) + 64;
}

int pr_occupancy_grid() {
    static int grid = 0;
    if (grid == 0) {
        int per_sm = 0;
        HYT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pr_iterate_kernel, kPRThreads, 0));
        grid = sm_count() * std::max(per_sm, 1);
    }
    return grid;
}

struct SolveOut {
    uint32_t iterations;
    uint32_t converged;
    double residual;
};

}  // namespace

// Shared by PageRank and personalized PageRank.
static void pr_solve(GraphImpl &g, bool personalized, uint32_t source, float damping, float tolerance,
                     uint32_t max_iter, uint32_t flags, cudaStream_t s, float *ranks_out, hyt_run_stats *stats) {
    if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PULL");
    const uint64_t V = g.V;
    // Workspaces (grown on demand, kept in the handle).
    for (int i = 0; i < 2; ++i) {
        if (g.rank[i].count < V) g.rank[i].allocate(V);
        if (g.contrib[i].count < V) g.contrib[i].allocate(V);
    }
    if (g.partial.count < 2 * std::max<uint64_t>(g.num_chunks, 1)) g.partial.allocate(2 * std::max<uint64_t>(g.num_chunks, 1));
    if (g.ticket.count < std::max<uint64_t>(g.num_long, 1)) g.ticket.allocate(std::max<uint64_t>(g.num_long, 1));
    const size_t sb = state_bytes(max_iter) + sizeof(PRArgs) + 256;
    if (g.pr_state.count < sb) g.pr_state.allocate(sb);

    unsigned char *base = g.pr_state.get();
    PRArgs *d_args = reinterpret_cast<PRArgs *>(base);
    unsigned char *p = base + ((sizeof(PRArgs) + 255) & ~size_t(255));
    PRHeader *hdr = reinterpret_cast<PRHeader *>(p);
    p += sizeof(PRHeader);
    double *residual = reinterpret_cast<double *>(p);
    p += size_t(max_iter) * sizeof(double);
    double *dangling = reinterpret_cast<double *>(p);
    p += size_t(max_iter + 1) * sizeof(double);
    uint32_t *task_counter = reinterpret_cast<uint32_t *>(p);
    p += size_t(max_iter) * sizeof(uint32_t);
    uint32_t *finished = reinterpret_cast<uint32_t *>(p);
    p += size_t(max_iter) * sizeof(uint32_t);
    const size_t zero_bytes = static_cast<size_t>(p - reinterpret_cast<unsigned char *>(hdr));

    PRArgs a{};
    a.in_off = g.in_offsets.get();
    a.in_src = g.in_sources.get();
    a.out_deg = g.out_degree.get();
    a.tile_start = g.tile_start.get();
    a.long_rows = g.long_rows.get();
    a.chunk_tasks = g.chunk_tasks.get();
    for (int i = 0; i < 2; ++i) {
        a.rank[i] = g.rank[i].get();
        a.contrib[i] = g.contrib[i].get();
    }
    a.partial = reinterpret_cast<float2 *>(g.partial.get());
    a.ticket = g.ticket.get();
    a.hdr = hdr;
    a.task_counter = task_counter;
    a.finished = finished;
    a.residual = residual;
    a.dangling = dangling;
    a.num_tiles = g.num_tiles;
    a.num_chunks = static_cast<uint32_t>(g.num_chunks);
    a.V = static_cast<uint32_t>(V);
    a.damping = damping;
    a.base = personalized ? 0.0f : (1.0f - damping) / static_cast<float>(V);
    a.tolerance = tolerance;
    a.max_iter = max_iter;
    a.source = source;
    a.personalized = personalized ? 1u : 0u;
    a.use_cond = 0;

    const bool use_graph = !(flags & HYT_RUN_NO_GRAPH) && !(flags & HYT_RUN_PROFILE);
    const int grid = pr_occupancy_grid();

    EventTimer total;
    total.start(s);
    HYT_CUDA(cudaMemsetAsync(hdr, 0, zero_bytes, s));
    HYT_CUDA(cudaMemsetAsync(g.ticket.get(), 0, g.ticket.bytes(), s));

    uint32_t launches = 0, hot_launches = 0;
    double kernel_ms = 0.0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (use_graph) {
        HYT_CUDA(cudaGraphCreate(&graph, 0));
        cudaGraphConditionalHandle cond;
        HYT_CUDA(cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault));
        a.cond = cond;
        a.use_cond = 1;
    }
    HYT_CUDA(cudaMemcpyAsync(d_args, &a, sizeof(PRArgs), cudaMemcpyHostToDevice, s));
    pr_init_kernel<<<grid_for(V, 256, 148 * 8), 256, 0, s>>>(d_args);
    HYT_CUDA(cudaGetLastError());
    ++launches;

    if (use_graph) {
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = a.cond;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        HYT_CUDA(cudaGraphAddNode(&cnode, graph, nullptr, 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaKernelNodeParams kp = {};
        void *kargs[] = {&d_args};
        kp.func = reinterpret_cast<void *>(pr_iterate_kernel);
        kp.gridDim = dim3(grid);
        kp.blockDim = dim3(kPRThreads);
        kp.sharedMemBytes = 0;
        kp.kernelParams = kargs;
        cudaGraphNode_t knode;
        HYT_CUDA(cudaGraphAddKernelNode(&knode, body, nullptr, 0, &kp));
        HYT_CUDA(cudaGraphInstantiate(&exec, graph, 0));
        HYT_CUDA(cudaGraphLaunch(exec, s));
    } else {
        EventTimer kt;
        for (uint32_t i = 0; i < max_iter; ++i) {
            if (flags & HYT_RUN_PROFILE) kt.start(s);
            pr_iterate_kernel<<<grid, kPRThreads, 0, s>>>(d_args);
            HYT_CUDA(cudaGetLastError());
            ++launches;
            if (flags & HYT_RUN_PROFILE) {
                kt.stop(s);
                const double ms = kt.ms();
                uint32_t done = 0;
                HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
                HYT_CUDA(cudaStreamSynchronize(s));
                kernel_ms += ms;
                ++hot_launches;
                if (done) break;
            } else if ((i & 3) == 3) {
                uint32_t done = 0;
                HYT_CUDA(cudaMemcpyAsync(&done, &hdr->done, sizeof(done), cudaMemcpyDeviceToHost, s));
                HYT_CUDA(cudaStreamSynchronize(s));
                if (done) break;
            }
        }
    }
    PRHeader h{};
    HYT_CUDA(cudaMemcpyAsync(&h, hdr, sizeof(h), cudaMemcpyDeviceToHost, s));
    total.stop(s);
    const double total_ms = total.ms();
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (use_graph) launches += h.iter;
    if (h.iter == 0) fail(HYT_E_INTERNAL, "PageRank made no progress");
    if (ranks_out) copy_from_device(ranks_out, g.rank[h.iter & 1].get(), V * sizeof(float), s);

    if (stats) {
        stats->iterations = h.iter;
        stats->converged = h.converged;
        stats->residual = h.last_residual;
        stats->device_ms = total_ms;
        stats->kernel_ms = kernel_ms;
        stats->kernel_launches = hot_launches;
        stats->total_launches = launches;
        stats->edges_processed = uint64_t(h.iter) * g.E;
        stats->vertices_processed = uint64_t(h.iter) * V;
        // 4 B source id + 4 B gathered contribution per edge; 8 B CSC offset
        // + 4 B rank read + 4 B rank write + 4 B contribution write per vertex.
        stats->algorithmic_bytes = uint64_t(h.iter) * (8ull * g.E + 20ull * V);
    }
}

void pagerank_run(GraphImpl &g, const hyt_pagerank_params &p, float *ranks_out, hyt_run_stats *stats) {
    if (!(p.damping >= 0.0f && p.damping < 1.0f)) fail(HYT_E_INVALID, "PageRank damping_factor must be in [0, 1)");
    if (!(p.tolerance > 0.0f) || !std::isfinite(p.tolerance))
        fail(HYT_E_INVALID, "PageRank tolerance must be finite and positive");
    if (p.max_iterations == 0) fail(HYT_E_INVALID, "PageRank max_iterations must be greater than zero");
    cudaStream_t s = p.stream ? static_cast<cudaStream_t>(p.stream) : g.stream;
    pr_solve(g, false, 0, p.damping, p.tolerance, p.max_iterations, p.flags, s, ranks_out, stats);
}

void ppr_run(GraphImpl &g, const hyt_ppr_params &p, float *ranks_out, hyt_run_stats *stats) {
    if (!(p.restart > 0.0f && p.restart <= 1.0f)) fail(HYT_E_INVALID, "personalized PageRank restart must be in (0, 1]");
    if (!(p.tolerance > 0.0f) || !std::isfinite(p.tolerance))
        fail(HYT_E_INVALID, "personalized PageRank tolerance must be finite and positive");
    if (p.max_iterations == 0) fail(HYT_E_INVALID, "personalized PageRank max_iterations must be greater than zero");
    if (p.source >= g.V) fail(HYT_E_INVALID, "personalized PageRank source vertex is out of range");
    cudaStream_t s = p.stream ? static_cast<cudaStream_t>(p.stream) : g.stream;
    pr_solve(g, true, p.source, 1.0f - p.restart, p.tolerance, p.max_iterations, p.flags, s, ranks_out, stats);
}

}  // namespace hyt
