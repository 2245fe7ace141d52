// Contribution-driven scheduling on the GPU: hyt_pagerank_contributions,
// hyt_sssp_contributions, hyt_contribution_schedule,
// hyt_partition_contributions.
//
// Contributions follow the reference's definitions
// (src/algorithms/pagerank.cpp:165-241, src/algorithms/sssp.cpp:236-290):
//   PageRank: |next(v) - current(v)| of one synchronous pull step,
//     next(v) = (1 - d)/n + d * dangling / n + d * sum_{u->v} current(u)/deg(u);
//     here the sums run in FP64 (one warp per row, a fixed-order warp
//     tree; dangling mass by per-block partials summed in a fixed order), so
//     the values are deterministic and agree with the reference's FP32 to
//     within its rounding;
//   SSSP: current - candidate when both are finite and the improvement
//     exceeds the tolerance, 1 when an unreachable vertex becomes
//     reachable, else 0 — the same FP32 operations, bit for bit.
// The schedule follows ContributionScheduler::schedule
// (src/scheduling/contribution_scheduler.cpp:23-121): items by descending
// contribution, ties by lower item index (deterministic tie-break; or input
// order otherwise), computed as two stable radix sorts (item index, then
// contribution), with the plan metrics (reordered, zero, redundant,
// log2(n) overhead).
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/cub.cuh>

#include "common.cuh"
#include "graph.cuh"
#include "scratch.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

constexpr int kPartBlocks = 1024;

// x[u] = current(u) / deg(u) in FP64 (0 for a dangling vertex), and the
// per-block partial sums of the dangling ranks.
__global__ void source_shares_kernel(const uint32_t *__restrict__ deg, const float *__restrict__ rank, uint64_t V,
                                     double *__restrict__ x, double *__restrict__ partial) {
    __shared__ double warp_sum[8];
    double acc = 0.0;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += uint64_t(gridDim.x) * blockDim.x) {
        const uint32_t d = deg[v];
        const double r = rank[v];
        x[v] = d ? r / double(d) : 0.0;
        if (d == 0) acc += r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; ++w) s += warp_sum[w];
        partial[blockIdx.x] = s;
    }
}

__device__ __forceinline__ double row_sum(const uint32_t *__restrict__ in_src, const uint32_t *__restrict__ hot_vertex,
                                          const double *__restrict__ x, uint64_t b, uint64_t e, int lane) {
    double acc = 0.0;
    for (uint64_t i = b + lane; i < e; i += 32) {
        uint32_t u = in_src[i];
        if (u & kHotTag) u = hot_vertex[u & ~kHotTag];
        acc += x[u];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    return acc;
}

// (1 - d)/n + d * dangling / n from the per-block dangling partials, summed
// by the block's first warp in a fixed order (lane l: partials l, l + 32,
// ...; then a shuffle tree), so no thread waits on one load per partial.
// Called by the first 32 threads; the result is in all of them.
__device__ __forceinline__ double base_share(const double *__restrict__ partial, int parts, uint64_t V, double d,
                                             int lane) {
    double dm = 0.0;
    for (int i = lane; i < parts; i += 32) dm += partial[i];
    dm = dev::warp_sum(dm);
    return (1.0 - d) / double(V) + d * dm / double(V);
}

// One warp per row below the long-row threshold (a fixed-order warp tree).
__global__ void pagerank_contrib_kernel(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_src,
                                        const uint32_t *__restrict__ hot_vertex, const double *__restrict__ x,
                                        const float *__restrict__ rank, uint64_t V, uint64_t long_from, double damping,
                                        const double *__restrict__ partial, int parts, double *__restrict__ out) {
    __shared__ double s_share;
    if (threadIdx.x < 32) {
        const double sh = base_share(partial, parts, V, damping, threadIdx.x);
        if (threadIdx.x == 0) s_share = sh;
    }
    __syncthreads();
    const double share = s_share;
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t v = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5; v < V; v += warps) {
        const uint64_t b = in_off[v], e = in_off[v + 1];
        if (e - b >= long_from) continue;  // summed by the chunk kernels
        const double acc = row_sum(in_src, hot_vertex, x, b, e, lane);
        if (lane == 0) out[v] = fabs(share + damping * acc - double(rank[v]));
    }
}

// One warp per chunk of a long row: its partial sum.
__global__ void contrib_chunks_kernel(const uint64_t *__restrict__ in_off, const uint32_t *__restrict__ in_src,
                                      const uint32_t *__restrict__ hot_vertex, const double *__restrict__ x,
                                      const LongRow *__restrict__ long_rows, const uint2 *__restrict__ tasks,
                                      uint64_t num_tasks, double *__restrict__ chunk_sum) {
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t t = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5; t < num_tasks; t += warps) {
        const uint2 task = tasks[t];
        const LongRow lr = long_rows[task.x];
        const uint64_t b = in_off[lr.row] + uint64_t(task.y) * kLongChunk;
        const uint64_t e = min(b + kLongChunk, in_off[lr.row + 1]);
        const double acc = row_sum(in_src, hot_vertex, x, b, e, lane);
        if (lane == 0) chunk_sum[lr.first_chunk + task.y] = acc;
    }
}

// One warp per long row: its chunks' partial sums in a fixed order.
__global__ void contrib_long_rows_kernel(const LongRow *__restrict__ long_rows, uint64_t num_long,
                                         const double *__restrict__ chunk_sum, const float *__restrict__ rank,
                                         uint64_t V, double damping, const double *__restrict__ partial, int parts,
                                         double *__restrict__ out) {
    __shared__ double s_share;
    if (threadIdx.x < 32) {
        const double sh = base_share(partial, parts, V, damping, threadIdx.x);
        if (threadIdx.x == 0) s_share = sh;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const uint64_t warps = uint64_t(gridDim.x) * (blockDim.x >> 5);
    for (uint64_t i = (blockIdx.x * uint64_t(blockDim.x) + threadIdx.x) >> 5; i < num_long; i += warps) {
        const LongRow lr = long_rows[i];
        double acc = 0.0;
        for (uint32_t c = lane; c < lr.num_chunks; c += 32) acc += chunk_sum[lr.first_chunk + c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) out[lr.row] = fabs(s_share + damping * acc - double(rank[lr.row]));
    }
}

__global__ void sssp_contrib_kernel(const float *__restrict__ cur, const float *__restrict__ cand, uint64_t n,
                                    float tol, double *__restrict__ out) {
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < n; v += uint64_t(gridDim.x) * blockDim.x) {
        const float c = cur[v], d = cand[v];
        double r = 0.0;
        if (isfinite(c) && isfinite(d)) {
            const float improvement = __fsub_rn(c, d);
            if (improvement > tol) r = double(improvement);
        } else if (!isfinite(c) && isfinite(d)) {
            r = 1.0;
        }
        out[v] = r;
    }
}

// Order-preserving unsigned image of a finite double (-0 and +0 equal).
__device__ __forceinline__ uint64_t double_key(double c) {
    uint64_t b = static_cast<uint64_t>(__double_as_longlong(c == 0.0 ? 0.0 : c));
    return (b >> 63) ? ~b : (b | (uint64_t(1) << 63));
}

__global__ void schedule_prep_kernel(const double *__restrict__ c, uint64_t n, double eps, uint64_t *__restrict__ pos,
                                     unsigned long long *__restrict__ counts) {
    unsigned long long zero = 0, nonfinite = 0;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x) {
        pos[i] = i;
        const double x = c[i];
        if (!isfinite(x)) ++nonfinite;
        if (fabs(x) <= eps) ++zero;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        zero += __shfl_xor_sync(0xffffffffu, zero, o);
        nonfinite += __shfl_xor_sync(0xffffffffu, nonfinite, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (zero) atomicAdd(counts, zero);
        if (nonfinite) atomicAdd(counts + 1, nonfinite);
    }
}

__global__ void contribution_keys_kernel(const double *__restrict__ c, const uint64_t *__restrict__ pos, uint64_t n,
                                         uint64_t *__restrict__ key) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        key[i] = double_key(c[pos[i]]);
}

// ordered[p] = item[order[p]]; counts[2] += moved positions.
__global__ void schedule_emit_kernel(const uint64_t *__restrict__ item, const uint64_t *__restrict__ order, uint64_t n,
                                     uint64_t *__restrict__ ordered, unsigned long long *__restrict__ counts) {
    unsigned long long moved = 0;
    for (uint64_t p = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; p < n; p += uint64_t(gridDim.x) * blockDim.x) {
        const uint64_t o = order[p];
        ordered[p] = item[o];
        moved += o != p;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) moved += __shfl_xor_sync(0xffffffffu, moved, o);
    if ((threadIdx.x & 31) == 0 && moved) atomicAdd(counts + 2, moved);
}

// counts[3] += adjacent equal item indices in the sorted copy.
__global__ void duplicates_kernel(const uint64_t *__restrict__ sorted, uint64_t n, unsigned long long *counts) {
    unsigned long long dup = 0;
    for (uint64_t i = 1 + blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += uint64_t(gridDim.x) * blockDim.x)
        dup += sorted[i] == sorted[i - 1];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dup += __shfl_xor_sync(0xffffffffu, dup, o);
    if ((threadIdx.x & 31) == 0 && dup) atomicAdd(counts + 3, dup);
}

unsigned grid_sm(unsigned per_sm) { return static_cast<unsigned>(sm_count()) * per_sm; }

// Stable radix sort of (key, value) pairs on key bits [0, bits).
template <class K, class V>
void sort_pairs(K *&keys, K *keys_alt, V *&vals, V *vals_alt, uint64_t n, bool descending, cudaStream_t s,
                int bits = int(sizeof(K) * 8)) {
    if (n < 2) return;
    cub::DoubleBuffer<K> kb(keys, keys_alt);
    cub::DoubleBuffer<V> vb(vals, vals_alt);
    size_t tb = 0;
    if (descending) {
        HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, bits, s));
    } else {
        HYT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, bits, s));
    }
    Scratch<uint8_t> tmp(tb, s);
    if (descending) {
        HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, bits, s));
    } else {
        HYT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, bits, s));
    }
    keys = kb.Current();
    vals = vb.Current();
}

}  // namespace

void pagerank_contributions(GraphImpl &g, const float *ranks, float damping, double *out, double *device_ms) {
    graph_require_caller_order(g, "hyt_pagerank_contributions");
    if (!(g.flags & HYT_GRAPH_PULL)) fail(HYT_E_INVALID, "graph was created without HYT_GRAPH_PULL");
    if (!ranks || !out) fail(HYT_E_INVALID, "NULL argument");
    if (!(damping >= 0.0f && damping < 1.0f)) fail(HYT_E_INVALID, "PageRank damping_factor must be in [0, 1)");
    const uint64_t V = g.V;
    if (V == 0) fail(HYT_E_INVALID, "PageRank requires at least one vertex");
    HYT_CUDA(cudaSetDevice(g.device));
    cudaStream_t s = g.stream;
    std::unique_ptr<Scratch<float>> rh;
    const float *r = device_view(ranks, V, rh, s);
    const bool out_dev = is_device_pointer(out);
    std::unique_ptr<Scratch<double>> oh;
    double *o = out;
    if (!out_dev) {
        oh = std::make_unique<Scratch<double>>(V, s);
        o = oh->get();
    }
    Scratch<double> partial(kPartBlocks, s), x(V, s);
    const uint64_t chunks = g.num_long ? g.num_chunks : 0;
    Scratch<double> chunk_sum(chunks ? chunks : 1, s);
    // a row is long (chunked) when its in-degree >= tile_cost
    const uint64_t long_from = g.num_long ? g.tile_cost : ~uint64_t(0);
    EventTimer t;
    t.start(s);
    source_shares_kernel<<<kPartBlocks, 256, 0, s>>>(g.out_degree.get(), r, V, x.get(), partial.get());
    pagerank_contrib_kernel<<<grid_sm(8), 256, 0, s>>>(g.in_offsets.get(), g.in_sources.get(), g.hot_vertex.get(),
                                                       x.get(), r, V, long_from, double(damping), partial.get(),
                                                       kPartBlocks, o);
    if (chunks) {
        contrib_chunks_kernel<<<grid_sm(8), 256, 0, s>>>(g.in_offsets.get(), g.in_sources.get(), g.hot_vertex.get(),
                                                         x.get(), g.long_rows.get(), g.chunk_tasks.get(), chunks,
                                                         chunk_sum.get());
        contrib_long_rows_kernel<<<grid_for(g.num_long * 32, 256), 256, 0, s>>>(
            g.long_rows.get(), g.num_long, chunk_sum.get(), r, V, double(damping), partial.get(), kPartBlocks, o);
    }
    HYT_CUDA(cudaGetLastError());
    t.stop(s);
    if (!out_dev) HYT_CUDA(cudaMemcpyAsync(out, o, V * 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (device_ms) *device_ms = t.ms();
}

void sssp_contributions(const float *cur, const float *cand, uint64_t n, float tol, double *out) {
    if (n && (!cur || !cand || !out)) fail(HYT_E_INVALID, "NULL argument");
    if (!(tol >= 0.0f) || !std::isfinite(tol))
        fail(HYT_E_INVALID, "SSSP contribution tolerance must be finite and non-negative");
    if (n == 0) return;
    StreamHold st;
    cudaStream_t s = st.s;
    std::unique_ptr<Scratch<float>> ch, dh;
    const float *c = device_view(cur, n, ch, s);
    const float *d = device_view(cand, n, dh, s);
    const bool out_dev = is_device_pointer(out);
    std::unique_ptr<Scratch<double>> oh;
    double *o = out;
    if (!out_dev) {
        oh = std::make_unique<Scratch<double>>(n, s);
        o = oh->get();
    }
    sssp_contrib_kernel<<<grid_for(n, 256), 256, 0, s>>>(c, d, n, tol, o);
    HYT_CUDA(cudaGetLastError());
    if (!out_dev) HYT_CUDA(cudaMemcpyAsync(out, o, n * 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void contribution_schedule(const uint64_t *item, const double *contribution, uint64_t n, bool deterministic,
                           double eps, uint64_t *ordered, hyt_contribution_metrics *m) {
    if (!m) fail(HYT_E_INVALID, "metrics is NULL");
    std::memset(m, 0, sizeof(*m));
    if (n && (!item || !contribution || !ordered)) fail(HYT_E_INVALID, "NULL argument");
    m->input_item_count = n;
    m->scheduled_item_count = n;
    if (n == 0) return;
    StreamHold st;
    cudaStream_t s = st.s;
    std::unique_ptr<Scratch<uint64_t>> ih;
    std::unique_ptr<Scratch<double>> chold;
    const uint64_t *it = device_view(item, n, ih, s);
    const double *c = device_view(contribution, n, chold, s);
    Scratch<uint64_t> pos(n, s), pos_alt(n, s), key(n, s), key_alt(n, s), out_d(n, s);
    Scratch<unsigned long long> counts(4, s);
    HYT_CUDA(cudaMemsetAsync(counts.get(), 0, 32, s));
    schedule_prep_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(c, n, eps, pos.get(), counts.get());
    HYT_CUDA(cudaGetLastError());
    // item sorts run on the bits the largest item index needs
    int item_bits = 1;
    {
        Scratch<uint64_t> mx(1, s);
        size_t tb = 0;
        HYT_CUDA(cub::DeviceReduce::Max(nullptr, tb, it, mx.get(), static_cast<int64_t>(n), s));
        Scratch<uint8_t> tmp(tb, s);
        HYT_CUDA(cub::DeviceReduce::Max(tmp.get(), tb, it, mx.get(), static_cast<int64_t>(n), s));
        uint64_t h = 0;
        HYT_CUDA(cudaMemcpyAsync(&h, mx.get(), 8, cudaMemcpyDeviceToHost, s));
        HYT_CUDA(cudaStreamSynchronize(s));
        item_bits = h ? 64 - __builtin_clzll(h) : 1;
    }
    // redundant work: equal neighbours among the sorted item indices
    HYT_CUDA(cudaMemcpyAsync(key.get(), it, n * 8, cudaMemcpyDeviceToDevice, s));
    uint64_t *vp = pos.get();
    {
        uint64_t *k = key.get();
        uint64_t *k_alt = key_alt.get();
        size_t tb = 0;
        cub::DoubleBuffer<uint64_t> kb(k, k_alt);
        HYT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, kb, static_cast<int64_t>(n), 0, item_bits, s));
        Scratch<uint8_t> tmp(tb, s);
        HYT_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(), tb, kb, static_cast<int64_t>(n), 0, item_bits, s));
        duplicates_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(kb.Current(), n, counts.get());
        HYT_CUDA(cudaGetLastError());
    }
    // the order: positions by item index (stable), then by descending
    // contribution (stable), or by contribution alone
    if (deterministic) {
        HYT_CUDA(cudaMemcpyAsync(key.get(), it, n * 8, cudaMemcpyDeviceToDevice, s));
        uint64_t *kp = key.get();
        sort_pairs(kp, key_alt.get(), vp, pos_alt.get(), n, false, s, item_bits);
    }
    uint64_t *ck = key.get(), *ck_alt = key_alt.get();
    uint64_t *vp_alt = vp == pos.get() ? pos_alt.get() : pos.get();
    contribution_keys_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(c, vp, n, ck);
    HYT_CUDA(cudaGetLastError());
    sort_pairs(ck, ck_alt, vp, vp_alt, n, true, s);
    const bool ordered_dev = is_device_pointer(ordered);
    uint64_t *od = ordered_dev ? ordered : out_d.get();
    schedule_emit_kernel<<<grid_for(n, 256, 148u * 8u), 256, 0, s>>>(it, vp, n, od, counts.get());
    HYT_CUDA(cudaGetLastError());
    if (!ordered_dev) HYT_CUDA(cudaMemcpyAsync(ordered, od, n * 8, cudaMemcpyDeviceToHost, s));
    unsigned long long h[4] = {};
    HYT_CUDA(cudaMemcpyAsync(h, counts.get(), 32, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (h[1]) fail(HYT_E_INVALID, "contribution priority must be finite");
    m->zero_contribution_count = h[0];
    m->reordered_item_count = h[2];
    m->redundant_work_count = h[3];
    m->scheduling_overhead = std::log2(static_cast<double>(n));
}

void partition_contributions(const double *contrib, uint64_t V, const uint64_t *bounds, uint64_t parts, double *out) {
    if (parts && (!bounds || !out)) fail(HYT_E_INVALID, "NULL argument");
    if (V && !contrib) fail(HYT_E_INVALID, "NULL argument");
    if (parts == 0) return;
    StreamHold st;
    cudaStream_t s = st.s;
    std::unique_ptr<Scratch<double>> ch;
    std::unique_ptr<Scratch<uint64_t>> bh;
    std::vector<uint64_t> hb(parts + 1);
    HYT_CUDA(cudaMemcpyAsync(hb.data(), bounds, (parts + 1) * 8, cudaMemcpyDefault, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    for (uint64_t i = 0; i < parts; ++i)
        if (hb[i] > hb[i + 1] || hb[i + 1] > V) fail(HYT_E_INVALID, "partition bounds must be non-decreasing and <= V");
    const double *c = device_view(contrib, V, ch, s);
    const uint64_t *b = device_view(bounds, parts + 1, bh, s);
    const bool out_dev = is_device_pointer(out);
    std::unique_ptr<Scratch<double>> oh;
    double *o = out;
    if (!out_dev) {
        oh = std::make_unique<Scratch<double>>(parts, s);
        o = oh->get();
    }
    size_t tb = 0;
    HYT_CUDA(cub::DeviceSegmentedReduce::Sum(nullptr, tb, c, o, static_cast<int64_t>(parts), b, b + 1, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceSegmentedReduce::Sum(tmp.get(), tb, c, o, static_cast<int64_t>(parts), b, b + 1, s));
    if (!out_dev) HYT_CUDA(cudaMemcpyAsync(out, o, parts * 8, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hyt
