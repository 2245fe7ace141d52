// Hub-vertex sorting and vertex reordering on the GPU (hyt_hub_sort,
// hyt_csr_reorder).
//
// Hub sort follows the reference's HubSorter::sort
// (src/scheduling/hub_sort.cpp:28-183):
//   H(v) = Do(v) * Di(v) / (Do_max * Di_max),
//   hub_count = round(V * fraction) when V * fraction is within 1e-12 of an
//               integer, else ceil(V * fraction), capped at V,
//   the hub_count highest scores first (ties: lower vertex id first), then
//   every other vertex in its original relative order.
// Scores equal the reference's bit for bit: its long-double quotient is
// the x86-64 extended format (64-bit significand), which the kernel
// reproduces with an exact integer long division rounded to 64 bits and then
// to 53 bits, both to nearest-even.  The ranking sorts those doubles' bit
// patterns (non-negative doubles order like their bits) with a stable
// descending radix sort over ids in ascending order, which is the
// reference's comparator.
//
// Reordering follows CSRGraph::reorder_vertices
// (src/graph/csr_graph.cpp:171-283): vertex_order[new] = old; new row
// `new` holds old row `old`'s edges in their original order, destinations
// renamed through the inverse permutation, weights carried along.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

#include "common.cuh"
#include "prims.cuh"

namespace hyt {
namespace {

enum : uint32_t { kBadOffsets = 1u, kBadTerminal = 2u, kBadColumn = 4u };

// The CSR checks of the reference's CSRGraph::validate: offsets start at 0,
// never decrease and end at E; every destination is a vertex.
__global__ void check_csr_kernel(const uint64_t *off, const uint32_t *cols, uint64_t V, uint64_t E, uint32_t *bad) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint32_t b = 0;
    for (uint64_t v = tid; v < V; v += stride)
        if (off[v + 1] < off[v]) b |= kBadOffsets;
    for (uint64_t e = tid; e < E; e += stride)
        if (cols[e] >= V) b |= kBadColumn;
    if (tid == 0) {
        if (off[0] != 0) b |= kBadOffsets;
        if (off[V] != E) b |= kBadTerminal;
    }
    if (b) atomicOr(bad, b);
}

__global__ void in_degree_count_kernel(const uint32_t *cols, uint64_t E, uint32_t *indeg) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < E; e += stride) atomicAdd(indeg + cols[e], 1u);
}

__global__ void out_degree_kernel(const uint64_t *off, uint64_t V, uint64_t *outdeg) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) outdeg[v] = off[v + 1] - off[v];
}

// n / d for 0 < n <= d < 2^64, rounded first to a 64-bit significand and
// then to a double, both to nearest-even: what x86-64 gives for
// (double)((long double)n / (long double)d).
__device__ double extended_quotient(uint64_t n, uint64_t d) {
    const int cn = __clzll(static_cast<long long>(n)), cd = __clzll(static_cast<long long>(d));
    const uint64_t a = n << cn, b = d << cd;  // both in [2^63, 2^64)
    // q = floor(a * 2^s / b) in [2^63, 2^64), s = 63 when a >= b else 64
    int s = 64;
    uint64_t q = 0, r = a;
    if (a >= b) {
        q = 1;
        r = a - b;
        s = 63;
    }
    for (int i = 0; i < s; ++i) {
        const bool carry = (r >> 63) != 0;
        r <<= 1;
        q <<= 1;
        if (carry || r >= b) {
            r -= b;
            q |= 1;
        }
    }
    int e = cd - cn - s;  // n / d = (q + r / b) * 2^e
    const uint64_t rest = b - r;
    if (r > rest || (r == rest && (q & 1))) {
        if (++q == 0) {
            q = uint64_t(1) << 63;
            ++e;
        }
    }
    const uint64_t low = q & 0x7FF;  // drop 11 bits: 64 -> 53
    uint64_t m = q >> 11;
    e += 11;
    if (low > 0x400 || (low == 0x400 && (m & 1))) {
        if (++m == (uint64_t(1) << 53)) {
            m >>= 1;
            ++e;
        }
    }
    // m * 2^e with m in [2^52, 2^53); e + 52 lies in [-64, 0]
    const uint64_t bits = (uint64_t(e + 52 + 1023) << 52) | (m & ((uint64_t(1) << 52) - 1));
    return __longlong_as_double(static_cast<long long>(bits));
}

// Scores and ranking keys (the score's bits), ids in ascending order.
__global__ void hub_scores_kernel(const uint64_t *outdeg, const uint32_t *indeg, uint64_t V, uint64_t denom,
                                  double *scores, uint64_t *key, uint32_t *id) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) {
        const uint64_t num = outdeg[v] * uint64_t(indeg[v]);
        const double sc = num ? extended_quotient(num, denom) : 0.0;
        if (scores) scores[v] = sc;
        key[v] = static_cast<uint64_t>(__double_as_longlong(sc));
        id[v] = static_cast<uint32_t>(v);
    }
}

__global__ void mark_kernel(const uint32_t *ids, uint64_t n, uint8_t *flag) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) flag[ids[i]] = 0;
}

// Permutation check and inverse: seen[old] counts occurrences.
__global__ void inverse_kernel(const uint32_t *order, uint64_t V, uint32_t *inv, uint32_t *seen, uint32_t *bad) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t nv = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; nv < V; nv += stride) {
        const uint32_t old = order[nv];
        if (old >= V) {
            atomicOr(bad, 1u);
            continue;
        }
        if (atomicAdd(seen + old, 1u) != 0) atomicOr(bad, 2u);
        inv[old] = static_cast<uint32_t>(nv);
    }
}

__global__ void new_degree_kernel(const uint64_t *off, const uint32_t *order, uint64_t V, uint64_t *ndeg) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t nv = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; nv < V; nv += stride) {
        const uint32_t old = order[nv];
        ndeg[nv] = off[old + 1] - off[old];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) ndeg[V] = 0;
}

// One thread per output edge: its new row by binary search over the new
// offsets, then the matching edge of the old row.
__global__ void permute_edges_kernel(const uint64_t *off, const uint32_t *cols, const uint32_t *w,
                                     const uint64_t *noff, const uint32_t *order, const uint32_t *inv, uint64_t V,
                                     uint64_t E, uint32_t *ncols, uint32_t *nw) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t e = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; e < E; e += stride) {
        uint64_t lo = 0, hi = V;  // noff[lo] <= e < noff[hi]
        while (hi - lo > 1) {
            const uint64_t mid = (lo + hi) >> 1;
            if (noff[mid] <= e) {
                lo = mid;
            } else {
                hi = mid;
            }
        }
        const uint64_t src = off[order[lo]] + (e - noff[lo]);
        ncols[e] = inv[cols[src]];
        if (nw) nw[e] = w[src];
    }
}

// Device copy of a host-or-device array (owned copy when on the host).
template <class T>
const T *device_view(const T *p, uint64_t n, DeviceArray<T> &hold, cudaStream_t s) {
    if (!p || n == 0 || is_device_pointer(p)) return p;
    hold.allocate(n);
    HYT_CUDA(cudaMemcpyAsync(hold.get(), p, n * sizeof(T), cudaMemcpyHostToDevice, s));
    return hold.get();
}

// Hub count rule of the reference (its long-double arithmetic, on the host).
uint64_t hub_count_for(uint64_t V, double fraction) {
    const long double requested = static_cast<long double>(V) * static_cast<long double>(fraction);
    const long double rounded = std::round(requested);
    const long double pick = std::fabs(requested - rounded) < 1e-12L ? rounded : std::ceil(requested);
    const uint64_t n = pick <= 0.0L ? 0 : static_cast<uint64_t>(pick);
    return n < V ? n : V;
}

// Rejects a malformed CSR before any kernel indexes through it.
void check_csr(const uint64_t *off, const uint32_t *cols, uint64_t V, uint64_t E, cudaStream_t s) {
    DeviceArray<uint32_t> bad(1);
    HYT_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
    check_csr_kernel<<<grid_for(std::max(V, E), 256), 256, 0, s>>>(off, cols, V, E, bad.get());
    HYT_CUDA(cudaGetLastError());
    uint32_t h = 0;
    HYT_CUDA(cudaMemcpyAsync(&h, bad.get(), 4, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (h & kBadOffsets) fail(HYT_E_INVALID, "row offsets must start at 0 and be non-decreasing");
    if (h & kBadTerminal) fail(HYT_E_INVALID, "terminal row offset must equal the number of edges");
    if (h & kBadColumn) fail(HYT_E_INVALID, "column index contains an invalid destination vertex ID");
}

struct StreamHold {
    cudaStream_t s = nullptr;
    StreamHold() { HYT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~StreamHold() { cudaStreamDestroy(s); }
};

}  // namespace

void hub_sort(const hyt_csr &csr, double fraction, uint32_t *order_out, double *scores_out, uint64_t *hub_count) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (!order_out) fail(HYT_E_INVALID, "vertex_order output is NULL");
    if (!std::isfinite(fraction) || fraction < 0.0 || fraction > 1.0)
        fail(HYT_E_INVALID, "HubSortOptions.hub_fraction must be finite and in [0, 1]");
    if (V > 0xFFFFFFFFull) fail(HYT_E_INVALID, "hub sorting takes graphs of < 2^32 vertices");
    if (hub_count) *hub_count = 0;
    if (V == 0) return;
    if (!csr.row_offsets || (E && !csr.column_indices)) fail(HYT_E_INVALID, "CSR arrays are NULL");
    StreamHold st;
    cudaStream_t s = st.s;
    DeviceArray<uint64_t> off_h;
    DeviceArray<uint32_t> cols_h;
    const uint64_t *off = device_view(csr.row_offsets, V + 1, off_h, s);
    const uint32_t *cols = device_view(csr.column_indices, E, cols_h, s);
    check_csr(off, cols, V, E, s);
    DeviceArray<uint32_t> indeg(V);
    DeviceArray<uint64_t> outdeg(V);
    HYT_CUDA(cudaMemsetAsync(indeg.get(), 0, V * 4, s));
    if (E) in_degree_count_kernel<<<grid_for(E, 256), 256, 0, s>>>(cols, E, indeg.get());
    out_degree_kernel<<<grid_for(V, 256), 256, 0, s>>>(off, V, outdeg.get());
    HYT_CUDA(cudaGetLastError());
    const uint64_t max_out = prims::reduce_max_u64(outdeg.get(), V, s);
    const uint64_t max_in = prims::reduce_max_u32(indeg.get(), V, s);
    if (max_in && max_out > ~uint64_t(0) / max_in) fail(HYT_E_INVALID, "degree product exceeds 2^64");
    // edgeless graph: every score is zero and the stable sort keeps id order
    DeviceArray<double> sc(scores_out ? V : 1);
    DeviceArray<uint64_t> key(V);
    DeviceArray<uint32_t> ids(V);
    hub_scores_kernel<<<grid_for(V, 256), 256, 0, s>>>(outdeg.get(), indeg.get(), V, max_out * max_in,
                                                      scores_out ? sc.get() : nullptr, key.get(), ids.get());
    HYT_CUDA(cudaGetLastError());
    if (scores_out) HYT_CUDA(cudaMemcpyAsync(scores_out, sc.get(), V * sizeof(double), cudaMemcpyDefault, s));
    prims::sort_pairs_desc_u64(key.get(), ids.get(), V, s);
    const uint64_t hubs = hub_count_for(V, fraction);
    // order = hubs (ranked) then the other vertices in id order
    DeviceArray<uint8_t> is_other(V);
    HYT_CUDA(cudaMemsetAsync(is_other.get(), 1, V, s));
    if (hubs) mark_kernel<<<grid_for(hubs, 256), 256, 0, s>>>(ids.get(), hubs, is_other.get());
    HYT_CUDA(cudaGetLastError());
    DeviceArray<uint32_t> order(V);
    if (hubs) HYT_CUDA(cudaMemcpyAsync(order.get(), ids.get(), hubs * 4, cudaMemcpyDeviceToDevice, s));
    const size_t rest = prims::select_flagged_index(is_other.get(), order.get() + hubs, V, s);
    if (rest + hubs != V) fail(HYT_E_INTERNAL, "hub ordering lost vertices");
    HYT_CUDA(cudaMemcpyAsync(order_out, order.get(), V * 4, cudaMemcpyDefault, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (hub_count) *hub_count = hubs;
}

void csr_reorder(const hyt_csr &csr, const uint32_t *vertex_order, bool on_device, hyt_csr_buffers *out) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (!out || !vertex_order) fail(HYT_E_INVALID, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    if (V > 0xFFFFFFFFull) fail(HYT_E_INVALID, "reordering takes graphs of < 2^32 vertices");
    if (csr.weight_kind == HYT_WEIGHTS_F32 || csr.weight_kind == HYT_WEIGHTS_U32) {
        if (!csr.weights && E) fail(HYT_E_INVALID, "weights are NULL");
    }
    const bool weighted = csr.weight_kind != HYT_WEIGHTS_NONE && E;
    StreamHold st;
    cudaStream_t s = st.s;
    DeviceArray<uint64_t> off_h;
    DeviceArray<uint32_t> cols_h, w_h, order_h;
    const uint64_t *off = device_view(csr.row_offsets, V + 1, off_h, s);
    const uint32_t *cols = device_view(csr.column_indices, E, cols_h, s);
    const uint32_t *w = weighted ? device_view(static_cast<const uint32_t *>(csr.weights), E, w_h, s) : nullptr;
    const uint32_t *order = device_view(vertex_order, V, order_h, s);
    if (!off || (E && !cols)) fail(HYT_E_INVALID, "CSR arrays are NULL");
    check_csr(off, cols, V, E, s);
    DeviceArray<uint32_t> inv(V ? V : 1), seen(V ? V : 1), bad(1);
    HYT_CUDA(cudaMemsetAsync(seen.get(), 0, (V ? V : 1) * 4, s));
    HYT_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
    if (V) inverse_kernel<<<grid_for(V, 256), 256, 0, s>>>(order, V, inv.get(), seen.get(), bad.get());
    HYT_CUDA(cudaGetLastError());
    uint32_t h_bad = 0;
    HYT_CUDA(cudaMemcpyAsync(&h_bad, bad.get(), 4, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    if (h_bad & 1u) fail(HYT_E_INVALID, "CSRGraph::reorder_vertices: vertex_order contains an out-of-range vertex ID");
    if (h_bad & 2u) fail(HYT_E_INVALID, "CSRGraph::reorder_vertices: vertex_order contains duplicate vertex IDs");
    // new offsets = exclusive scan of the permuted degrees
    DeviceArray<uint64_t> ndeg(V + 1), noff(V + 1);
    new_degree_kernel<<<grid_for(V + 1, 256), 256, 0, s>>>(off, order, V, ndeg.get());
    HYT_CUDA(cudaGetLastError());
    prims::exclusive_scan_u64(ndeg.get(), noff.get(), V + 1, s);
    DeviceArray<uint32_t> ncols(E ? E : 1), nw(weighted ? E : 1);
    if (E)
        permute_edges_kernel<<<grid_for(E, 256), 256, 0, s>>>(off, cols, w, noff.get(), order, inv.get(), V, E,
                                                             ncols.get(), weighted ? nw.get() : nullptr);
    HYT_CUDA(cudaGetLastError());
    HYT_CUDA(cudaStreamSynchronize(s));
    out->num_vertices = V;
    out->num_edges = E;
    out->on_device = on_device ? 1u : 0u;
    auto alloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (on_device) {
            HYT_CUDA(cudaMalloc(&p, bytes ? bytes : 16));
        } else {
            p = std::malloc(bytes ? bytes : 16);
            if (!p) fail(HYT_E_OOM, "host allocation failed");
        }
        return p;
    };
    out->row_offsets = static_cast<uint64_t *>(alloc((V + 1) * 8));
    out->column_indices = static_cast<uint32_t *>(alloc(E * 4));
    if (weighted) out->weights = static_cast<uint32_t *>(alloc(E * 4));
    HYT_CUDA(cudaMemcpyAsync(out->row_offsets, noff.get(), (V + 1) * 8, cudaMemcpyDefault, s));
    if (E) HYT_CUDA(cudaMemcpyAsync(out->column_indices, ncols.get(), E * 4, cudaMemcpyDefault, s));
    if (weighted) HYT_CUDA(cudaMemcpyAsync(out->weights, nw.get(), E * 4, cudaMemcpyDefault, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hyt
