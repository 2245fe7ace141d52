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
#include <memory>
#include <mutex>
#include <unordered_map>

#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "common.cuh"
#include "scratch.cuh"
#include "solvers.cuh"

namespace hyt {
namespace {

using dev::ld_stream;
using dev::policy_evict_last;

// Read-only 32-bit gather with an L2 eviction policy (no volatile: the
// compiler may batch independent gathers).
__device__ __forceinline__ uint32_t ld_nc_keep(const uint32_t *p, uint64_t pol) {
    uint32_t v;
    asm("ld.global.nc.L2::cache_hint.b32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
    return v;
}

enum : uint32_t {
    kBadOffsets = 1u,     // offsets do not start at 0 or decrease
    kBadTerminal = 2u,    // last offset != E
    kBadColumn = 4u,      // destination >= V
    kBadOrderRange = 8u,  // vertex_order entry >= V
    kBadOrderDup = 16u,   // vertex_order entry repeated
    kBadOverflow = 32u,   // Do_max * Di_max >= 2^64
};

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// One pass over the CSR: in-degrees by atomics, out-degrees, the largest
// out-degree, and the structure checks of the reference's
// CSRGraph::validate (offsets start at 0, never decrease, end at E; every
// destination is a vertex).
__global__ void degree_pass_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ cols, uint64_t V,
                                   uint64_t E, uint32_t *__restrict__ indeg, uint64_t *__restrict__ outdeg,
                                   unsigned long long *__restrict__ maxes, uint32_t *__restrict__ bad) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint32_t b = 0;
    for (uint64_t e = tid; e < E; e += stride) {
        const uint32_t c = ld_stream(cols + e);
        if (c < V) {
            atomicAdd(indeg + c, 1u);
        } else {
            b |= kBadColumn;
        }
    }
    uint64_t mo = 0;
    for (uint64_t v = tid; v < V; v += stride) {
        const uint64_t a = off[v], z = off[v + 1];
        uint64_t d = 0;
        if (z < a) {
            b |= kBadOffsets;
        } else {
            d = z - a;
        }
        outdeg[v] = d;
        mo = max(mo, d);
    }
    if (tid == 0) {
        if (off[0] != 0) b |= kBadOffsets;
        if (off[V] != E) b |= kBadTerminal;
    }
    mo = warp_max_u64(mo);
    if ((threadIdx.x & 31) == 0 && mo) atomicMax(maxes, static_cast<unsigned long long>(mo));
    if (b) atomicOr(bad, b);
}

__global__ void max_in_degree_kernel(const uint32_t *__restrict__ indeg, uint64_t V, unsigned long long *maxes) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    uint64_t m = 0;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) m = max(m, uint64_t(indeg[v]));
    m = warp_max_u64(m);
    if ((threadIdx.x & 31) == 0 && m) atomicMax(maxes + 1, static_cast<unsigned long long>(m));
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

// Scores and ranking keys (the score's bits), ids in ascending order.  The
// denominator Do_max * Di_max is read from device memory (maxes[0..1]).
__global__ void hub_scores_kernel(const uint64_t *__restrict__ outdeg, const uint32_t *__restrict__ indeg, uint64_t V,
                                  const unsigned long long *__restrict__ maxes, double *__restrict__ scores,
                                  uint64_t *__restrict__ key, uint32_t *__restrict__ id, uint32_t *__restrict__ bad) {
    const uint64_t max_out = maxes[0], max_in = maxes[1];
    const bool overflow = max_in && max_out > ~uint64_t(0) / max_in;
    if (overflow && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(bad, kBadOverflow);
    const uint64_t denom = max_out * max_in;
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t v = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; v < V; v += stride) {
        const uint64_t num = outdeg[v] * uint64_t(indeg[v]);
        const double sc = (num && !overflow) ? extended_quotient(num, denom) : 0.0;
        if (scores) scores[v] = sc;
        key[v] = static_cast<uint64_t>(__double_as_longlong(sc));
        id[v] = static_cast<uint32_t>(v);
    }
}

__global__ void mark_kernel(const uint32_t *ids, uint64_t n, uint8_t *flag) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < n; i += stride) flag[ids[i]] = 0;
}

// Permutation check, inverse permutation (inv pre-filled with ~0: a second
// writer of the same old id is a duplicate), permuted degrees, and the
// offset checks.  ndeg[V] = 0 so an exclusive scan over V + 1 entries
// yields the new offsets.
__global__ void order_pass_kernel(const uint64_t *__restrict__ off, const uint32_t *__restrict__ order, uint64_t V,
                                  uint64_t E, uint32_t *__restrict__ inv, uint64_t *__restrict__ ndeg,
                                  uint32_t *__restrict__ bad) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    const uint64_t tid = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x;
    uint32_t b = 0;
    for (uint64_t nv = tid; nv < V; nv += stride) {
        const uint32_t old = order[nv];
        uint64_t d = 0;
        if (old >= V) {
            b |= kBadOrderRange;
        } else {
            if (atomicExch(inv + old, static_cast<uint32_t>(nv)) != 0xFFFFFFFFu) b |= kBadOrderDup;
            const uint64_t a = off[old], z = off[old + 1];
            if (z < a) {
                b |= kBadOffsets;
            } else {
                d = z - a;
            }
        }
        ndeg[nv] = d;
    }
    if (tid == 0) {
        if (off[0] != 0) b |= kBadOffsets;
        if (off[V] != E) b |= kBadTerminal;
        ndeg[V] = 0;
    }
    if (b) atomicOr(bad, b);
}

// Largest r < V with noff[r] <= e, for e < noff[V].
__device__ __forceinline__ uint64_t row_of(const uint64_t *__restrict__ noff, uint64_t V, uint64_t e) {
    uint64_t lo = 0, hi = V;  // noff[lo] <= e < noff[hi]
    while (hi - lo > 1) {
        const uint64_t mid = (lo + hi) >> 1;
        if (noff[mid] <= e) {
            lo = mid;
        } else {
            hi = mid;
        }
    }
    return lo;
}

constexpr int kPermThreads = 256;
constexpr int kPermEdges = 8;
constexpr uint64_t kTileEdges = uint64_t(kPermThreads) * kPermEdges;
constexpr uint32_t kTileRows = 2048;

// tile_row[t] = row holding the tile's first edge, for t < tiles;
// tile_row[tiles] = row holding the last edge.  Requires E > 0.
__global__ void tile_rows_kernel(const uint64_t *__restrict__ noff, uint64_t V, uint64_t E, uint64_t tiles,
                                 uint64_t *__restrict__ tile_row) {
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t t = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; t <= tiles; t += stride)
        tile_row[t] = row_of(noff, V, t < tiles ? t * kTileEdges : E - 1);
}

// New edge e of new row r copies old edge off[order[r]] + (e - noff[r]),
// destination renamed through inv, weight carried.  Tiles of 2048
// consecutive output edges; rows tile_row[t] .. tile_row[t + 1] cover the
// tile.  Their new and old starts are staged in shared memory, and each
// edge's row comes from a load-balanced search: every row start inside the
// tile marks its position, and an inclusive max-scan over the 2048
// positions hands each edge the last row starting at or before it (empty
// rows share a start with the next row and lose to its larger index).  A
// tile spanning more than 2048 rows (long runs of empty rows) searches the
// global offsets per edge instead.  Consecutive lanes take consecutive
// edges, so id / weight reads and writes are coalesced within a row; each
// thread keeps its 8 edges' loads in flight together (ids and weights, then
// the renaming gathers).
__global__ void __launch_bounds__(kPermThreads) permute_edges_kernel(
    const uint64_t *__restrict__ off, const uint32_t *__restrict__ cols, const uint32_t *__restrict__ w,
    const uint64_t *__restrict__ noff, const uint64_t *__restrict__ tile_row, const uint32_t *__restrict__ order,
    const uint32_t *__restrict__ inv, uint64_t V, uint64_t E, uint32_t *__restrict__ ncols,
    uint32_t *__restrict__ nw, uint32_t *__restrict__ bad) {
    __shared__ uint64_t s_noff[kTileRows + 1];
    __shared__ uint64_t s_base[kTileRows];
    __shared__ __align__(16) uint32_t s_row[kTileEdges];
    __shared__ uint32_t s_warp[kPermThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t b = 0;
    const uint64_t pol = policy_evict_last();
    const uint64_t tiles = (E + kTileEdges - 1) / kTileEdges;
    for (uint64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint64_t e0 = t * kTileEdges, e1 = min(e0 + kTileEdges, E);
        const uint64_t r0 = tile_row[t];
        const uint64_t rows = tile_row[t + 1] - r0 + 1;  // r0 + rows <= V
        const bool staged = rows <= kTileRows;
        if (staged) {
#pragma unroll
            for (int j = 0; j < kPermEdges; ++j) s_row[j * kPermThreads + threadIdx.x] = 0;
            for (uint64_t k = threadIdx.x; k <= rows; k += kPermThreads) {
                s_noff[k] = noff[r0 + k];
                if (k < rows) s_base[k] = off[order[r0 + k]];
            }
            __syncthreads();
            // rows k >= 1 start after e0 (row r0 holds e0); mark the ones
            // starting inside the tile
            for (uint32_t k = 1 + threadIdx.x; k < rows; k += kPermThreads) {
                const uint64_t pos = s_noff[k] - e0;
                if (pos < kTileEdges) atomicMax(s_row + pos, k);
            }
            __syncthreads();
            // inclusive max-scan; thread i owns positions [8i, 8i + 8)
            const uint4 lo4 = reinterpret_cast<const uint4 *>(s_row)[2 * threadIdx.x];
            const uint4 hi4 = reinterpret_cast<const uint4 *>(s_row)[2 * threadIdx.x + 1];
            uint32_t v[8] = {lo4.x, lo4.y, lo4.z, lo4.w, hi4.x, hi4.y, hi4.z, hi4.w};
#pragma unroll
            for (int j = 1; j < 8; ++j) v[j] = max(v[j], v[j - 1]);
            uint32_t run = v[7];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, run, o);
                if (lane >= o) run = max(run, y);
            }
            if (lane == 31) s_warp[warp] = run;
            uint32_t before = __shfl_up_sync(0xffffffffu, run, 1);
            if (lane == 0) before = 0;
            __syncthreads();
            for (int q = 0; q < warp; ++q) before = max(before, s_warp[q]);
#pragma unroll
            for (int j = 0; j < 8; ++j) v[j] = max(v[j], before);
            reinterpret_cast<uint4 *>(s_row)[2 * threadIdx.x] = make_uint4(v[0], v[1], v[2], v[3]);
            reinterpret_cast<uint4 *>(s_row)[2 * threadIdx.x + 1] = make_uint4(v[4], v[5], v[6], v[7]);
            __syncthreads();
        }
        uint64_t src[kPermEdges];
#pragma unroll
        for (int i = 0; i < kPermEdges; ++i) {
            const uint64_t e = e0 + uint64_t(i) * kPermThreads + threadIdx.x;
            src[i] = 0;
            if (e < e1) {
                if (staged) {
                    const uint32_t k = s_row[i * kPermThreads + threadIdx.x];
                    src[i] = s_base[k] + (e - s_noff[k]);
                } else {
                    const uint64_t r = row_of(noff, V, e);
                    src[i] = off[order[r]] + (e - noff[r]);
                }
            }
        }
        uint32_t c[kPermEdges], wv[kPermEdges];
#pragma unroll
        for (int i = 0; i < kPermEdges; ++i) {
            const bool live = e0 + uint64_t(i) * kPermThreads + threadIdx.x < e1;
            c[i] = live ? ld_stream(cols + src[i]) : 0u;
            wv[i] = (live && w) ? ld_stream(w + src[i]) : 0u;
        }
        uint32_t nc[kPermEdges];
#pragma unroll
        for (int i = 0; i < kPermEdges; ++i) {
            const bool live = e0 + uint64_t(i) * kPermThreads + threadIdx.x < e1;
            nc[i] = 0;
            if (live && c[i] < V) {
                nc[i] = ld_nc_keep(inv + c[i], pol);
            } else if (live) {
                b |= kBadColumn;
            }
        }
#pragma unroll
        for (int i = 0; i < kPermEdges; ++i) {
            const uint64_t e = e0 + uint64_t(i) * kPermThreads + threadIdx.x;
            if (e < e1) {
                __stcs(ncols + e, nc[i]);
                if (nw) __stcs(nw + e, wv[i]);
            }
        }
        __syncthreads();  // the next tile overwrites the staged rows
    }
    if (b) atomicOr(bad, b);
}

// Stable descending sort of (key, id) pairs on key bits [0, end_bit); the
// result ends in *keys / *ids (which may swap with the alternate buffers).
void sort_desc(uint64_t *&keys, uint64_t *keys_alt, uint32_t *&ids, uint32_t *ids_alt, uint64_t n, int end_bit,
               cudaStream_t s) {
    if (n < 2) return;
    cub::DoubleBuffer<uint64_t> kb(keys, keys_alt);
    cub::DoubleBuffer<uint32_t> vb(ids, ids_alt);
    size_t tb = 0;
    HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, end_bit, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, end_bit, s));
    keys = kb.Current();
    ids = vb.Current();
}

// out = indices i < n with flags[i] != 0, ascending (count to *count).
void select_index(const uint8_t *flags, uint32_t *out, uint64_t n, uint64_t *count, cudaStream_t s) {
    thrust::counting_iterator<uint32_t> it(0);
    size_t tb = 0;
    HYT_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flags, out, count, static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, it, flags, out, count, static_cast<int64_t>(n), s));
}

void exclusive_scan(const uint64_t *in, uint64_t *out, uint64_t n, cudaStream_t s) {
    size_t tb = 0;
    HYT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, in, out, static_cast<int64_t>(n), s));
}

// Hub count rule of the reference (its long-double arithmetic, on the host).
uint64_t hub_count_for(uint64_t V, double fraction) {
    const long double requested = static_cast<long double>(V) * static_cast<long double>(fraction);
    const long double rounded = std::round(requested);
    const long double pick = std::fabs(requested - rounded) < 1e-12L ? rounded : std::ceil(requested);
    const uint64_t n = pick <= 0.0L ? 0 : static_cast<uint64_t>(pick);
    return n < V ? n : V;
}

uint32_t read_flags(const uint32_t *bad, cudaStream_t s) {
    uint32_t h = 0;
    HYT_CUDA(cudaMemcpyAsync(&h, bad, 4, cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    return h;
}

void fail_on_csr_flags(uint32_t h) {
    if (h & kBadOffsets) fail(HYT_E_INVALID, "row offsets must start at 0 and be non-decreasing");
    if (h & kBadTerminal) fail(HYT_E_INVALID, "terminal row offset must equal the number of edges");
    if (h & kBadColumn) fail(HYT_E_INVALID, "column index contains an invalid destination vertex ID");
}

unsigned grid_sm(unsigned per_sm) { return static_cast<unsigned>(sm_count()) * per_sm; }

}  // namespace

void hub_sort(const hyt_csr &csr, double fraction, uint32_t *order_out, double *scores_out, uint64_t *hub_count,
              hyt_reorder_stats *stats) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!order_out && V) fail(HYT_E_INVALID, "vertex_order output is NULL");
    if (!std::isfinite(fraction) || fraction < 0.0 || fraction > 1.0)
        fail(HYT_E_INVALID, "HubSortOptions.hub_fraction must be finite and in [0, 1]");
    if (V > 0xFFFFFFFFull) fail(HYT_E_INVALID, "hub sorting takes graphs of < 2^32 vertices");
    if (hub_count) *hub_count = 0;
    if (V == 0) return;
    if (!csr.row_offsets || (E && !csr.column_indices)) fail(HYT_E_INVALID, "CSR arrays are NULL");
    StreamHold st;
    cudaStream_t s = st.s;
    EventTimer whole, main_k;
    whole.start(s);
    std::unique_ptr<Scratch<uint64_t>> off_h;
    std::unique_ptr<Scratch<uint32_t>> cols_h;
    const uint64_t *off = device_view(csr.row_offsets, V + 1, off_h, s);
    const uint32_t *cols = device_view(csr.column_indices, E, cols_h, s);
    Scratch<uint32_t> indeg(V, s), bad(1, s), ids(V, s), ids_alt(V, s);
    Scratch<uint64_t> outdeg(V, s), key(V, s), key_alt(V, s), rest(1, s);
    Scratch<unsigned long long> maxes(2, s);
    HYT_CUDA(cudaMemsetAsync(indeg.get(), 0, V * 4, s));
    HYT_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
    HYT_CUDA(cudaMemsetAsync(maxes.get(), 0, 16, s));
    main_k.start(s);
    degree_pass_kernel<<<grid_sm(8), 256, 0, s>>>(off, cols, V, E, indeg.get(), outdeg.get(), maxes.get(), bad.get());
    main_k.stop(s);
    max_in_degree_kernel<<<grid_for(V, 256, 148u * 8u), 256, 0, s>>>(indeg.get(), V, maxes.get());
    const bool scores_dev = scores_out && is_device_pointer(scores_out);
    std::unique_ptr<Scratch<double>> sc;
    if (scores_out && !scores_dev) sc = std::make_unique<Scratch<double>>(V, s);
    double *scores_d = scores_dev ? scores_out : (sc ? sc->get() : nullptr);
    hub_scores_kernel<<<grid_sm(8), 256, 0, s>>>(outdeg.get(), indeg.get(), V, maxes.get(), scores_d, key.get(),
                                                 ids.get(), bad.get());
    HYT_CUDA(cudaGetLastError());
    if (scores_out && !scores_dev) HYT_CUDA(cudaMemcpyAsync(scores_out, scores_d, V * 8, cudaMemcpyDeviceToHost, s));
    // scores lie in [0, 1]: their bit patterns fit in 62 bits
    uint64_t *keys = key.get();
    uint32_t *ranked = ids.get();
    sort_desc(keys, key_alt.get(), ranked, ids_alt.get(), V, 62, s);
    const uint64_t hubs = hub_count_for(V, fraction);
    // order = hubs (ranked) then the other vertices in id order
    Scratch<uint8_t> is_other(V, s);
    HYT_CUDA(cudaMemsetAsync(is_other.get(), 1, V, s));
    if (hubs) mark_kernel<<<grid_for(hubs, 256), 256, 0, s>>>(ranked, hubs, is_other.get());
    HYT_CUDA(cudaGetLastError());
    const bool order_dev = is_device_pointer(order_out);
    std::unique_ptr<Scratch<uint32_t>> ord;
    if (!order_dev) ord = std::make_unique<Scratch<uint32_t>>(V, s);
    uint32_t *order_d = order_dev ? order_out : ord->get();
    if (hubs) HYT_CUDA(cudaMemcpyAsync(order_d, ranked, hubs * 4, cudaMemcpyDeviceToDevice, s));
    select_index(is_other.get(), order_d + hubs, V, rest.get(), s);
    if (!order_dev) HYT_CUDA(cudaMemcpyAsync(order_out, order_d, V * 4, cudaMemcpyDeviceToHost, s));
    whole.stop(s);
    uint64_t h_rest = 0;
    HYT_CUDA(cudaMemcpyAsync(&h_rest, rest.get(), 8, cudaMemcpyDeviceToHost, s));
    const uint32_t h = read_flags(bad.get(), s);
    fail_on_csr_flags(h);
    if (h & kBadOverflow) fail(HYT_E_INVALID, "degree product exceeds 2^64");
    if (h_rest + hubs != V) fail(HYT_E_INTERNAL, "hub ordering lost vertices");
    if (hub_count) *hub_count = hubs;
    if (stats) {
        stats->device_ms = whole.ms();
        stats->kernel_ms = main_k.ms();
        stats->kernel_bytes = 4 * E + 16 * V;  // ids read; offsets read, out-degrees written
        // + in-degrees, scores / keys / ids written, the radix sort (12 B per
        // vertex read and written per 8-bit digit), the order and scores out
        stats->algorithmic_bytes = stats->kernel_bytes + 4 * V + 28 * V + 8 * 24 * V + 12 * V;
        stats->kernel_launches = hubs ? 4 : 3;
        stats->library_calls = 2;
    }
}

void csr_reorder(const hyt_csr &csr, const uint32_t *vertex_order, bool on_device, hyt_csr_buffers *out,
                 hyt_reorder_stats *stats, bool pooled) {
    const uint64_t V = csr.num_vertices, E = csr.num_edges;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (!out || (!vertex_order && V)) fail(HYT_E_INVALID, "NULL argument");
    std::memset(out, 0, sizeof(*out));
    if (V > 0xFFFFFFFFull) fail(HYT_E_INVALID, "reordering takes graphs of < 2^32 vertices");
    if (csr.weight_kind != HYT_WEIGHTS_NONE && csr.weight_kind != HYT_WEIGHTS_F32 && csr.weight_kind != HYT_WEIGHTS_U32)
        fail(HYT_E_INVALID, "unknown weight kind");
    if (csr.weight_kind != HYT_WEIGHTS_NONE && E && !csr.weights) fail(HYT_E_INVALID, "weights are NULL");
    if (!csr.row_offsets || (E && !csr.column_indices)) fail(HYT_E_INVALID, "CSR arrays are NULL");
    const bool weighted = csr.weight_kind != HYT_WEIGHTS_NONE && E;
    StreamHold st;
    cudaStream_t s = st.s;
    EventTimer whole, main_k;
    whole.start(s);
    std::unique_ptr<Scratch<uint64_t>> off_h;
    std::unique_ptr<Scratch<uint32_t>> cols_h, w_h, order_h;
    const uint64_t *off = device_view(csr.row_offsets, V + 1, off_h, s);
    const uint32_t *cols = device_view(csr.column_indices, E, cols_h, s);
    const uint32_t *w = weighted ? device_view(static_cast<const uint32_t *>(csr.weights), E, w_h, s) : nullptr;
    const uint32_t *order = device_view(vertex_order, V, order_h, s);
    Scratch<uint32_t> inv(V, s), bad(1, s);
    Scratch<uint64_t> ndeg(V + 1, s);
    HYT_CUDA(cudaMemsetAsync(inv.get(), 0xFF, std::max<uint64_t>(V, 1) * 4, s));
    HYT_CUDA(cudaMemsetAsync(bad.get(), 0, 4, s));
    order_pass_kernel<<<grid_sm(8), 256, 0, s>>>(off, order, V, E, inv.get(), ndeg.get(), bad.get());
    HYT_CUDA(cudaGetLastError());
    // the permutation and the offsets must be valid before any kernel
    // indexes through them
    uint32_t h = read_flags(bad.get(), s);
    if (h & kBadOrderRange)
        fail(HYT_E_INVALID, "CSRGraph::reorder_vertices: vertex_order contains an out-of-range vertex ID");
    if (h & kBadOrderDup) fail(HYT_E_INVALID, "CSRGraph::reorder_vertices: vertex_order contains duplicate vertex IDs");
    fail_on_csr_flags(h);
    auto alloc = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (on_device && pooled) {
            int dev = 0;
            HYT_CUDA(cudaGetDevice(&dev));
            HYT_CUDA(cudaMallocFromPoolAsync(&p, bytes ? bytes : 16, graph_pool(dev), cudaStreamLegacy));
            HYT_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
        } else if (on_device) {
            HYT_CUDA(cudaMalloc(&p, bytes ? bytes : 16));
        } else {
            p = std::malloc(bytes ? bytes : 16);
            if (!p) fail(HYT_E_OOM, "host allocation failed");
        }
        return p;
    };
    struct OutGuard {  // frees the outputs if a later step fails
        hyt_csr_buffers *o;
        bool pooled;
        bool armed = true;
        ~OutGuard() {
            if (!armed) return;
            if (pooled) {
                free_pooled_buffers(o);
            } else {
                hyt_csr_buffers_free(o);
            }
        }
    } guard{out, pooled && on_device};
    out->num_vertices = V;
    out->num_edges = E;
    out->on_device = on_device ? 1u : 0u;
    out->weight_kind = weighted ? csr.weight_kind : HYT_WEIGHTS_NONE;
    out->row_offsets = static_cast<uint64_t *>(alloc((V + 1) * 8));
    out->column_indices = static_cast<uint32_t *>(alloc(E * 4));
    if (weighted) out->weights = static_cast<uint32_t *>(alloc(E * 4));
    // host output: the kernels write device scratch, copied out at the end
    std::unique_ptr<Scratch<uint64_t>> noff_s;
    std::unique_ptr<Scratch<uint32_t>> ncols_s, nw_s;
    uint64_t *noff = out->row_offsets;
    uint32_t *ncols = out->column_indices, *nw = out->weights;
    if (!on_device) {
        noff_s = std::make_unique<Scratch<uint64_t>>(V + 1, s);
        ncols_s = std::make_unique<Scratch<uint32_t>>(E, s);
        noff = noff_s->get();
        ncols = ncols_s->get();
        if (weighted) {
            nw_s = std::make_unique<Scratch<uint32_t>>(E, s);
            nw = nw_s->get();
        }
    }
    exclusive_scan(ndeg.get(), noff, V + 1, s);
    const uint64_t tiles = (E + kTileEdges - 1) / kTileEdges;
    Scratch<uint64_t> tile_row(tiles + 1, s);
    if (E) tile_rows_kernel<<<grid_for(tiles + 1, 256), 256, 0, s>>>(noff, V, E, tiles, tile_row.get());
    main_k.start(s);
    if (E) {
        const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(tiles, grid_sm(5)));
        permute_edges_kernel<<<grid, kPermThreads, 0, s>>>(off, cols, w, noff, tile_row.get(), order, inv.get(), V, E,
                                                           ncols, weighted ? nw : nullptr, bad.get());
    }
    main_k.stop(s);
    HYT_CUDA(cudaGetLastError());
    if (!on_device) {
        HYT_CUDA(cudaMemcpyAsync(out->row_offsets, noff, (V + 1) * 8, cudaMemcpyDeviceToHost, s));
        if (E) HYT_CUDA(cudaMemcpyAsync(out->column_indices, ncols, E * 4, cudaMemcpyDeviceToHost, s));
        if (weighted) HYT_CUDA(cudaMemcpyAsync(out->weights, nw, E * 4, cudaMemcpyDeviceToHost, s));
    }
    whole.stop(s);
    h = read_flags(bad.get(), s);
    fail_on_csr_flags(h);
    guard.armed = false;
    if (stats) {
        stats->device_ms = whole.ms();
        stats->kernel_ms = main_k.ms();
        // ids read, renamed through inv and written; weights read and
        // written; per row a new start, an order entry and an old start
        stats->kernel_bytes = 12 * E + (weighted ? 8 * E : 0) + 20 * V;
        // + the order pass (order, offset pairs, inverse, degrees) and the scan
        stats->algorithmic_bytes = stats->kernel_bytes + 4 * V + 16 * V + 4 * V + 8 * V + 16 * V;
        stats->kernel_launches = E ? 3 : 1;
        stats->library_calls = 1;
    }
}

void free_pooled_buffers(hyt_csr_buffers *b) {
    if (!b) return;
    cudaDeviceSynchronize();
    for (void *p : {static_cast<void *>(b->row_offsets), static_cast<void *>(b->column_indices),
                    static_cast<void *>(b->weights)})
        if (p) cudaFreeAsync(p, cudaStreamLegacy);
    cudaStreamSynchronize(cudaStreamLegacy);
    std::memset(b, 0, sizeof(*b));
}

}  // namespace hyt
