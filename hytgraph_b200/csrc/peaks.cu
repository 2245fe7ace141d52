// Measured bandwidth peaks of one GPU: the denominators a caller needs for
// the path's rooflines (HBM for in-HBM solves, the host link for
// out-of-HBM solves).  Every figure is the best of several timed
// repetitions with CUDA events on a private stream.
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "graph.cuh"
#include "scratch.cuh"

namespace hyt {
namespace {

// Reads `n16` 16-byte words of mapped host memory (the zero-copy path of
// out-of-HBM solves); the xor keeps the loads alive.
__global__ void peaks_zc_read_kernel(const uint4 *p, uint64_t n16, unsigned long long *sink) {
    uint32_t acc = 0;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n16; i += uint64_t(gridDim.x) * blockDim.x) {
        const uint4 v = __ldcv(p + i);
        acc ^= v.x ^ v.y ^ v.z ^ v.w;
    }
    if (acc == 0x9E3779B9u) atomicAdd(sink, 1ull);
}

template <class F>
double best_ms(cudaStream_t s, int reps, F &&body) {
    EventTimer t;
    double best = 1e30;
    for (int r = 0; r < reps; ++r) {
        t.start(s);
        body();
        t.stop(s);
        best = std::min(best, t.ms());
    }
    return best;
}

}  // namespace

void measure_peaks(int device, uint64_t copy_bytes, hyt_peaks *out) {
    std::memset(out, 0, sizeof(*out));
    HYT_CUDA(cudaSetDevice(device));
    if (copy_bytes == 0) copy_bytes = uint64_t(1) << 30;
    copy_bytes = std::max<uint64_t>(copy_bytes & ~uint64_t(15), 1 << 20);
    const uint64_t link_bytes = std::min<uint64_t>(copy_bytes, uint64_t(256) << 20);

    int v = 0;
    HYT_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device));
    out->sm_count = static_cast<uint32_t>(v);
    HYT_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrL2CacheSize, device));
    out->l2_bytes = static_cast<uint64_t>(v);
    HYT_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrGlobalMemoryBusWidth, device));
    out->mem_bus_bits = static_cast<uint32_t>(v);
    size_t free_b = 0, total_b = 0;
    HYT_CUDA(cudaMemGetInfo(&free_b, &total_b));
    out->hbm_bytes = total_b;
    if (free_b < 2 * copy_bytes + (uint64_t(64) << 20))
        fail(HYT_E_OOM, "hyt_measure_peaks: not enough free device memory for the copy buffers");

    StreamHold sh;
    const cudaStream_t s = sh.s;
    DeviceArray<unsigned char> a(copy_bytes), b(copy_bytes);
    HYT_CUDA(cudaMemsetAsync(a.get(), 1, copy_bytes, s));
    HYT_CUDA(cudaMemcpyAsync(b.get(), a.get(), copy_bytes, cudaMemcpyDeviceToDevice, s));  // warm-up
    const double copy_ms = best_ms(s, 5, [&] {
        HYT_CUDA(cudaMemcpyAsync(b.get(), a.get(), copy_bytes, cudaMemcpyDeviceToDevice, s));
    });
    out->hbm_copy_gbs = 2.0 * double(copy_bytes) / (copy_ms * 1e-3) / 1e9;  // read + write

    PinnedArray<unsigned char> h(link_bytes, cudaHostAllocMapped);
    std::memset(h.ptr, 1, link_bytes);
    const double h2d_ms = best_ms(s, 5, [&] {
        HYT_CUDA(cudaMemcpyAsync(a.get(), h.ptr, link_bytes, cudaMemcpyHostToDevice, s));
    });
    const double d2h_ms = best_ms(s, 5, [&] {
        HYT_CUDA(cudaMemcpyAsync(h.ptr, a.get(), link_bytes, cudaMemcpyDeviceToHost, s));
    });
    out->h2d_gbs = double(link_bytes) / (h2d_ms * 1e-3) / 1e9;
    out->d2h_gbs = double(link_bytes) / (d2h_ms * 1e-3) / 1e9;

    void *zp = nullptr;
    HYT_CUDA(cudaHostGetDevicePointer(&zp, h.ptr, 0));
    DeviceArray<unsigned long long> sink(1);
    const unsigned grid = out->sm_count * 8u;
    const double zc_ms = best_ms(s, 3, [&] {
        peaks_zc_read_kernel<<<grid, 256, 0, s>>>(static_cast<const uint4 *>(zp), link_bytes / 16, sink.get());
        HYT_CUDA(cudaGetLastError());
    });
    out->zero_copy_gbs = double(link_bytes) / (zc_ms * 1e-3) / 1e9;
    out->copy_bytes = copy_bytes;
    out->link_bytes = link_bytes;
    HYT_CUDA(cudaStreamSynchronize(s));
}

}  // namespace hyt

extern "C" int hyt_measure_peaks(int device, uint64_t copy_bytes, hyt_peaks *out) {
    return hyt::guarded([&] {
        if (!out) hyt::fail(HYT_E_INVALID, "out is NULL");
        int n = 0;
        if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
            (void)cudaGetLastError();
            hyt::fail(HYT_E_NO_DEVICE, "no CUDA device is available");
        }
        if (device < 0 || device >= n) hyt::fail(HYT_E_INVALID, "hyt_measure_peaks: device index out of range");
        int cur = 0;
        HYT_CUDA(cudaGetDevice(&cur));
        try {
            hyt::measure_peaks(device, copy_bytes, out);
        } catch (...) {
            cudaSetDevice(cur);
            throw;
        }
        HYT_CUDA(cudaSetDevice(cur));
    });
}
