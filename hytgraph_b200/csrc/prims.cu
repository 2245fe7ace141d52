// CUB-backed setup primitives; see prims.cuh.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include "common.cuh"
#include "prims.cuh"
#include "scratch.cuh"

namespace hyt::prims {

void sort_pairs_u32(uint32_t *keys, uint32_t *vals, size_t n, int end_bit, cudaStream_t s) {
    if (n < 2) return;
    Scratch<uint32_t> k2(n, s), v2(n, s);
    cub::DoubleBuffer<uint32_t> kb(keys, k2.get()), vb(vals, v2.get());
    size_t tb = 0;
    HYT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, end_bit, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, end_bit, s));
    if (kb.Current() != keys)
        HYT_CUDA(cudaMemcpyAsync(keys, kb.Current(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    if (vb.Current() != vals)
        HYT_CUDA(cudaMemcpyAsync(vals, vb.Current(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void sort_pairs_u32_u64(uint32_t *keys, uint64_t *vals, size_t n, int end_bit, cudaStream_t s) {
    if (n < 2) return;
    Scratch<uint32_t> k2(n, s);
    Scratch<uint64_t> v2(n, s);
    cub::DoubleBuffer<uint32_t> kb(keys, k2.get());
    cub::DoubleBuffer<uint64_t> vb(vals, v2.get());
    size_t tb = 0;
    HYT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, end_bit, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceRadixSort::SortPairs(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, end_bit, s));
    if (kb.Current() != keys)
        HYT_CUDA(cudaMemcpyAsync(keys, kb.Current(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    if (vb.Current() != vals)
        HYT_CUDA(cudaMemcpyAsync(vals, vb.Current(), n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void sort_pairs_desc_u32(uint32_t *keys, uint32_t *vals, size_t n, cudaStream_t s) {
    if (n < 2) return;
    Scratch<uint32_t> k2(n, s), v2(n, s);
    cub::DoubleBuffer<uint32_t> kb(keys, k2.get()), vb(vals, v2.get());
    size_t tb = 0;
    HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, 32, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, 32, s));
    if (kb.Current() != keys)
        HYT_CUDA(cudaMemcpyAsync(keys, kb.Current(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    if (vb.Current() != vals)
        HYT_CUDA(cudaMemcpyAsync(vals, vb.Current(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void sort_pairs_desc_u64(uint64_t *keys, uint32_t *vals, size_t n, cudaStream_t s) {
    if (n < 2) return;
    Scratch<uint64_t> k2(n, s);
    Scratch<uint32_t> v2(n, s);
    cub::DoubleBuffer<uint64_t> kb(keys, k2.get());
    cub::DoubleBuffer<uint32_t> vb(vals, v2.get());
    size_t tb = 0;
    HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb, kb, vb, static_cast<int64_t>(n), 0, 64, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceRadixSort::SortPairsDescending(tmp.get(), tb, kb, vb, static_cast<int64_t>(n), 0, 64, s));
    if (kb.Current() != keys)
        HYT_CUDA(cudaMemcpyAsync(keys, kb.Current(), n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    if (vb.Current() != vals)
        HYT_CUDA(cudaMemcpyAsync(vals, vb.Current(), n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void inclusive_max_scan_u32(const uint32_t *in, uint32_t *out, size_t n, cudaStream_t s) {
    if (n == 0) return;
    size_t tb = 0;
    HYT_CUDA(cub::DeviceScan::InclusiveScan(nullptr, tb, in, out, cub::Max(), static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceScan::InclusiveScan(tmp.get(), tb, in, out, cub::Max(), static_cast<int64_t>(n), s));
}

void sort_keys_u64(uint64_t *keys, size_t n, int end_bit, cudaStream_t s) {
    if (n < 2) return;
    Scratch<uint64_t> k2(n, s);
    cub::DoubleBuffer<uint64_t> kb(keys, k2.get());
    size_t tb = 0;
    HYT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, kb, static_cast<int64_t>(n), 0, end_bit, s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceRadixSort::SortKeys(tmp.get(), tb, kb, static_cast<int64_t>(n), 0, end_bit, s));
    if (kb.Current() != keys)
        HYT_CUDA(cudaMemcpyAsync(keys, kb.Current(), n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void exclusive_scan_u64(const uint64_t *in, uint64_t *out, size_t n, cudaStream_t s) {
    if (n == 0) return;
    size_t tb = 0;
    HYT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, in, out, static_cast<int64_t>(n), s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, size_t n, cudaStream_t s) {
    if (n == 0) return;
    size_t tb = 0;
    HYT_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, in, out, static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), tb, in, out, static_cast<int64_t>(n), s));
    HYT_CUDA(cudaStreamSynchronize(s));
}

size_t select_flagged_u64(const uint64_t *in, const uint8_t *flags, uint64_t *out, size_t n,
                          cudaStream_t s) {
    if (n == 0) return 0;
    Scratch<uint64_t> cnt(1, s);
    size_t tb = 0;
    HYT_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, in, flags, out, cnt.get(), static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, in, flags, out, cnt.get(), static_cast<int64_t>(n), s));
    uint64_t h = 0;
    HYT_CUDA(cudaMemcpyAsync(&h, cnt.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    return static_cast<size_t>(h);
}

size_t select_flagged_index(const uint8_t *flags, uint32_t *out, size_t n, cudaStream_t s) {
    if (n == 0) return 0;
    Scratch<uint64_t> cnt(1, s);
    thrust::counting_iterator<uint32_t> it(0);
    size_t tb = 0;
    HYT_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, it, flags, out, cnt.get(), static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceSelect::Flagged(tmp.get(), tb, it, flags, out, cnt.get(), static_cast<int64_t>(n), s));
    uint64_t h = 0;
    HYT_CUDA(cudaMemcpyAsync(&h, cnt.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    return static_cast<size_t>(h);
}

template <class T>
T reduce_max(const T *in, size_t n, cudaStream_t s) {
    if (n == 0) return 0;
    Scratch<T> r(1, s);
    size_t tb = 0;
    HYT_CUDA(cub::DeviceReduce::Max(nullptr, tb, in, r.get(), static_cast<int64_t>(n), s));
    Scratch<uint8_t> tmp(tb, s);
    HYT_CUDA(cub::DeviceReduce::Max(tmp.get(), tb, in, r.get(), static_cast<int64_t>(n), s));
    T h = 0;
    HYT_CUDA(cudaMemcpyAsync(&h, r.get(), sizeof(h), cudaMemcpyDeviceToHost, s));
    HYT_CUDA(cudaStreamSynchronize(s));
    return h;
}

uint32_t reduce_max_u32(const uint32_t *in, size_t n, cudaStream_t s) { return reduce_max(in, n, s); }
uint64_t reduce_max_u64(const uint64_t *in, size_t n, cudaStream_t s) { return reduce_max(in, n, s); }

}  // namespace hyt::prims
