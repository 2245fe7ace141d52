// Setup-time device primitives (sorting, scans, selection).  They run once
// per graph (CSC transpose, R-MAT construction, work-tile lists), never on
// the per-iteration path.  Implemented over CUB in prims.cu so the heavy
// template instantiations live in a single translation unit.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace hyt::prims {

// Stable LSD radix sort of (key, value) pairs on key bits [0, end_bit).
// keys/vals are sorted in place (temporary double buffers are allocated).
void sort_pairs_u32(uint32_t *keys, uint32_t *vals, size_t n, int end_bit, cudaStream_t s);

// Stable LSD radix sort of (u32 key, u64 value) pairs on key bits
// [0, end_bit), in place.
void sort_pairs_u32_u64(uint32_t *keys, uint64_t *vals, size_t n, int end_bit, cudaStream_t s);

// Same, descending by key (stable: equal keys keep their input order).
void sort_pairs_desc_u32(uint32_t *keys, uint32_t *vals, size_t n, cudaStream_t s);

// Stable descending sort of (u64 key, u32 value) pairs, in place.
void sort_pairs_desc_u64(uint64_t *keys, uint32_t *vals, size_t n, cudaStream_t s);

// Radix sort of 64-bit keys on bits [0, end_bit), in place.
void sort_keys_u64(uint64_t *keys, size_t n, int end_bit, cudaStream_t s);

// out[i] = sum_{j<i} in[j]; out has n elements (exclusive scan).
void exclusive_scan_u64(const uint64_t *in, uint64_t *out, size_t n, cudaStream_t s);
void exclusive_scan_u32(const uint32_t *in, uint32_t *out, size_t n, cudaStream_t s);

// out[i] = max_{j<=i} in[j] (inclusive max scan); in and out distinct.
void inclusive_max_scan_u32(const uint32_t *in, uint32_t *out, size_t n, cudaStream_t s);

// Keeps in[i] where flags[i] != 0 (order preserved); returns the count.
size_t select_flagged_u64(const uint64_t *in, const uint8_t *flags, uint64_t *out, size_t n,
                          cudaStream_t s);
// Indices i in [0, n) with flags[i] != 0, ascending; returns the count.
size_t select_flagged_index(const uint8_t *flags, uint32_t *out, size_t n, cudaStream_t s);

// Max of a u32 array (0 for n == 0).
uint32_t reduce_max_u32(const uint32_t *in, size_t n, cudaStream_t s);
uint64_t reduce_max_u64(const uint64_t *in, size_t n, cudaStream_t s);

}  // namespace hyt::prims
