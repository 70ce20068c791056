// Chunked bucket partition (a radix-partition pass keyed by bucket id).
//
// Each CTA takes contiguous chunks of kPartChunk keys. A chunk's keys fall into one
// contiguous bucket range (all buckets of a plain build, or the buckets of the few sets a
// batched chunk spans). When that range has at most kPartBins buckets the CTA counts its
// keys per bucket in shared memory, reserves each bucket's slice with one global atomic per
// non-empty bin, and places its keys by shared-memory ranks, so global atomics drop from
// one per key to one per (chunk, bucket). Wider ranges fall back to one global atomic per
// key. The order of keys inside a bucket is not deterministic; nothing downstream depends
// on it (every seed depends only on the set of a node's keys).
#pragma once

#include "rsb_common.cuh"

namespace rsb {

constexpr uint32_t kPartThreads = 256;
constexpr uint32_t kPartChunk = kPartThreads * 32;
constexpr uint32_t kPartBins = 8192;  // 32 KB of counters

// Largest s with a[s] <= v among a[0..n] (a non-decreasing, a[0] <= v).
__device__ __forceinline__ uint32_t part_upper_index(const uint64_t *a, uint32_t n, uint64_t v) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) / 2;
        if (a[mid] <= v) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Bucket of key i of a plain build: remap128(first, nb) (AbstractParallelRecSplit.hpp:322).
struct PlainBuckets {
    uint64_t nb;
    __device__ void chunk(uint64_t, uint64_t, uint64_t &b0, uint64_t &nbins) const {
        b0 = 0;
        nbins = nb;
    }
    __device__ uint32_t bucket(const ulonglong2 *keys, uint64_t i) const { return (uint32_t)remap128(keys[i].x, nb); }
};

// Bucket of key i of a batched build, as assigned by the count pass (bucket_id[i]); a chunk
// spans the buckets of the sets that own its first and last key.
struct SetBuckets {
    const uint64_t *set_key, *set_bucket;
    uint32_t nsets;
    const uint32_t *bucket_id;
    __device__ void chunk(uint64_t c0, uint64_t c1, uint64_t &b0, uint64_t &nbins) const {
        const uint32_t lo = part_upper_index(set_key, nsets, c0), hi = part_upper_index(set_key, nsets, c1 - 1);
        b0 = set_bucket[lo];
        nbins = set_bucket[hi + 1] - b0;
    }
    __device__ uint32_t bucket(const ulonglong2 *, uint64_t i) const { return bucket_id[i]; }
};

template <class Map>
__global__ void __launch_bounds__(kPartThreads) k_chunk_scatter(const ulonglong2 *__restrict__ keys, uint64_t n, Map map,
                                                                 const uint64_t *__restrict__ acc, uint32_t *cursor,
                                                                 uint64_t *out) {
    __shared__ uint32_t bins[kPartBins];
    __shared__ uint64_t s_b0, s_nbins;
    for (uint64_t c0 = (uint64_t)blockIdx.x * kPartChunk; c0 < n; c0 += (uint64_t)gridDim.x * kPartChunk) {
        const uint64_t c1 = c0 + kPartChunk < n ? c0 + kPartChunk : n;
        __syncthreads();
        if (threadIdx.x == 0) {
            uint64_t b0, nbins;
            map.chunk(c0, c1, b0, nbins);
            s_b0 = b0;
            s_nbins = nbins;
        }
        __syncthreads();
        const uint64_t b0 = s_b0, nbins = s_nbins;
        if (nbins > kPartBins) {  // wide chunk: one global atomic per key
            for (uint64_t i = c0 + threadIdx.x; i < c1; i += kPartThreads) {
                const uint32_t b = map.bucket(keys, i);
                out[acc[b] + atomicAdd(&cursor[b], 1u)] = keys[i].y;
            }
            continue;
        }
        for (uint32_t j = threadIdx.x; j < nbins; j += kPartThreads) bins[j] = 0;
        __syncthreads();
        for (uint64_t i = c0 + threadIdx.x; i < c1; i += kPartThreads) atomicAdd(&bins[map.bucket(keys, i) - b0], 1u);
        __syncthreads();
        // reserve each bucket's slice for this chunk; the bin then holds the slice start
        for (uint32_t j = threadIdx.x; j < nbins; j += kPartThreads)
            if (bins[j]) bins[j] = atomicAdd(&cursor[b0 + j], bins[j]);
        __syncthreads();
        for (uint64_t i = c0 + threadIdx.x; i < c1; i += kPartThreads) {
            const uint32_t b = map.bucket(keys, i);
            out[acc[b] + atomicAdd(&bins[b - b0], 1u)] = keys[i].y;
        }
    }
}

}  // namespace rsb
