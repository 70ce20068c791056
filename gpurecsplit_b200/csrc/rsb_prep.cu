// Preparation kernels: key hashing, bucket assignment (histogram -> scan -> scatter),
// per-bucket sort with duplicate detection, tree emission and stage lists.
//
// Reference steps replaced (all run on the host there):
//   string hashing            GPURecSplit.cuh:443-468, util/Hash128.h:32-36
//   sort + partition          AbstractParallelRecSplit.hpp:339-359, src/Sorter.cpp:4-5
//   grouping by bucket size   GPURecSplit.cuh:675-695
#include <atomic>
#include <mutex>
#include <set>
#include <utility>

#include "rsb_kernels.cuh"
#include "rsb_partition.cuh"
#include "rsb_spooky.cuh"

namespace rsb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint64_t warp_incl_scan(uint64_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

// Block-wide exclusive scan of one value per thread; returns the block total in *total.
template <int THREADS>
__device__ uint64_t block_excl_scan(uint64_t v, uint64_t *total) {
    __shared__ uint64_t warp_tot[THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint64_t inc = warp_incl_scan(v);
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        const uint64_t t = lane < THREADS / 32 ? warp_tot[lane] : 0;
        const uint64_t ti = warp_incl_scan(t);
        if (lane < THREADS / 32) warp_tot[lane] = ti - t;
        if (lane == THREADS / 32 - 1) *total = ti;
    }
    __syncthreads();
    const uint64_t res = warp_tot[warp] + inc - v;
    __syncthreads();
    return res;
}

__global__ void k_scan_reduce(const uint32_t *in, size_t n, uint64_t *block_sums) {
    const size_t base = (size_t)blockIdx.x * kScanTile;
    uint64_t s = 0;
    for (int k = 0; k < kScanItems; ++k) {
        const size_t i = base + (size_t)k * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    __shared__ uint64_t tot;
    block_excl_scan<kScanThreads>(s, &tot);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = tot;
}

__global__ void k_scan_blocks(uint64_t *block_sums, size_t nblocks) {
    // single block of kScanThreads: exclusive scan of the block sums in place. Every kernel of
    // the engine keeps its CTA within 16K registers, so that it always fits beside another
    // engine's persistent kernels running at 75 % of the SM (a build service's small lane).
    __shared__ uint64_t carry;
    __shared__ uint64_t tot;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (size_t b0 = 0; b0 < nblocks; b0 += blockDim.x) {
        const size_t i = b0 + threadIdx.x;
        const uint64_t v = i < nblocks ? block_sums[i] : 0;
        const uint64_t ex = block_excl_scan<kScanThreads>(v, &tot);
        if (i < nblocks) block_sums[i] = carry + ex;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
}

__global__ void k_scan_final(const uint32_t *in, size_t n, const uint64_t *block_sums, uint64_t *out) {
    const size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const size_t i = base + k;
        v[k] = i < n ? in[i] : 0;
        s += v[k];
    }
    __shared__ uint64_t tot;
    uint64_t ex = block_excl_scan<kScanThreads>(s, &tot) + block_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const size_t i = base + k;
        if (i < n) out[i] = ex;
        ex += v[k];
        if (i + 1 == n) out[n] = ex;
    }
    if (n == 0 && blockIdx.x == 0 && threadIdx.x == 0) out[0] = 0;
}

}  // namespace

size_t scan_blocks(size_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

void exclusive_scan_u32(const uint32_t *in, uint64_t *out, size_t n, ScanTmp tmp, cudaStream_t st) {
    const size_t blocks = n == 0 ? 1 : (n + kScanTile - 1) / kScanTile;
    use_max_smem(k_scan_reduce);
    k_scan_reduce<<<blocks, kScanThreads, 0, st>>>(in, n, tmp.block_sums);
    use_max_smem(k_scan_blocks);
    k_scan_blocks<<<1, kScanThreads, 0, st>>>(tmp.block_sums, blocks);
    use_max_smem(k_scan_final);
    k_scan_final<<<blocks, kScanThreads, 0, st>>>(in, n, tmp.block_sums, out);
    count_launches(3);
}

// ---------------------------------------------------------------------------------------
// Key hashing.
// ---------------------------------------------------------------------------------------
namespace {

__device__ __forceinline__ uint64_t fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}
__device__ __forceinline__ uint64_t stafford13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__global__ void k_hash_u64(const uint64_t *__restrict__ keys, uint64_t n, ulonglong2 *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        out[i] = make_ulonglong2(fmix64(k), stafford13(k + 0x9e3779b97f4a7c15ULL));
    }
}

// Key i is bytes[offsets[i] - base, offsets[i + 1] - base). Each warp takes 32 consecutive
// keys, whose bytes are contiguous: it copies them into shared memory with coalesced 16-byte
// loads (the unaligned head and tail byte by byte, so that no load leaves the warp's own
// bytes), then each lane hashes its key from there through aligned 32-bit reads (byte reads
// of the warp's keys at scattered offsets cost a shared-memory wavefront per byte). A warp
// whose bytes exceed its buffer, or whose offsets are not non-decreasing, hashes from global
// memory, one key per lane.
constexpr int kHashThreads = 128;
constexpr uint32_t kHashWarpBytes = 2048;  // staged bytes per warp, from the 16-byte block of the first

__global__ void __launch_bounds__(kHashThreads) k_hash_strings(const uint8_t *__restrict__ bytes,
                                                               const uint64_t *__restrict__ offsets, uint64_t n,
                                                               uint64_t base, ulonglong2 *__restrict__ out) {
    __shared__ __align__(16) uint8_t staged[kHashThreads / 32][kHashWarpBytes];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint8_t *buf = staged[warp];
    const uint64_t stride = (uint64_t)gridDim.x * kHashThreads;
    for (uint64_t i0 = blockIdx.x * (uint64_t)kHashThreads + warp * 32u; i0 < n; i0 += stride) {
        const uint64_t i = i0 + lane;
        const bool valid = i < n;
        const uint64_t iend = n - i0 < 32 ? n : i0 + 32;
        const uint64_t gb = offsets[i0], ge = offsets[iend];  // the warp's bytes, before rebasing
        const uint64_t b = valid ? offsets[i] : gb, e = valid ? offsets[i + 1] : gb;
        const uintptr_t a0 = (uintptr_t)(bytes + (gb - base)), a1 = (uintptr_t)(bytes + (ge - base));
        const uintptr_t al0 = a0 & ~(uintptr_t)15;
        const bool inside = gb <= b && b <= e && e <= ge;
        const bool stage = __all_sync(0xffffffffu, inside) && gb <= ge && a1 - al0 <= kHashWarpBytes;
        uint64_t h0 = 0, h1 = 0;
        if (stage) {
            const uintptr_t m0 = (a0 + 15) & ~(uintptr_t)15, m1 = a1 & ~(uintptr_t)15;
            if (m0 < m1) {
                for (uintptr_t a = a0 + lane; a < m0; a += 32) buf[a - al0] = *(const uint8_t *)a;
                for (uintptr_t a = m0 + 16u * lane; a < m1; a += 16u * 32)
                    *(uint4 *)(buf + (a - al0)) = *(const uint4 *)a;
                for (uintptr_t a = m1 + lane; a < a1; a += 32) buf[a - al0] = *(const uint8_t *)a;
            } else {
                for (uintptr_t a = a0 + lane; a < a1; a += 32) buf[a - al0] = *(const uint8_t *)a;
            }
            __syncwarp();
            if (valid) spooky128<true>(buf + (a0 - al0) + (b - gb), e - b, h0, h1);  // word reads
            __syncwarp();  // buf is rewritten by the next 32 keys
        } else if (valid) {
            spooky128(bytes + (b - base), e - b, h0, h1);
        }
        if (valid) out[i] = make_ulonglong2(h1, h0);  // first = h1, second = h0 (util/Hash128.h:35)
    }
}

// ---------------------------------------------------------------------------------------
// Bucket assignment: bucket = remap128(first, nbuckets) (AbstractParallelRecSplit.hpp:322).
// ---------------------------------------------------------------------------------------
constexpr uint64_t kSmemHistMax = 12288;

__global__ void k_bucket_count_smem(const ulonglong2 *__restrict__ keys, uint64_t n, uint64_t nb, uint32_t *counts) {
    extern __shared__ uint32_t hist[];
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&hist[remap128(keys[i].x, nb)], 1u);
    __syncthreads();
    for (uint64_t b = threadIdx.x; b < nb; b += blockDim.x)
        if (hist[b]) atomicAdd(&counts[b], hist[b]);
}

__global__ void k_bucket_count_global(const ulonglong2 *__restrict__ keys, uint64_t n, uint64_t nb, uint32_t *counts) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&counts[remap128(keys[i].x, nb)], 1u);
}

__global__ void k_bucket_check(const uint32_t *counts, uint64_t nb, DevStatus *status) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x)
        if (counts[b] >= (uint32_t)kMaxBucketSize) set_error(status, RSB_ERR_BUCKET_TOO_LARGE, b);
}

// Duplicate check: two keys with the same second half in one bucket always collide, so the
// reference's search would never end (GPURecSplit.cuh:436); here the build fails with
// RSB_ERR_DUPLICATE_KEY. A warp (buckets of at most 256 keys) or a CTA (larger buckets)
// inserts a bucket's second halves into an open-addressing table in shared memory (read-only
// pass over the keys); a second key equal to the empty-slot marker is counted instead. The
// key order inside a bucket is
// left as the scatter produced it: every seed depends only on the set of a node's keys.
constexpr int kSortThreads = 256;
constexpr int kSortCap = 4096;  // > 2 * (kMaxBucketSize - 1) / 1.5: table at most 3/4 full
constexpr uint64_t kEmptyKey = ~0ull;
static_assert(4 * (kMaxBucketSize - 1) <= 3 * kSortCap, "duplicate table too small");

constexpr uint32_t kWarpDupMax = 256;                           // buckets up to this size: one warp each
constexpr uint32_t kWarpDupSlots = kSortCap / (kSortThreads / 32);  // a warp's slice of the table
static_assert(2 * kWarpDupMax <= kWarpDupSlots, "warp table too small");

// Inserts k into the open-addressing table tab[0, size); returns whether it was there.
__device__ __forceinline__ bool dup_insert(uint64_t *tab, uint32_t size, uint64_t k) {
    // `second` is a hash output, so its low bits are a uniform slot; linear probing visits at
    // most `size` slots and the table is at most 3/4 full.
    uint32_t slot = (uint32_t)k & (size - 1);
    for (uint32_t probe = 0; probe < size; ++probe) {
        const uint64_t prev = atomicCAS((unsigned long long *)&tab[slot], kEmptyKey, k);
        if (prev == kEmptyKey) return false;
        if (prev == k) return true;
        slot = (slot + 1) & (size - 1);
    }
    return false;
}

__global__ void __launch_bounds__(kSortThreads) k_bucket_dupcheck(const uint64_t *sorted, const uint64_t *acc,
                                                                  uint64_t nb, DevStatus *status) {
    __shared__ uint64_t tab[kSortCap];
    __shared__ uint32_t n_empty_key;  // keys equal to the empty-slot marker
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // Buckets of at most kWarpDupMax keys: one warp each, in its own slice of the table, so
    // the warps of a CTA check different buckets at once.
    uint64_t *wt = tab + warp * kWarpDupSlots;
    const uint64_t nw = (uint64_t)gridDim.x * (kSortThreads / 32);
    for (uint64_t b = blockIdx.x * (uint64_t)(kSortThreads / 32) + warp; b < nb; b += nw) {
        const uint64_t off = acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - off);
        if (m <= 1 || m > kWarpDupMax) continue;
        uint32_t size = 64;
        while (size < 2 * m) size <<= 1;
        for (uint32_t i = lane; i < size; i += 32) wt[i] = kEmptyKey;
        __syncwarp();
        bool dup = false;
        uint32_t empties = 0;
        for (uint32_t i = lane; i < m; i += 32) {
            const uint64_t k = sorted[off + i];
            if (k == kEmptyKey) ++empties;
            else dup |= dup_insert(wt, size, k);
        }
        empties = __reduce_add_sync(0xffffffffu, empties);
        if (__any_sync(0xffffffffu, dup) || empties > 1) {
            if (lane == 0) set_error(status, RSB_ERR_DUPLICATE_KEY, b);
        }
        __syncwarp();  // the slice is cleared for the warp's next bucket
    }
    __syncthreads();  // the whole table serves the larger buckets below
    for (uint64_t b = blockIdx.x; b < nb; b += gridDim.x) {
        const uint64_t off = acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - off);
        if (m <= kWarpDupMax || m > (uint32_t)kMaxBucketSize) continue;  // oversize buckets: k_bucket_check
        uint32_t size = 64;
        while (size < 2 * m && size < (uint32_t)kSortCap) size <<= 1;
        for (uint32_t i = threadIdx.x; i < size; i += kSortThreads) tab[i] = kEmptyKey;
        if (threadIdx.x == 0) n_empty_key = 0;
        __syncthreads();
        bool dup = false;
        for (uint32_t i = threadIdx.x; i < m; i += kSortThreads) {
            const uint64_t k = sorted[off + i];
            if (k == kEmptyKey) {
                dup |= atomicAdd(&n_empty_key, 1u) > 0;
                continue;
            }
            dup |= dup_insert(tab, size, k);
        }
        if (dup) set_error(status, RSB_ERR_DUPLICATE_KEY, b);
        __syncthreads();
    }
}

__global__ void k_bucket_nodes(const uint64_t *acc, uint64_t nb, DevTables tab, uint32_t *node_count) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t m = acc[b + 1] - acc[b];
        node_count[b] = m < (uint64_t)kMaxBucketSize ? tab.nodes[m] : 0;
    }
}

// ---------------------------------------------------------------------------------------
// Tree emission: the tree of a bucket depends only on its size (SplittingStrategy), so
// every node's key range is known before any search. Nodes are numbered in DFS pre-order,
// the order of the descriptor stream (SIMDRecSplit.hpp:624-693).
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void dev_split_params(const Shape &s, uint32_t m, uint32_t &fanout, uint32_t &unit) {
    if (m > s.upper) {
        unit = s.upper * (uint16_t(m / 2 + s.upper - 1) / s.upper);
        fanout = 2;
    } else if (m > s.lower) {
        unit = s.lower;
        fanout = uint16_t(m + s.lower - 1) / s.lower;
    } else {
        unit = s.leaf;
        fanout = uint16_t(m + s.leaf - 1) / s.leaf;
    }
}

__device__ __forceinline__ uint8_t stage_of(const Shape &s, uint32_t m, uint32_t depth) {
    if (m <= s.leaf) return (s.rotate && m == s.leaf) ? kStageLeafRot : kStageLeafBF;
    if (m > s.upper) return (uint8_t)depth;
    return m > s.lower ? kStageUpper : kStageLower;
}

struct Frame {
    uint32_t off;
    uint16_t m;
    uint8_t depth;
    uint8_t child;
};

__global__ void k_tree_emit(const uint64_t *acc, uint64_t nb, const uint64_t *node_base, Shape sh, NodeArrays nodes) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < nb; b += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t off = (uint32_t)acc[b];
        const uint32_t m = (uint32_t)(acc[b + 1] - acc[b]);
        if (m <= 1 || m >= (uint32_t)kMaxBucketSize) continue;
        uint32_t id = (uint32_t)node_base[b];
        Frame stack[24];
        int sp = 0;
        nodes.start[id] = off;
        nodes.size[id] = (uint16_t)m;
        nodes.stage[id] = stage_of(sh, m, 0);
        ++id;
        if (m > sh.leaf) stack[sp++] = Frame{off, (uint16_t)m, 0, 0};
        while (sp > 0) {
            Frame &f = stack[sp - 1];
            uint32_t fanout, unit;
            dev_split_params(sh, f.m, fanout, unit);
            if (f.child >= fanout) {
                --sp;
                continue;
            }
            const uint32_t c = f.child++;
            const uint32_t cm = c + 1 < fanout ? unit : f.m - (fanout - 1) * unit;
            if (cm <= 1) continue;
            const uint32_t coff = f.off + c * unit;
            const uint32_t cd = f.depth + 1;
            nodes.start[id] = coff;
            nodes.size[id] = (uint16_t)cm;
            nodes.stage[id] = stage_of(sh, cm, cd);
            ++id;
            if (cm > sh.leaf) stack[sp++] = Frame{coff, (uint16_t)cm, (uint8_t)cd, 0};
        }
    }
}

// Stage lists (counting sort of node ids by stage, warp-aggregated atomics).
__global__ void k_stage_hist(const uint8_t *stage, const uint64_t *total, uint32_t *stage_info) {
    __shared__ uint32_t h[kNumStages];
    for (int s = threadIdx.x; s < kNumStages; s += blockDim.x) h[s] = 0;
    __syncthreads();
    const uint64_t n = *total;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        atomicAdd(&h[stage[i]], 1u);
    __syncthreads();
    for (int s = threadIdx.x; s < kNumStages; s += blockDim.x)
        if (h[s]) atomicAdd(&stage_info[s], h[s]);
}

__global__ void k_stage_bases(uint32_t *stage_info) {
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int s = 0; s < kNumStages; ++s) {
            stage_info[kNumStages + s] = acc;
            stage_info[2 * kNumStages + s] = acc;  // fill cursor
            acc += stage_info[s];
        }
    }
}

__global__ void k_stage_scatter(const uint8_t *stage, const uint64_t *total, uint32_t *stage_info, uint32_t *lists) {
    const uint64_t n = *total;
    const int lane = threadIdx.x & 31;
    for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x; i0 < n; i0 += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t i = i0 + threadIdx.x;
        const bool valid = i < n;
        const int s = valid ? stage[i] : -1;
        const unsigned peers = __match_any_sync(0xffffffffu, s);
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (valid && lane == leader) base = atomicAdd(&stage_info[2 * kNumStages + s], (uint32_t)__popc(peers));
        base = __shfl_sync(0xffffffffu, base, leader);
        if (valid) lists[base + __popc(peers & ((1u << lane) - 1))] = (uint32_t)i;
    }
}

int grid_for(uint64_t n, int threads, int cap) {
    uint64_t g = (n + threads - 1) / threads;
    if (g < 1) g = 1;
    if (g > (uint64_t)cap) g = cap;
    return (int)g;
}

// Part builds: the keys of buckets [lo, lo + nbp) of an nb_total-bucket function become the
// keys of an nbp-bucket function with the same buckets. `first` of a key of bucket lo + j is
// replaced by (j + 1) * q - 1 with q = floor((2^64 - 1) / nbp), which remap128 sends to j:
// (j + 1) q nbp - nbp lies in [j 2^64, (j + 1) 2^64) for nbp < 2^32. The second halves, which
// alone decide the seeds, are unchanged. A key outside the range sets RSB_ERR_BAD_ARG.
__global__ void k_part_first(ulonglong2 *keys, uint64_t n, uint64_t nb_total, uint64_t lo, uint64_t nbp, uint64_t q,
                             DevStatus *status) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = remap128(keys[i].x, nb_total);
        if (b < lo || b - lo >= nbp) {
            set_error(status, RSB_ERR_BAD_ARG, i);
            continue;
        }
        keys[i].x = (b - lo + 1) * q - 1;
    }
}

}  // namespace

void launch_part_first(uint64_t *keys128, uint64_t n, uint64_t nb_total, uint64_t lo, uint64_t nbp, DevStatus *status,
                       cudaStream_t st) {
    use_max_smem(k_part_first);
    k_part_first<<<grid_for(n, 256, device_sm_count() * 16), 256, 0, st>>>((ulonglong2 *)keys128, n, nb_total, lo, nbp,
                                                                           ~0ull / nbp, status);
    count_launches(1);
}

void launch_hash_u64(const uint64_t *keys, uint64_t n, uint64_t *out128, cudaStream_t st) {
    use_max_smem(k_hash_u64);
    k_hash_u64<<<grid_for(n, 256, device_sm_count() * 16), 256, 0, st>>>(keys, n, (ulonglong2 *)out128);
    count_launches(1);
}

void launch_hash_strings(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t base, uint64_t *out128,
                         cudaStream_t st) {
    use_max_smem(k_hash_strings);
    k_hash_strings<<<grid_for(n, kHashThreads, device_sm_count() * 32), kHashThreads, 0, st>>>(bytes, offsets, n, base, (ulonglong2 *)out128);
    count_launches(1);
}

void launch_bucket_count(const uint64_t *keys128, uint64_t n, uint64_t nb, uint32_t *counts, cudaStream_t st) {
    cudaMemsetAsync(counts, 0, nb * sizeof(uint32_t), st);
    if (nb <= kSmemHistMax) {
        use_max_smem(k_bucket_count_smem);
        k_bucket_count_smem<<<grid_for(n, 512, device_sm_count() * 4), 512, nb * sizeof(uint32_t), st>>>((const ulonglong2 *)keys128, n,
                                                                                            nb, counts);
    } else {
        use_max_smem(k_bucket_count_global);
        k_bucket_count_global<<<grid_for(n, 256, device_sm_count() * 16), 256, 0, st>>>((const ulonglong2 *)keys128, n, nb, counts);
    }
    count_launches(1);
}

void launch_bucket_check(const uint32_t *counts, uint64_t nb, DevStatus *status, cudaStream_t st) {
    use_max_smem(k_bucket_check);
    k_bucket_check<<<grid_for(nb, 256, device_sm_count() * 8), 256, 0, st>>>(counts, nb, status);
    count_launches(1);
}

void launch_bucket_scatter(const uint64_t *keys128, uint64_t n, uint64_t nb, const uint64_t *acc, uint32_t *cursor,
                           uint64_t *sorted, cudaStream_t st) {
    cudaMemsetAsync(cursor, 0, nb * sizeof(uint32_t), st);
    use_max_smem(k_chunk_scatter<PlainBuckets>);
    k_chunk_scatter<<<grid_for(n, kPartChunk, device_sm_count() * 6), kPartThreads, 0, st>>>((const ulonglong2 *)keys128, n,
                                                                               PlainBuckets{nb}, acc, cursor, sorted);
    count_launches(1);
}

void launch_bucket_dupcheck(const uint64_t *sorted, const uint64_t *acc, uint64_t nb, DevStatus *status,
                            cudaStream_t st) {
    use_max_smem(k_bucket_dupcheck);
    k_bucket_dupcheck<<<grid_for(nb, 1, device_sm_count() * 7), kSortThreads, 0, st>>>(sorted, acc, nb, status);
    count_launches(1);
}

void launch_bucket_nodes(const uint64_t *acc, uint64_t nb, DevTables tab, uint32_t *node_count, cudaStream_t st) {
    use_max_smem(k_bucket_nodes);
    k_bucket_nodes<<<grid_for(nb, 256, device_sm_count() * 8), 256, 0, st>>>(acc, nb, tab, node_count);
    count_launches(1);
}

void launch_tree_emit(const uint64_t *acc, uint64_t nb, const uint64_t *node_base, Shape sh, NodeArrays nodes,
                      cudaStream_t st) {
    use_max_smem(k_tree_emit);
    k_tree_emit<<<grid_for(nb, 64, device_sm_count() * 16), 64, 0, st>>>(acc, nb, node_base, sh, nodes);
    count_launches(1);
}

void launch_stage_lists(const uint8_t *stage, const uint64_t *total_nodes, uint32_t max_nodes, uint32_t *stage_info,
                        uint32_t *lists, cudaStream_t st) {
    cudaMemsetAsync(stage_info, 0, 3 * kNumStages * sizeof(uint32_t), st);
    const int g = grid_for(max_nodes, 256, device_sm_count() * 8);
    use_max_smem(k_stage_hist);
    k_stage_hist<<<g, 256, 0, st>>>(stage, total_nodes, stage_info);
    use_max_smem(k_stage_bases);
    k_stage_bases<<<1, 32, 0, st>>>(stage_info);
    use_max_smem(k_stage_scatter);
    k_stage_scatter<<<g, 256, 0, st>>>(stage, total_nodes, stage_info, lists);
    count_launches(3);
}


int device_sm_count() {
    constexpr int kMaxDev = 64;
    static std::atomic<int> cache[kMaxDev];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
        cudaGetLastError();
        return 148;
    }
    int v = cache[dev].load(std::memory_order_relaxed);
    if (v <= 0) {
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0) {
            cudaGetLastError();
            return 148;  // B200's count; the attribute query does not fail on a working device
        }
        cache[dev].store(v, std::memory_order_relaxed);
    }
    return v;
}

void prefer_shared_memory(const void *func) {
    static std::mutex mu;
    static std::set<std::pair<const void *, int>> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    std::lock_guard<std::mutex> lock(mu);
    if (!done.insert({func, dev}).second) return;
    if (cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared) !=
        cudaSuccess)
        cudaGetLastError();  // a preference only: launches work without it
}

}  // namespace rsb
