// Device helpers and launch sizing shared by the seed-search kernels (rsb_search.cu: fanout-2
// searches, dispatch and the evaluation probe; rsb_search_impl.cuh: aggregation and leaf
// searches, instantiated per leaf size in rsb_search_inst_*.cu).
#pragma once

#include <algorithm>
#include <cstdio>

#include "rsb_fp32.cuh"
#include "rsb_kernels.cuh"

namespace rsb {

namespace {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr int kWarpsPerCta = 8;
constexpr int kThreads = kWarpsPerCta * 32;

// (lower_aggr, upper_aggr) per leaf size 2..24, the values of AbstractParallelRecSplit.hpp:133,135;
// checked against make_shape() when an engine first uses a leaf size.
__host__ __device__ constexpr uint32_t lower_of(int leaf) {
    constexpr uint32_t t[25] = {0, 0, 4, 6, 8, 15, 18, 21, 32, 36, 40, 55, 60, 78, 84, 90, 112, 119, 126, 152, 160, 168, 198, 207, 216};
    return t[leaf];
}
__host__ __device__ constexpr uint32_t upper_of(int leaf) {
    constexpr uint32_t t[25] = {0, 0, 8, 12, 16, 30, 36, 63, 96, 108, 120, 220, 240, 312, 336, 450, 560, 595, 630, 760, 960, 1008, 1188, 1242, 1296};
    return t[leaf];
}

__device__ __forceinline__ uint64_t vload64(const uint64_t *p) { return *(const volatile uint64_t *)p; }
__device__ __forceinline__ uint32_t vload32(const uint32_t *p) { return *(const volatile uint32_t *)p; }
__device__ __forceinline__ int status_code(const DevStatus *s) { return *(const volatile int *)&s->code; }

// Shared state that decides a whole warp's path (the status, a node's seed, a counter) is
// read by lane 0 and broadcast: the lanes of a warp need not execute a load at the same
// time, so a word that another warp writes could otherwise differ between them and split
// the warp around its warp-wide operations.
__device__ __forceinline__ uint64_t warp_load64(const uint64_t *a) {
    uint64_t v = 0;
    if ((threadIdx.x & 31) == 0) v = vload64(a);
    return __shfl_sync(0xffffffffu, v, 0);
}
__device__ __forceinline__ uint32_t warp_load32(const uint32_t *a) {
    uint32_t v = 0;
    if ((threadIdx.x & 31) == 0) v = vload32(a);
    return __shfl_sync(0xffffffffu, v, 0);
}
__device__ __forceinline__ int warp_status(const DevStatus *s) {
    int v = 0;
    if ((threadIdx.x & 31) == 0) v = status_code(s);
    return __shfl_sync(0xffffffffu, v, 0);
}

// shl.b32 clamps shift amounts >= 32 to 32 (result 0), PTX ISA "shl".
__device__ __forceinline__ uint32_t shl_clamp(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("shl.b32 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
    return d;
}

// Low 16 bits of remix32(hi ^ lo) of a 64-bit candidate.
__device__ __forceinline__ uint32_t hash16(uint64_t v) { return remix32(uint32_t(v >> 32) ^ uint32_t(v)) & 0xFFFFu; }

// Keys of an aggregation node per phase-A pass: after each chunk the window is abandoned if
// the node's best seed has dropped to its first candidate.
constexpr uint32_t kAbortChunk = 64;

// acc[s] += the part index p(k, x) of candidate x = bu + lane + 32 s, summed over the len <=
// kAbortChunk keys sk[0, len) (in add_part's form), where bu is the warp-uniform window base;
// mult is fan for a full node. When the low 16 bits of key + bu cannot overflow within the
// window (all but ~S*32 / 2^16 of the keys), every candidate differs from key + bu only in
// bits 0..15: with lo = low word, hi = high word and L = lo & 0xFFFF, remix32's input
// (hi ^ lo) ^ (hi ^ lo) >> 16 is (L + j) ^ K' for the candidate bu + j, where
// K' = hi ^ hi >> 16 ^ lo >> 16 ^ (lo & 0xFFFF0000) is one per-key constant. The warp first
// computes (K', L) of every such key of the chunk, one key per lane, into pk[0, nf) (shared
// memory), and the indexes of the other keys into pk[kAbortChunk - ns, kAbortChunk); then a
// candidate costs a 32-bit add and an xor before the two multiply rounds, and the few other
// keys take the plain 64-bit form. An exactly balanced split has sum_j j * size_j, so this
// sum is a necessary condition.
template <int S, bool FULL>
__device__ __forceinline__ void moment_sums(const uint64_t *sk, uint32_t len, uint64_t bu, uint32_t mult,
                                            uint2 *pk, uint32_t *acc) {
    constexpr uint32_t kSpan = 32u * S;
    static_assert(kSpan <= 0x10000u, "window wider than the hoisting allows");
    const uint32_t lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1;
    const float cf = (float)mult * 0x1p-16f;
    uint32_t nf = 0, ns = 0;
    for (uint32_t c0 = 0; c0 < len; c0 += 32) {
        const uint32_t i = c0 + lane;
        const bool valid = i < len;
        const uint64_t tu = (valid ? sk[i] : 0) + bu;
        const uint32_t lo = (uint32_t)tu, hi = (uint32_t)(tu >> 32);
        const bool fast = (lo & 0xFFFFu) <= 0x10000u - kSpan;
        const unsigned bf = __ballot_sync(0xffffffffu, valid && fast);
        const unsigned bs = __ballot_sync(0xffffffffu, valid && !fast);
        if (valid && fast)
            pk[nf + __popc(bf & below)] = make_uint2(hi ^ (hi >> 16) ^ (lo >> 16) ^ (lo & 0xFFFF0000u), lo & 0xFFFFu);
        if (valid && !fast) pk[kAbortChunk - 1 - ns - __popc(bs & below)].x = i;
        nf += __popc(bf);
        ns += __popc(bs);
    }
    __syncwarp();
#pragma unroll 4
    for (uint32_t j = 0; j < nf; ++j) {
        const uint2 e = pk[j];
        const uint32_t l0 = e.y + lane;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            uint32_t z = (l0 + 32u * s) ^ e.x;
            z *= 0x85ebca6bu;
            z ^= z >> 13;
            add_part<FULL>(z * 0xc2b2ae35u, mult, cf, acc[s]);
        }
    }
    for (uint32_t j = 0; j < ns; ++j) {
        const uint64_t tu = sk[pk[kAbortChunk - 1 - j].x] + bu;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const uint64_t v = tu + lane + 32u * s;
            add_part<FULL>(remix32_core(uint32_t(v >> 32) ^ uint32_t(v)), mult, cf, acc[s]);
        }
    }
    __syncwarp();  // pk is rewritten by the next chunk
}

__device__ __forceinline__ uint64_t budget_for(const SearchCtx &c, uint32_t m) {
    const uint32_t g = c.tab.memo[m] >> 27;
    const uint32_t sh = min(g + c.budget_shift, 62u);
    const uint64_t b = 1ull << sh;
    return b > c.budget_min ? b : c.budget_min;
}

// Merges a candidate seed into a node's seed. The warp whose merge first moves the seed off
// kSeedNotFound (a success or a failure) counts the node as finished in `found`, the stage's
// finished-node counter, so that idle warps can stop looking for nodes to help once every
// node of the stage has a seed.
__device__ __forceinline__ void merge_seed(uint64_t *node_seed, uint64_t v, uint32_t *found) {
    const unsigned long long old = atomicMin((unsigned long long *)node_seed, (unsigned long long)v);
    if (old == kSeedNotFound) atomicAdd(found, 1u);
}

// Scans the help slots of the launched warps (node ids of owners, from a pseudo-random
// start, four slots per lane per step) for a node of the current stage whose search has not
// found a seed yet.
__device__ uint32_t find_help(const SearchCtx &c, uint32_t start) {
    constexpr uint32_t U = 4;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = min(c.nslots, gridDim.x * (uint32_t)kWarpsPerCta);
    start %= nw;
    for (uint32_t k = 0; k < nw; k += 32 * U) {
        uint32_t nd[U];
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) {
            const uint32_t off = k + j * 32 + lane;
            uint32_t idx = start + off;
            if (idx >= nw) idx -= nw;
            nd[j] = off < nw ? vload32(&c.slots[idx]) : kEmpty;
        }
        uint64_t sd[U];
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) sd[j] = nd[j] != kEmpty ? vload64(&c.nodes.seed[nd[j]]) : 0;
        uint32_t pick = kEmpty;
#pragma unroll
        for (uint32_t j = 0; j < U; ++j)
            if (pick == kEmpty && nd[j] != kEmpty && sd[j] == kSeedNotFound) pick = nd[j];
        const unsigned b = __ballot_sync(0xffffffffu, pick != kEmpty);
        if (b) return __shfl_sync(0xffffffffu, pick, __ffs(b) - 1);
    }
    return kEmpty;
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, v, d);
        v = o < v ? o : v;
    }
    return v;
}


// Per-SM resources of the current device (registers, shared memory incl. the per-CTA
// reserve, threads, CTA slots).
struct SmResources {
    long regs, smem, smem_reserved, threads, blocks;
};

SmResources sm_resources() {
    static SmResources r{};
    static bool done = false;
    if (!done) {
        int dev = 0;
        cudaDeviceProp p{};
        if (cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&p, dev) == cudaSuccess) {
            r = SmResources{p.regsPerMultiprocessor, (long)p.sharedMemPerMultiprocessor, (long)p.reservedSharedMemPerBlock,
                            p.maxThreadsPerMultiProcessor, p.maxBlocksPerMultiProcessor};
            done = true;
        } else {
            cudaGetLastError();
        }
    }
    return r;
}

// Resident CTAs of a persistent kernel: full occupancy on every SM, or - when the engine
// shares the GPU with another stream's persistent kernels - as many CTAs per SM as fit in
// `pct` percent of EVERY per-SM resource (registers at warp allocation granularity, shared
// memory with its per-CTA reserve, threads, CTA slots). Lanes whose percentages add up to
// at most 100 therefore always fit side by side, and neither lane's grid has CTAs waiting
// for the other lane's kernel to finish (a persistent kernel ends only after all of its CTAs
// have started). At least one CTA per SM.
template <typename K>
int persistent_grid(K kernel, size_t smem, int num_sms, int threads = kThreads, int pct = 100) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (pct > 0 && pct < 100) {
        cudaFuncAttributes a{};
        const SmResources R = sm_resources();
        if (cudaFuncGetAttributes(&a, kernel) == cudaSuccess && R.regs > 0) {
            const long warps = (threads + 31) / 32;
            const long cta_regs = warps * (((long)a.numRegs * 32 + 255) / 256) * 256;
            const long cta_smem = (long)a.sharedSizeBytes + (long)smem + R.smem_reserved;
            long cap = pct * R.blocks / 100;
            if (cta_regs > 0) cap = std::min(cap, pct * R.regs / 100 / cta_regs);
            cap = std::min(cap, pct * R.smem / 100 / cta_smem);
            cap = std::min(cap, pct * R.threads / 100 / (warps * 32));
            per_sm = (int)std::min<long>(per_sm, cap);
        } else {
            cudaGetLastError();
            per_sm = per_sm * pct / 100;
        }
    }
    if (per_sm < 1) per_sm = 1;
    return per_sm * num_sms;
}

}  // namespace

}  // namespace rsb
