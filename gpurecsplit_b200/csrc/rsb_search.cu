// Seed searches of RecSplit construction on sm_100a.
//
// Every search returns the minimum seed x >= 0 (counted from the level's start seed) for
// which the node's keys split as required, as SIMDRecSplit does:
//   fanout-2 split      SIMDRecSplit.hpp:250-317   (GPURecSplit.cuh:107-156)
//   aggregation levels  SIMDRecSplit.hpp:319-423   (GPURecSplit.cuh:164-264)
//   leaf, brute force   SIMDRecSplit.hpp:510-599   (GPURecSplit.cuh:351-392)
//   leaf, rotation      SIMDRecSplit.hpp:452-509   (GPURecSplit.cuh:309-350)
//
// Work distribution. Fanout-2 nodes (few, cheap) get one CTA each, which searches and then
// partitions the node in place. Aggregation nodes and leaves are searched by persistent
// warps: a node hands out ascending windows of W candidate seeds from an atomic counter;
// the warp that took the node from the stage list owns it, and warps that run out of fresh
// nodes help unfinished ones (taking further windows of the same node). A window whose
// first seed is not below the node's current best is never evaluated, every other window
// is evaluated completely, and successes are merged with atomicMin — so at kernel end each
// node holds the minimum successful seed, independent of scheduling. No warp ever waits on
// another warp: the kernels contain no spin loops.
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

// ---------------------------------------------------------------------------------------
// Fanout-2 nodes: one CTA per node, search and stable 2-way partition.
// remap(k + x, m) < split  <=>  hash16(k + x) < ceil(split * 2^16 / m).
// ---------------------------------------------------------------------------------------
// A node needs about sqrt(2*pi*m*p*(1-p)) (tens of) seeds, so small CTAs keep the
// last window's overshoot small: 64 threads, one seed each per window.
constexpr int kHigherThreads = 64;
constexpr int kHigherWarps = kHigherThreads / 32;
constexpr int kHigherSeedsPerThread = 1;

__global__ void __launch_bounds__(kHigherThreads) k_search_higher(SearchCtx c, int depth) {
    extern __shared__ uint64_t sk[];
    __shared__ unsigned long long s_best;
    __shared__ uint32_t s_warp[kHigherWarps];
    __shared__ int s_stop;
    const uint32_t count = c.stage_info[depth];
    const uint32_t base = c.stage_info[kNumStages + depth];
    const uint64_t seed = start_seed(depth);
    const uint32_t upper = c.sh.upper;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t li = blockIdx.x; li < count; li += gridDim.x) {
        if (threadIdx.x == 0) s_stop = status_code(c.status);
        __syncthreads();
        if (s_stop) return;
        const uint32_t id = c.lists[base + li];
        const uint32_t start = c.nodes.start[id];
        const uint32_t m = c.nodes.size[id];
        const uint32_t split = upper * (uint16_t(m / 2 + upper - 1) / upper);
        const uint32_t thr = (uint32_t)((((uint64_t)split << 16) + m - 1) / m);
        for (uint32_t i = threadIdx.x; i < m; i += kHigherThreads) sk[i] = c.keys[start + i];
        if (threadIdx.x == 0) s_best = kSeedNotFound;
        __syncthreads();
        const uint64_t budget = budget_for(c, m);
        constexpr uint32_t W = kHigherThreads * kHigherSeedsPerThread;
        bool failed = false;
        for (uint64_t x0 = 0;; x0 += W) {
#pragma unroll
            for (int s = 0; s < kHigherSeedsPerThread; ++s) {
                const uint64_t x = x0 + threadIdx.x + (uint64_t)s * kHigherThreads;
                const uint64_t sx = seed + x;
                uint32_t cnt = 0;
                for (uint32_t i = 0; i < m; ++i) cnt += hash16(sk[i] + sx) < thr;
                if (cnt == split) atomicMin(&s_best, (unsigned long long)x);
            }
            __syncthreads();
            const bool done = s_best != kSeedNotFound;
            __syncthreads();
            if (done) break;
            if (x0 + W >= budget) {
                failed = true;
                break;
            }
        }
        const uint64_t x = failed ? kSeedFailed : (uint64_t)s_best;
        if (threadIdx.x == 0) c.nodes.seed[id] = x;
        if (failed) {
            if (threadIdx.x == 0) set_error(c.status, RSB_ERR_SEARCH_BUDGET, id);
            return;
        }
        // Stable partition: keys remapping below `split` first (SIMDRecSplit.hpp:288-306).
        const uint32_t per = (m + kHigherThreads - 1) / kHigherThreads;
        const uint32_t b0 = min(m, threadIdx.x * per), b1 = min(m, b0 + per);
        const uint64_t sx = seed + x;
        uint32_t left = 0;
        for (uint32_t i = b0; i < b1; ++i) left += hash16(sk[i] + sx) < thr;
        // block exclusive scan of `left`
        uint32_t inc = left;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t o = __shfl_up_sync(0xffffffffu, inc, d);
            if (lane >= d) inc += o;
        }
        if (lane == 31) s_warp[warp] = inc;
        __syncthreads();
        uint32_t wbase = 0;
        for (int w = 0; w < warp; ++w) wbase += s_warp[w];
        uint32_t lpos = wbase + inc - left;
        uint32_t rpos = split + (b0 - lpos);
        for (uint32_t i = b0; i < b1; ++i) {
            const uint64_t k = sk[i];
            if (hash16(k + sx) < thr) c.keys[start + lpos++] = k;
            else c.keys[start + rpos++] = k;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Aggregation levels. Part counts are packed in bytes: parts 0-3 in `lo`, 4-7 in `hi`; with
// fanout 9 the last part is implied by the others. Every target is below 255 and a node
// holds at most fanout * SPLIT keys, so a byte can only carry into the next one on
// candidates that already fail — packed equality is exact equality.
// ---------------------------------------------------------------------------------------
//
// Two-phase evaluation. A seed can only split a node exactly if the sum over its keys of
// the part index equals sum_j j * size_j — a necessary condition that costs one fused
// multiply-add per key on a full node (two integer ops more on other nodes; moment_sums and
// add_part) instead of a packed part count, and that
// about 1 / (2.5 * sqrt(m * var(p))) of the seeds pass (1.9 % at m = 112, fanout 7).
// Phase A applies it to every seed of a window (8 or 12 per lane); the survivors go to a per-warp
// queue in shared memory, and phase B gives each lane one queued seed for the exact part
// count. A warp drains its queue before it leaves a node, so every seed below the node's
// final best is still fully checked and the minimum is unchanged.
// ---------------------------------------------------------------------------------------

// Candidates per lane of a window, by leaf size (measured on one B200): 12 amortise the
// per-key work better where nodes need thousands of candidates or more (l = 16: 253 -> 247
// ns/key; l = 12 batched: +1.5 % keys/s); at l <= 11 a node needs only a few hundred, so the
// larger window's overshoot costs more (l = 8: 1.84 -> 1.93 ms per 1M keys) and 8 stay.
__host__ __device__ constexpr int aggr_seeds_per_lane(int leaf) { return leaf >= 12 ? 12 : 8; }

template <int LEAF, int STAGE>
struct AggrCfg {
    static constexpr int S = aggr_seeds_per_lane(LEAF);
    static constexpr uint32_t W = 32u * S;                  // candidates of one window
    static constexpr int QCAP = 32 + (int)W;                // < 32 pending after a drain + one window
    static constexpr uint32_t SPLIT = STAGE == kStageUpper ? lower_of(LEAF) : (uint32_t)LEAF;
    static constexpr uint32_t MAXM = STAGE == kStageUpper ? upper_of(LEAF) : lower_of(LEAF);
    static constexpr uint32_t MAXF = (MAXM + SPLIT - 1) / SPLIT;
    static constexpr bool WIDE = MAXF > 4;
    static constexpr uint64_t SEED_INDEX = STAGE == kStageUpper ? 17 : 18;
    static constexpr uint32_t WARP_WORDS = MAXM + QCAP + kAbortChunk;  // keys, candidate queue, key terms
    static_assert(129u * MAXF * MAXM < (1u << 23), "full-node accumulator leaves [2^23, 2^24)");
};

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        const uint64_t o = __shfl_xor_sync(0xffffffffu, v, d);
        v = o < v ? o : v;
    }
    return v;
}

// Exact (packed) part counts of one candidate seed sx over the node's keys.
template <int LEAF, int STAGE, bool WIDE>
__device__ __forceinline__ bool aggr_exact(const uint64_t *sk, uint32_t m, uint32_t fan, bool full, uint64_t sx,
                                           uint32_t tlo, uint32_t thi) {
    using C = AggrCfg<LEAF, STAGE>;
    uint32_t lo = 0, hi = 0;
    if (full) {
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t p = (hash16(sk[i] + sx) * fan) >> 16;
            if (WIDE) {
                lo += shl_clamp(1u, 8 * p);
                hi += shl_clamp(1u, 8 * p - 32);
            } else {
                lo += 1u << (8 * p);
            }
        }
    } else {
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t p = ((hash16(sk[i] + sx) * m) >> 16) / C::SPLIT;
            if (WIDE) {
                lo += shl_clamp(1u, 8 * p);
                hi += shl_clamp(1u, 8 * p - 32);
            } else {
                lo += 1u << (8 * p);
            }
        }
    }
    return lo == tlo && (!WIDE || hi == thi);
}

// Phase B: checks the last `take` (<= 32) queued candidates, one per lane, and merges the
// smallest success into the node's seed. Candidates not below `best` cannot lower it.
template <int LEAF, int STAGE>
__device__ __forceinline__ void aggr_drain(const uint64_t *sk, uint64_t *q, uint32_t &qn, uint32_t take, uint32_t m,
                                           uint32_t fan, bool full, uint64_t seed, uint32_t tlo, uint32_t thi,
                                           uint64_t best, uint64_t *node_seed, uint32_t *found) {
    using C = AggrCfg<LEAF, STAGE>;
    const int lane = threadIdx.x & 31;
    const bool active = lane < (int)take;
    const uint64_t x = active ? q[qn - take + lane] : ~0ull;
    __syncwarp();
    bool ok = false;
    if (active && x < best) ok = aggr_exact<LEAF, STAGE, C::WIDE>(sk, m, fan, full, seed + x, tlo, thi);
    const uint64_t v = warp_min_u64(ok ? x : ~0ull);
    if (lane == 0 && v != ~0ull) merge_seed(node_seed, v, found);
    qn -= take;
}

template <int LEAF, int STAGE>
__global__ void __launch_bounds__(kThreads) k_search_aggr(SearchCtx c) {
    using C = AggrCfg<LEAF, STAGE>;
    constexpr int S = C::S;
    constexpr uint32_t W = C::W;
    extern __shared__ uint64_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *sk = smem + warp * C::WARP_WORDS;
    uint64_t *q = sk + C::MAXM;
    uint2 *pk = reinterpret_cast<uint2 *>(q + C::QCAP);
    const unsigned below = (1u << lane) - 1;
    const uint32_t gw = blockIdx.x * kWarpsPerCta + warp;
    const uint32_t count = c.stage_info[STAGE];
    const uint32_t base = c.stage_info[kNumStages + STAGE];
    uint32_t *found = &c.sched[kNumStages + STAGE];  // nodes of this stage with a seed
    const uint64_t seed = start_seed(C::SEED_INDEX);
    uint32_t rng = gw * 2654435761u + 12345u;
    uint32_t node = kEmpty, m = 0, fan = 0, tlo = 0, thi = 0, t1 = 0, mult = 0, qn = 0;
    bool owner = false, full = false;
    uint64_t budget = 0;
    for (;;) {
        if (node == kEmpty) {
            if (status_code(c.status)) break;
            uint32_t f = 0;
            if (lane == 0) f = atomicAdd(&c.sched[STAGE], 1u);
            f = __shfl_sync(0xffffffffu, f, 0);
            if (f < count) {
                node = c.lists[base + f];
                owner = true;
                if (lane == 0) c.slots[gw] = node;
            } else {
                owner = false;
                if (vload32(found) >= count) break;  // every node of the stage has a seed
                rng = rng * 1664525u + 1013904223u;
                node = find_help(c, rng);
                if (node == kEmpty) break;
            }
            const uint32_t start = c.nodes.start[node];
            m = c.nodes.size[node];
            __syncwarp();
            for (uint32_t i = lane; i < m; i += 32) sk[i] = c.keys[start + i];
            __syncwarp();
            fan = uint16_t(m + C::SPLIT - 1) / C::SPLIT;
            full = m == fan * C::SPLIT;
            tlo = thi = 0;
            for (uint32_t j = 0; j < 8 && j < fan; ++j) {
                const uint32_t t = j + 1 < fan ? C::SPLIT : m - (fan - 1) * C::SPLIT;
                if (j < 4) tlo |= t << (8 * j);
                else thi |= t << (8 * (j - 4));
            }
            // phase A target: sum_j j * size_j, in add_part's form; part-index multiplier of
            // non-full nodes
            mult = (uint32_t)((((uint64_t)m << 28) + C::SPLIT - 1) / C::SPLIT);
            t1 = full ? kAccF0 + 128u * fan * m : 0u;
            for (uint32_t j = 1; j < fan; ++j) t1 += j * (j + 1 < fan ? C::SPLIT : m - (fan - 1) * C::SPLIT);
            budget = budget_for(c, m);
            qn = 0;
        }
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(&c.nodes.next_win[node], 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        const uint64_t x0 = (uint64_t)w * W;
        uint64_t best = vload64(&c.nodes.seed[node]);
        if (x0 >= best || x0 >= budget) {
            while (qn > 0) {
                best = vload64(&c.nodes.seed[node]);
                aggr_drain<LEAF, STAGE>(sk, q, qn, min(qn, 32u), m, fan, full, seed, tlo, thi, best, &c.nodes.seed[node], found);
            }
            if (x0 < best && lane == 0) merge_seed(&c.nodes.seed[node], kSeedFailed, found);
            if (owner && lane == 0) c.slots[gw] = kEmpty;
            node = kEmpty;
            continue;
        }
        // phase A: part-index sums for S seeds per lane (seeds x0 + lane + 32 s)
        uint32_t cnt[S];
#pragma unroll
        for (int s = 0; s < S; ++s) cnt[s] = full ? kAccF0 : 0u;
        // The keys go in chunks; after each chunk the window is abandoned if the node's best
        // seed has dropped to x0 or below (another warp succeeded below this window), since
        // then none of its candidates can lower the minimum.
        bool abandoned = false;
        for (uint32_t i0 = 0; i0 < m; i0 += kAbortChunk) {
            const uint32_t len = min(kAbortChunk, m - i0);
            if (full) moment_sums<S, true>(sk + i0, len, seed + x0, fan, pk, cnt);
            else moment_sums<S, false>(sk + i0, len, seed + x0, mult, pk, cnt);
            if (i0 + len < m) {
                uint64_t b = 0;
                if (lane == 0) b = vload64(&c.nodes.seed[node]);
                if (__shfl_sync(0xffffffffu, b, 0) <= x0) {
                    abandoned = true;
                    break;
                }
            }
        }
        if (abandoned) continue;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const bool pass = cnt[s] == t1;
            const unsigned b = __ballot_sync(0xffffffffu, pass);
            if (pass) q[qn + __popc(b & below)] = x0 + lane + 32u * s;
            qn += __popc(b);
        }
        __syncwarp();
        while (qn >= 32) {
            best = vload64(&c.nodes.seed[node]);
            aggr_drain<LEAF, STAGE>(sk, q, qn, 32u, m, fan, full, seed, tlo, thi, best, &c.nodes.seed[node], found);
        }
    }
}

// Stable fanout-way partition of aggregation nodes once their stage is complete
// (SIMDRecSplit.hpp:395-412), one warp per node.
template <int LEAF, int STAGE>
__global__ void __launch_bounds__(kThreads) k_partition_aggr(SearchCtx c) {
    using C = AggrCfg<LEAF, STAGE>;
    extern __shared__ uint64_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *sk = smem + warp * C::MAXM;
    const uint32_t count = c.stage_info[STAGE];
    const uint32_t base = c.stage_info[kNumStages + STAGE];
    const uint64_t seed = start_seed(C::SEED_INDEX);
    const uint32_t nwarps = gridDim.x * kWarpsPerCta;
    for (uint32_t li = blockIdx.x * kWarpsPerCta + warp; li < count; li += nwarps) {
        const uint32_t id = c.lists[base + li];
        const uint64_t x = c.nodes.seed[id];
        if (x >= kSeedFailed) {
            if (lane == 0) set_error(c.status, RSB_ERR_SEARCH_BUDGET, id);
            continue;
        }
        const uint32_t start = c.nodes.start[id];
        const uint32_t m = c.nodes.size[id];
        for (uint32_t i = lane; i < m; i += 32) sk[i] = c.keys[start + i];
        __syncwarp();
        const uint32_t fan = uint16_t(m + C::SPLIT - 1) / C::SPLIT;
        uint32_t cur[C::MAXF];
#pragma unroll
        for (uint32_t j = 0; j < C::MAXF; ++j) cur[j] = j * C::SPLIT;
        const uint64_t sx = seed + x;
        for (uint32_t c0 = 0; c0 < m; c0 += 32) {
            const uint32_t i = c0 + lane;
            const bool valid = i < m;
            const uint64_t k = valid ? sk[i] : 0;
            const uint32_t p = valid ? remap16(k + sx, m) / C::SPLIT : 0xFFu;
            uint32_t dst = 0;
#pragma unroll
            for (uint32_t j = 0; j < C::MAXF; ++j) {
                if (j < fan) {
                    const unsigned b = __ballot_sync(0xffffffffu, p == j);
                    if (p == j) dst = cur[j] + __popc(b & ((1u << lane) - 1));
                    cur[j] += __popc(b);
                }
            }
            if (valid) c.keys[start + dst] = k;
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------------------
// Leaves. Rotation leaves (m == LEAF): left = even `second`, right = odd; for base b the
// encoded seed is b*LEAF + r with r the least left rotation of the right mask that fills
// the complement of the left mask. A base can only succeed if the left keys land on
// distinct bits, so phase A computes the left mask of every base and queues (base, mask)
// for the few collision-free ones; phase B computes their right masks and rotations.
// Brute-force leaves: the first x whose m bit positions are all distinct.
// ---------------------------------------------------------------------------------------
constexpr int kLeafSeedsPerLane = 8;
constexpr int kLeafQueueCap = 32 + 32 * kLeafSeedsPerLane;

template <int LEAF>
__device__ __forceinline__ uint32_t rotl_leaf(uint32_t v, uint32_t r) {
    constexpr uint32_t full = (LEAF == 32) ? 0xFFFFFFFFu : ((1u << LEAF) - 1);
    return ((v << r) | (v >> (LEAF - r))) & full;
}

// Left-mask sums (add_bit) of the S bases x0 + lane + 32 s of a rotation-leaf window
// (bu = SEED + x0*LEAF) over the nl < 32 left keys sk[0, nl), with moment_sums' per-key terms:
// the window spans 32*S*LEAF seeds, each key's (K', L) goes to pk[0, nf) and the indexes of
// keys whose low half can overflow within the window to pk[LEAF - ns, LEAF).
template <int LEAF, int S>
__device__ __forceinline__ void left_masks(const uint64_t *sk, uint32_t nl, uint64_t bu, uint2 *pk, uint32_t *ml) {
    constexpr uint32_t kSpan = 32u * S * LEAF;
    static_assert(kSpan <= 0x10000u, "window wider than the hoisting allows");
    const uint32_t lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1;
    const bool valid = lane < nl;
    const uint64_t tu = (valid ? sk[lane] : 0) + bu;
    const uint32_t lo = (uint32_t)tu, hi = (uint32_t)(tu >> 32);
    const bool fast = (lo & 0xFFFFu) <= 0x10000u - kSpan;
    const unsigned bf = __ballot_sync(0xffffffffu, valid && fast);
    const unsigned bs = __ballot_sync(0xffffffffu, valid && !fast);
    if (valid && fast)
        pk[__popc(bf & below)] = make_uint2(hi ^ (hi >> 16) ^ (lo >> 16) ^ (lo & 0xFFFF0000u), lo & 0xFFFFu);
    if (valid && !fast) pk[LEAF - 1 - __popc(bs & below)].x = lane;
    const uint32_t nf = __popc(bf), ns = __popc(bs);
    __syncwarp();
#pragma unroll 2
    for (uint32_t i = 0; i < nf; ++i) {
        const uint2 e = pk[i];
        const uint32_t l0 = e.y + lane * LEAF;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            uint32_t z = (l0 + 32u * s * LEAF) ^ e.x;
            z *= 0x85ebca6bu;
            z ^= z >> 13;
            add_bit<LEAF>(z * 0xc2b2ae35u, ml[s]);
        }
    }
    for (uint32_t i = 0; i < ns; ++i) {
        const uint64_t t = sk[pk[LEAF - 1 - i].x] + bu;
#pragma unroll
        for (int s = 0; s < S; ++s) {
            const uint64_t v = t + (lane + 32u * s) * LEAF;
            add_bit<LEAF>(remix32_core(uint32_t(v >> 32) ^ uint32_t(v)), ml[s]);
        }
    }
    __syncwarp();  // pk is rewritten by the next window
}

// Phase B of rotation leaves: each lane takes one queued (base, left mask).
template <int LEAF>
__device__ __forceinline__ void leaf_drain(const uint64_t *sk, uint32_t nl, const uint64_t *qb, const uint32_t *qm,
                                           uint32_t &qn, uint32_t take, uint64_t seed, uint64_t best,
                                           uint64_t *node_seed, uint32_t *found) {
    constexpr uint32_t full = (1u << LEAF) - 1;
    const int lane = threadIdx.x & 31;
    const bool active = lane < (int)take;
    const uint64_t b = active ? qb[qn - take + lane] : 0;
    const uint32_t ml = active ? qm[qn - take + lane] : 0;
    __syncwarp();
    uint64_t enc = ~0ull;
    if (active && b * LEAF < best) {
        const uint64_t bx = seed + b * LEAF;
        uint32_t mr = 0;
        for (uint32_t i = nl; i < (uint32_t)LEAF; ++i) mr |= 1u << remap16(sk[i] + bx, LEAF);
        if (__popc(mr) == LEAF - (int)nl) {
            const uint32_t want = full & ~ml;
            for (uint32_t r = 0; r < (uint32_t)LEAF; ++r) {
                if (rotl_leaf<LEAF>(mr, r) == want) {
                    enc = b * LEAF + r;
                    break;
                }
            }
        }
    }
    enc = warp_min_u64(enc);
    if (lane == 0 && enc != ~0ull) merge_seed(node_seed, enc, found);
    qn -= take;
}

template <int LEAF, bool ROT>
__global__ void __launch_bounds__(kThreads) k_search_leaf(SearchCtx c) {
    constexpr int STAGE = ROT ? kStageLeafRot : kStageLeafBF;
    constexpr int S = kLeafSeedsPerLane;
    constexpr uint32_t W = 32 * S;
    __shared__ uint64_t skeys[kWarpsPerCta][LEAF];
    __shared__ uint2 s_pk[ROT ? kWarpsPerCta : 1][ROT ? LEAF : 1];
    __shared__ uint64_t s_qb[ROT ? kWarpsPerCta : 1][ROT ? kLeafQueueCap : 1];
    __shared__ uint32_t s_qm[ROT ? kWarpsPerCta : 1][ROT ? kLeafQueueCap : 1];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t *sk = skeys[warp];
    uint64_t *qb = s_qb[ROT ? warp : 0];
    uint32_t *qm = s_qm[ROT ? warp : 0];
    uint32_t qn = 0;
    const uint32_t gw = blockIdx.x * kWarpsPerCta + warp;
    const uint32_t count = c.stage_info[STAGE];
    const uint32_t base = c.stage_info[kNumStages + STAGE];
    uint32_t *found = &c.sched[kNumStages + STAGE];  // nodes of this stage with a seed
    const uint64_t seed = start_seed(kNumStartSeeds - 1);
    uint32_t rng = gw * 2654435761u + 777u;
    uint32_t node = kEmpty, m = 0, nl = 0;
    bool owner = false;
    uint64_t budget = 0;
    for (;;) {
        if (node == kEmpty) {
            if (status_code(c.status)) break;
            uint32_t f = 0;
            if (lane == 0) f = atomicAdd(&c.sched[STAGE], 1u);
            f = __shfl_sync(0xffffffffu, f, 0);
            if (f < count) {
                node = c.lists[base + f];
                owner = true;
                if (lane == 0) c.slots[gw] = node;
            } else {
                owner = false;
                if (vload32(found) >= count) break;  // every node of the stage has a seed
                rng = rng * 1664525u + 1013904223u;
                node = find_help(c, rng);
                if (node == kEmpty) break;
            }
            const uint32_t start = c.nodes.start[node];
            m = c.nodes.size[node];
            const uint64_t k = lane < (int)m ? c.keys[start + lane] : 0;
            __syncwarp();
            if (ROT) {
                const unsigned even = __ballot_sync(0xffffffffu, lane < (int)m && (k & 1) == 0);
                const unsigned odd = __ballot_sync(0xffffffffu, lane < (int)m && (k & 1) == 1);
                nl = __popc(even);
                const unsigned below = (1u << lane) - 1;
                if (lane < (int)m) sk[(k & 1) ? nl + __popc(odd & below) : __popc(even & below)] = k;
            } else {
                if (lane < (int)m) sk[lane] = k;
            }
            __syncwarp();
            budget = budget_for(c, m);
            qn = 0;
        }
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(&c.nodes.next_win[node], 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        const uint64_t x0 = (uint64_t)w * W;                   // first base (ROT) or seed of the window
        const uint64_t enc0 = ROT ? x0 * LEAF : x0;            // first encoded seed of the window
        uint64_t best = vload64(&c.nodes.seed[node]);
        if (enc0 >= best || enc0 >= budget) {
            if (ROT) {
                while (qn > 0) {
                    best = vload64(&c.nodes.seed[node]);
                    leaf_drain<LEAF>(sk, nl, qb, qm, qn, min(qn, 32u), seed, best, &c.nodes.seed[node], found);
                }
            }
            if (enc0 < best && lane == 0) merge_seed(&c.nodes.seed[node], kSeedFailed, found);
            if (owner && lane == 0) c.slots[gw] = kEmpty;
            node = kEmpty;
            continue;
        }
        uint32_t off = 0xFFFFFFFFu;
        if (ROT) {
            // phase A: left-mask sums of S bases per lane; queue the collision-free ones
            const unsigned below = (1u << lane) - 1;
            uint32_t ml[S];
#pragma unroll
            for (int s = 0; s < S; ++s) ml[s] = 0;
            left_masks<LEAF, S>(sk, nl, seed + x0 * LEAF, s_pk[ROT ? warp : 0], ml);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint64_t b = x0 + lane + 32u * s;
                const uint32_t mk = left_mask_of<LEAF>(ml[s], nl);
                const bool pass = mk != ~0u;
                const unsigned bal = __ballot_sync(0xffffffffu, pass);
                if (pass) {
                    qb[qn + __popc(bal & below)] = b;
                    qm[qn + __popc(bal & below)] = mk;
                }
                qn += __popc(bal);
            }
            __syncwarp();
            while (qn >= 32) {
                best = vload64(&c.nodes.seed[node]);
                leaf_drain<LEAF>(sk, nl, qb, qm, qn, 32u, seed, best, &c.nodes.seed[node], found);
            }
            continue;
        } else {
            const uint32_t full = (1u << m) - 1;
#pragma unroll
            for (int s = S - 1; s >= 0; --s) {
                const uint64_t bx = seed + x0 + lane + 32u * s;
                uint32_t mask = 0;
                for (uint32_t i = 0; i < m; ++i) mask |= 1u << remap16(sk[i] + bx, m);
                if (mask == full) off = lane + 32u * s;
            }
        }
        off = __reduce_min_sync(0xffffffffu, off);
        if (off != 0xFFFFFFFFu && lane == 0)
            merge_seed(&c.nodes.seed[node], enc0 + off, found);
    }
}

// ---- host-side dispatch -------------------------------------------------------------

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

template <int LEAF>
void run_aggr(const SearchCtx &c, int stage, cudaStream_t st) {
    if (stage == kStageUpper) {
        using C = AggrCfg<LEAF, kStageUpper>;
        const size_t smem = kWarpsPerCta * C::WARP_WORDS * sizeof(uint64_t);
        auto k = k_search_aggr<LEAF, kStageUpper>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int g = persistent_grid(k, smem, c.num_sms, kThreads, c.occupancy_pct);
        g = min(g, (int)(c.nslots / kWarpsPerCta));
        SearchCtx cc = c;
        cc.nslots = g * kWarpsPerCta;
        use_max_smem(k);
        k<<<g, kThreads, smem, st>>>(cc);
    } else {
        using C = AggrCfg<LEAF, kStageLower>;
        const size_t smem = kWarpsPerCta * C::WARP_WORDS * sizeof(uint64_t);
        auto k = k_search_aggr<LEAF, kStageLower>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int g = persistent_grid(k, smem, c.num_sms, kThreads, c.occupancy_pct);
        g = min(g, (int)(c.nslots / kWarpsPerCta));
        SearchCtx cc = c;
        cc.nslots = g * kWarpsPerCta;
        use_max_smem(k);
        k<<<g, kThreads, smem, st>>>(cc);
    }
}

template <int LEAF>
void run_partition(const SearchCtx &c, int stage, cudaStream_t st) {
    if (stage == kStageUpper) {
        using C = AggrCfg<LEAF, kStageUpper>;
        const size_t smem = kWarpsPerCta * C::MAXM * sizeof(uint64_t);
        auto k = k_partition_aggr<LEAF, kStageUpper>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        use_max_smem(k);
        k<<<persistent_grid(k, smem, c.num_sms, kThreads, c.occupancy_pct), kThreads, smem, st>>>(c);
    } else {
        using C = AggrCfg<LEAF, kStageLower>;
        const size_t smem = kWarpsPerCta * C::MAXM * sizeof(uint64_t);
        auto k = k_partition_aggr<LEAF, kStageLower>;
        cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        use_max_smem(k);
        k<<<persistent_grid(k, smem, c.num_sms, kThreads, c.occupancy_pct), kThreads, smem, st>>>(c);
    }
}

template <int LEAF>
void run_leaves(const SearchCtx &c, int stage, cudaStream_t st) {
    SearchCtx cc = c;
    if (stage == kStageLeafRot) {
        auto k = k_search_leaf<LEAF, true>;
        int g = min(persistent_grid(k, 0, c.num_sms, kThreads, c.occupancy_pct), (int)(c.nslots / kWarpsPerCta));
        cc.nslots = g * kWarpsPerCta;
        use_max_smem(k);
        k<<<g, kThreads, 0, st>>>(cc);
    } else {
        auto k = k_search_leaf<LEAF, false>;
        int g = min(persistent_grid(k, 0, c.num_sms, kThreads, c.occupancy_pct), (int)(c.nslots / kWarpsPerCta));
        cc.nslots = g * kWarpsPerCta;
        use_max_smem(k);
        k<<<g, kThreads, 0, st>>>(cc);
    }
}

#define RSB_LEAF_SWITCH(leaf, FN, ...)          \
    switch (leaf) {                             \
        case 2: FN<2>(__VA_ARGS__); break;      \
        case 3: FN<3>(__VA_ARGS__); break;      \
        case 4: FN<4>(__VA_ARGS__); break;      \
        case 5: FN<5>(__VA_ARGS__); break;      \
        case 6: FN<6>(__VA_ARGS__); break;      \
        case 7: FN<7>(__VA_ARGS__); break;      \
        case 8: FN<8>(__VA_ARGS__); break;      \
        case 9: FN<9>(__VA_ARGS__); break;      \
        case 10: FN<10>(__VA_ARGS__); break;    \
        case 11: FN<11>(__VA_ARGS__); break;    \
        case 12: FN<12>(__VA_ARGS__); break;    \
        case 13: FN<13>(__VA_ARGS__); break;    \
        case 14: FN<14>(__VA_ARGS__); break;    \
        case 15: FN<15>(__VA_ARGS__); break;    \
        case 16: FN<16>(__VA_ARGS__); break;    \
        case 17: FN<17>(__VA_ARGS__); break;    \
        case 18: FN<18>(__VA_ARGS__); break;    \
        case 19: FN<19>(__VA_ARGS__); break;    \
        case 20: FN<20>(__VA_ARGS__); break;    \
        case 21: FN<21>(__VA_ARGS__); break;    \
        case 22: FN<22>(__VA_ARGS__); break;    \
        case 23: FN<23>(__VA_ARGS__); break;    \
        case 24: FN<24>(__VA_ARGS__); break;    \
        default: break;                         \
    }

}  // namespace

uint32_t search_slots_needed(int num_sms) { return (uint32_t)num_sms * 64u; }  // 64 resident warps per SM at most

uint32_t window_candidates(int leaf, int stage) {
    if (stage == kStageUpper || stage == kStageLower) return 32u * aggr_seeds_per_lane(leaf);
    if (stage == kStageLeafRot || stage == kStageLeafBF) return 32u * kLeafSeedsPerLane;
    return 0;
}

bool shape_matches_kernels(const Shape &s) { return s.lower == lower_of((int)s.leaf) && s.upper == upper_of((int)s.leaf); }

void search_higher(const SearchCtx &c, int depth, cudaStream_t st) {
    const size_t smem = kMaxBucketSize * sizeof(uint64_t);
    cudaFuncSetAttribute(k_search_higher, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    use_max_smem(k_search_higher);
    k_search_higher<<<persistent_grid(k_search_higher, smem, c.num_sms, kHigherThreads, c.occupancy_pct), kHigherThreads, smem, st>>>(c,
                                                                                                           depth);
    count_launches(1);
}

void search_aggr(const SearchCtx &c, int stage, cudaStream_t st) {
    RSB_LEAF_SWITCH(c.sh.leaf, run_aggr, c, stage, st);
    count_launches(1);
}
void partition_aggr(const SearchCtx &c, int stage, cudaStream_t st) {
    RSB_LEAF_SWITCH(c.sh.leaf, run_partition, c, stage, st);
    count_launches(1);
}
void search_leaves(const SearchCtx &c, int stage, cudaStream_t st) {
    RSB_LEAF_SWITCH(c.sh.leaf, run_leaves, c, stage, st);
    count_launches(1);
}

// ---- eval-rate probe ------------------------------------------------------------------
// The cheapest complete candidate evaluation of any search (key + seed, remix32, 16-bit
// remap to a part index, sum) in the exact form of the aggregation filter (moment_sums on a
// full node in chunks of kAbortChunk keys: per-key terms in shared memory, 12 candidates per
// lane, unrolled key loop), run at full occupancy with no scheduling, no queues and no
// reductions: the ceiling for remixAndRemap32 evaluations on this device.
namespace {
constexpr uint32_t kProbeKeys = 128;
constexpr int kProbeIters = 32;
constexpr int kProbeSeeds = 12;
__global__ void __launch_bounds__(kThreads) k_probe(unsigned long long *sink) {
    __shared__ uint64_t sk[kProbeKeys];
    __shared__ uint2 pk[kWarpsPerCta][kAbortChunk];
    for (int i = threadIdx.x; i < kProbeKeys; i += kThreads) sk[i] = start_seed(i % 20) * (2 * i + 1);
    __syncthreads();
    uint32_t cnt[kProbeSeeds];
#pragma unroll
    for (int s = 0; s < kProbeSeeds; ++s) cnt[s] = kAccF0;
    uint64_t bu = start_seed(17) + (blockIdx.x * (uint64_t)kWarpsPerCta + (threadIdx.x >> 5)) * 32 * kProbeSeeds;
    for (int it = 0; it < kProbeIters; ++it) {
#pragma unroll 1
        for (uint32_t i0 = 0; i0 < kProbeKeys; i0 += kAbortChunk)
            moment_sums<kProbeSeeds, true>(sk + i0, kAbortChunk, bu, 7u, pk[threadIdx.x >> 5], cnt);
        bu += 1ull << 32;
    }
    uint32_t tot = 0;
#pragma unroll
    for (int s = 0; s < kProbeSeeds; ++s) tot += cnt[s];
    if (tot == 0xFFFFFFFFu) atomicAdd(sink, 1ull);  // keeps the loop alive
}
}  // namespace

void probe_eval_rate(int num_sms, uint64_t *out_evals, cudaStream_t st) {
    const int g = persistent_grid(k_probe, 0, num_sms) * 4;
    unsigned long long *sink = nullptr;
    cudaMallocAsync((void **)&sink, 8, st);
    use_max_smem(k_probe);
    k_probe<<<g, kThreads, 0, st>>>(sink);
    cudaFreeAsync(sink, st);
    count_launches(1);
    *out_evals = (uint64_t)g * kThreads * kProbeIters * kProbeKeys * kProbeSeeds;
}

}  // namespace rsb
