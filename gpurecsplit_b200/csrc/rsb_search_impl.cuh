// Aggregation and leaf seed searches (persistent warps), templated on the leaf size and on the
// candidates per lane of a window; rsb_search_inst_*.cu instantiate them per leaf size and
// rsb_search.cu dispatches to them with the engine's schedule.
#pragma once

#include "rsb_search_common.cuh"
#include "rsb_search_stages.h"

namespace rsb {

namespace {

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
// Phase A applies it to every seed of a window (4, 8, 12 or 16 per lane); the survivors go to a
// per-warp queue in shared memory, and phase B gives each lane one queued seed for the exact
// part count, lowest seeds first, before the warp takes its next window (aggr_phase_b), so
// every seed below the node's final best is fully checked and the minimum is unchanged.
// ---------------------------------------------------------------------------------------

// S = candidates per lane of a window (a stage schedule parameter, StageSchedule): larger
// windows amortise the per-key work of a window over more candidates, smaller ones overshoot
// a node's minimum seed by less.
template <int LEAF, int STAGE, int S_ = 8>
struct AggrCfg {
    static constexpr int S = S_;
    static constexpr uint32_t W = 32u * S;                  // candidates of one window
    static constexpr int QCAP = 32 + (int)W;                // < 32 carried over + one window's survivors
    static constexpr uint32_t SPLIT = STAGE == kStageUpper ? lower_of(LEAF) : (uint32_t)LEAF;
    static constexpr uint32_t MAXM = STAGE == kStageUpper ? upper_of(LEAF) : lower_of(LEAF);
    static constexpr uint32_t MAXF = (MAXM + SPLIT - 1) / SPLIT;
    static constexpr bool WIDE = MAXF > 4;
    static constexpr uint64_t SEED_INDEX = STAGE == kStageUpper ? 17 : 18;
    static constexpr uint32_t WARP_WORDS = MAXM + QCAP + kAbortChunk;  // keys, candidate queue, key terms
    static_assert(129u * MAXF * MAXM < (1u << 23), "full-node accumulator leaves [2^23, 2^24)");
};


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

// Phase B: checks the candidates q[0, take) (take <= 32), one per lane, merges the smallest
// success into the node's seed and returns whether there was one. Candidates not below
// `best` cannot lower it.
template <int LEAF, int STAGE>
__device__ __forceinline__ bool aggr_check(const uint64_t *sk, const uint64_t *q, uint32_t take, uint32_t m,
                                           uint32_t fan, bool full, uint64_t seed, uint32_t tlo, uint32_t thi,
                                           uint64_t best, uint64_t *node_seed, uint32_t *found) {
    using C = AggrCfg<LEAF, STAGE>;
    const int lane = threadIdx.x & 31;
    const bool active = lane < (int)take;
    const uint64_t x = active ? q[lane] : ~0ull;
    bool ok = false;
    if (active && x < best) ok = aggr_exact<LEAF, STAGE, C::WIDE>(sk, m, fan, full, seed + x, tlo, thi);
    const uint64_t v = warp_min_u64(ok ? x : ~0ull);
    if (lane == 0 && v != ~0ull) merge_seed(node_seed, v, found);
    return v != ~0ull;
}

// Phase B of the queued candidates q[0, qn) (ascending): lowest first, 32 at a time, while more
// than `keep` are queued, until a batch holds a success (every later candidate is larger) or
// the node's best is at or below the next candidate; then nothing queued can lower the seed and
// the queue is emptied. Checked batches leave the queue (the rest moves down).
//
// How many a window leaves queued is the node's choice (search_eagerly): a node expected to
// need few windows checks all of its survivors before its next window (keep = 0), so that its
// seed is known at once - survivors carried over would let the warp search on past a minimum
// that sits in its own queue, which at l = 12 doubled the windows per node; a node expected to
// need hundreds of windows checks full batches only (keep = 31), since a partial batch of a
// few survivors costs as much as a full one.
template <int LEAF, int STAGE>
__device__ __forceinline__ void aggr_phase_b(const uint64_t *sk, uint64_t *q, uint32_t &qn, uint32_t keep, uint32_t m,
                                             uint32_t fan, bool full, uint64_t seed, uint32_t tlo, uint32_t thi,
                                             uint64_t *node_seed, uint32_t *found) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t qh = 0;
    while (qn - qh > keep) {
        const uint64_t best = warp_load64(node_seed);
        const uint32_t take = min(qn - qh, 32u);
        if (q[qh] >= best ||
            aggr_check<LEAF, STAGE>(sk, q + qh, take, m, fan, full, seed, tlo, thi, best, node_seed, found)) {
            qn = 0;
            return;
        }
        qh += take;
    }
    // the (fewer than 32) unchecked candidates move to the front; qh >= 32 > their count
    const uint32_t rest = qn - qh;
    if (qh > 0 && rest > 0) {
        const uint64_t v = lane < rest ? q[qh + lane] : 0;
        __syncwarp();
        if (lane < rest) q[lane] = v;
        __syncwarp();
    }
    qn = rest;
}

// Whether a node checks every window's survivors before its next window (keep = 0 above): its
// Golomb-Rice parameter g puts its expected seed near 2^g; `window` is the window's width in
// the same units (seeds, or encoded seeds b * LEAF + r of rotation leaves).
__device__ __forceinline__ bool search_eagerly(const SearchCtx &c, uint32_t m, uint64_t window) {
    return (1ull << (c.tab.memo[m] >> 27)) <= 32ull * window;
}

template <int LEAF, int STAGE, int S_>
__global__ void __launch_bounds__(kThreads) k_search_aggr(SearchCtx c) {
    using C = AggrCfg<LEAF, STAGE, S_>;
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
    uint32_t node = kEmpty, m = 0, fan = 0, tlo = 0, thi = 0, t1 = 0, mult = 0, qn = 0, keep = 0;
    bool owner = false, full = false;
    uint64_t budget = 0;
    for (;;) {
        if (node == kEmpty) {
            if (warp_status(c.status)) break;
            uint32_t f = 0;
            if (lane == 0) f = atomicAdd(&c.sched[STAGE], 1u);
            f = __shfl_sync(0xffffffffu, f, 0);
            if (f < count) {
                node = c.lists[base + f];
                owner = true;
                if (lane == 0) c.slots[gw] = node;
            } else {
                owner = false;
                if (warp_load32(found) >= count) break;  // every node of the stage has a seed
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
            keep = search_eagerly(c, m, W) ? 0 : 31;
        }
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(&c.nodes.next_win[node], 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        const uint64_t x0 = (uint64_t)w * W;
        const uint64_t best = warp_load64(&c.nodes.seed[node]);
        if (x0 >= best || x0 >= budget) {
            aggr_phase_b<LEAF, STAGE>(sk, q, qn, 0, m, fan, full, seed, tlo, thi, &c.nodes.seed[node], found);
            if (x0 < warp_load64(&c.nodes.seed[node]) && lane == 0) merge_seed(&c.nodes.seed[node], kSeedFailed, found);
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
        // The warp stays on the node after a success here: its next window starts above the seed
        // and ends the node for it (leaving at once measured 6 % slower on 200k-key l = 24 builds).
        aggr_phase_b<LEAF, STAGE>(sk, q, qn, keep, m, fan, full, seed, tlo, thi, &c.nodes.seed[node], found);
        __syncwarp();  // q is appended to by the next window
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
// the complement of the left mask. A base can only succeed if both halves land on distinct
// bits, so phase A computes the mask of one half for every base and queues (base, mask) for
// the collision-free ones; phase B computes the other half's mask of those, phase C the
// rotation. Phase A takes the larger half (the odd keys when there are more of them): its
// keys collide more often, so fewer bases reach the per-base work of phase B - for a leaf
// of 3 even and 9 odd keys at l = 12, 1.5 % of the bases instead of 76 %.
// Brute-force leaves: the first x whose m bit positions are all distinct.
// ---------------------------------------------------------------------------------------
// Rotation leaves: S bases per lane of a window (a stage schedule parameter); the queue holds
// the survivors of one window plus fewer than 32 carried over (leaf_phase_bc).
template <int S> __host__ __device__ constexpr int leaf_queue_cap() { return 32 + 32 * S; }

template <int LEAF>
__device__ __forceinline__ uint32_t rotl_leaf(uint32_t v, uint32_t r) {
    constexpr uint32_t full = (LEAF == 32) ? 0xFFFFFFFFu : ((1u << LEAF) - 1);
    return ((v << r) | (v >> (LEAF - r))) & full;
}

// Mask sums (add_bit) of the S bases x0 + lane + 32 s of a rotation-leaf window
// (bu = SEED + x0*LEAF) over the nl phase-A keys sk[0, nl), with moment_sums' per-key terms:
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

// Phase B of rotation leaves: each lane takes one queued (base, left mask) of qb/qm[0, take)
// and computes the base's right mask; the bases whose right keys also land on distinct bits
// go, with both masks, to the rotation queue cb/cm[0, cn) for phase C, in the same order.
// Bases not below `best` cannot lower it.
constexpr uint32_t kRotQueueCap = 64;  // < 32 carried over + the phase-B passes of one batch

// The keys are ordered phase-A half first (na keys) and `odd_first` says which half that is;
// the rotation queue holds (left mask, right mask) whichever half came first.
template <int LEAF>
__device__ __forceinline__ uint32_t leaf_check(const uint64_t *sk, uint32_t na, bool odd_first, const uint64_t *qb,
                                               const uint32_t *qm, uint32_t take, uint64_t seed, uint64_t best,
                                               uint64_t *cb, uint2 *cm) {
    const int lane = threadIdx.x & 31;
    const bool active = lane < (int)take;
    const uint64_t b = active ? qb[lane] : 0;
    const uint32_t ml = active ? qm[lane] : 0;
    bool pass = false;
    uint32_t mr = 0;
    if (active && b * LEAF < best) {
        const uint64_t bx = seed + b * LEAF;
        for (uint32_t i = na; i < (uint32_t)LEAF; ++i) mr |= 1u << remap16(sk[i] + bx, LEAF);
        pass = __popc(mr) == LEAF - (int)na;
    }
    const unsigned bal = __ballot_sync(0xffffffffu, pass);
    if (pass) {
        const uint32_t at = __popc(bal & ((1u << lane) - 1));
        cb[at] = b;
        cm[at] = odd_first ? make_uint2(mr, ml) : make_uint2(ml, mr);
    }
    __syncwarp();
    return __popc(bal);
}

// Phase C: each lane takes one base of cb/cm[0, cn) whose halves are both collision-free and
// finds the least left rotation r of the right mask that fills the complement of the left
// mask; the warp's least b * LEAF + r is merged into the node's seed. Returns whether there
// was one.
template <int LEAF>
__device__ __forceinline__ bool rot_check(const uint64_t *cb, const uint2 *cm, uint32_t cn, uint64_t best,
                                          uint64_t *node_seed, uint32_t *found) {
    constexpr uint32_t full = (1u << LEAF) - 1;
    const int lane = threadIdx.x & 31;
    const bool active = lane < (int)cn;
    const uint64_t b = active ? cb[lane] : 0;
    const uint2 mk = active ? cm[lane] : make_uint2(0, 0);
    uint64_t enc = ~0ull;
    if (active && b * LEAF < best) {
        const uint32_t want = full & ~mk.x;
        for (uint32_t r = 0; r < (uint32_t)LEAF; ++r) {
            if (rotl_leaf<LEAF>(mk.y, r) == want) {
                enc = b * LEAF + r;
                break;
            }
        }
    }
    enc = warp_min_u64(enc);
    if (lane == 0 && enc != ~0ull) merge_seed(node_seed, enc, found);
    __syncwarp();  // cb/cm are rewritten by the next batch
    return enc != ~0ull;
}

// Phases B and C of the queued bases qb/qm[0, qn) (ascending), as aggr_phase_b: phase B takes
// them lowest first, 32 at a time, while more than `keep` are queued; its passes collect in the
// rotation queue cb/cm, which phase C checks whenever it holds more than `ckeep` (up to 32 at a
// time) and, at the end, whatever is left. A phase-C batch with a success ends the checks (every
// later base is larger, and so is its encoded seed b * LEAF + r), as does a best below the next
// queued base. ckeep = 0 suits leaves that succeed within a window (each phase-B batch may hold
// the seed and end the window early), 31 the others (full phase-C batches). Returns true when
// the leaf's seed is known to lie below the next window (a success here, or a best at or below a
// queued base): the warp can leave the leaf without taking another window.
template <int LEAF>
__device__ __forceinline__ bool leaf_phase_bc(const uint64_t *sk, uint32_t na, bool odd_first, uint64_t *qb,
                                              uint32_t *qm, uint32_t &qn,
                                              uint32_t keep, uint32_t ckeep, uint64_t seed, uint64_t *cb, uint2 *cm,
                                              uint64_t *node_seed, uint32_t *found) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t qh = 0, cn = 0;
    bool spent = false;  // every base still queued is at or above the best
    while (qn - qh > keep) {
        const uint64_t best = warp_load64(node_seed);
        if (qb[qh] * LEAF >= best) {
            spent = true;
            break;
        }
        const uint32_t take = min(qn - qh, 32u);
        cn += leaf_check<LEAF>(sk, na, odd_first, qb + qh, qm + qh, take, seed, best, cb + cn, cm + cn);
        qh += take;
        if (cn > ckeep) {
            const uint32_t ct = min(cn, 32u);
            if (rot_check<LEAF>(cb, cm, ct, warp_load64(node_seed), node_seed, found)) {
                qn = 0;
                return true;
            }
            cn -= ct;  // the rest (fewer than 32) moves to the front
            const uint64_t b = lane < cn ? cb[ct + lane] : 0;
            const uint2 mk = lane < cn ? cm[ct + lane] : make_uint2(0, 0);
            __syncwarp();
            if (lane < cn) {
                cb[lane] = b;
                cm[lane] = mk;
            }
            __syncwarp();
        }
    }
    if (cn > 0 && rot_check<LEAF>(cb, cm, cn, warp_load64(node_seed), node_seed, found)) spent = true;
    if (spent) {
        qn = 0;
        return true;
    }
    const uint32_t rest = qn - qh;  // fewer than 32 unchecked bases move to the front
    if (qh > 0 && rest > 0) {
        const uint64_t b = lane < rest ? qb[qh + lane] : 0;
        const uint32_t mk = lane < rest ? qm[qh + lane] : 0;
        __syncwarp();
        if (lane < rest) {
            qb[lane] = b;
            qm[lane] = mk;
        }
        __syncwarp();
    }
    qn = rest;
    return false;
}

// Per-warp shared memory of the leaf search, in bytes: keys and per-key terms (LEAF each),
// then for rotation leaves the (base, left mask) queue of phase A and the rotation queue.
template <int LEAF, bool ROT, int S>
__host__ __device__ constexpr size_t leaf_warp_bytes() {
    return ROT ? (size_t)LEAF * 16 + (size_t)leaf_queue_cap<S>() * 12 + kRotQueueCap * 16 : (size_t)LEAF * 8;
}

template <int LEAF, bool ROT, int S>
__global__ void __launch_bounds__(kThreads) k_search_leaf(SearchCtx c) {
    constexpr int STAGE = ROT ? kStageLeafRot : kStageLeafBF;
    constexpr uint32_t W = 32 * S;
    constexpr int QCAP = leaf_queue_cap<S>();
    extern __shared__ uint64_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // per warp: keys | per-key terms | phase-A queue: bases, left masks | rotation queue: bases, masks
    uint64_t *sk = smem + warp * (leaf_warp_bytes<LEAF, ROT, S>() / 8);
    uint2 *pk = reinterpret_cast<uint2 *>(sk + LEAF);
    uint64_t *qb = sk + 2 * LEAF;
    uint32_t *qm = reinterpret_cast<uint32_t *>(qb + QCAP);
    uint64_t *cb = reinterpret_cast<uint64_t *>(qm + QCAP);
    uint2 *cm = reinterpret_cast<uint2 *>(cb + kRotQueueCap);
    const uint32_t gw = blockIdx.x * kWarpsPerCta + warp;
    const uint32_t count = c.stage_info[STAGE];
    const uint32_t base = c.stage_info[kNumStages + STAGE];
    uint32_t *found = &c.sched[kNumStages + STAGE];  // nodes of this stage with a seed
    const uint64_t seed = start_seed(kNumStartSeeds - 1);
    uint32_t rng = gw * 2654435761u + 777u;
    uint32_t node = kEmpty, m = 0, na = 0, qn = 0, keep = 0, ckeep = 0;
    bool owner = false, odd_first = false;
    uint64_t budget = 0;
    for (;;) {
        if (node == kEmpty) {
            if (warp_status(c.status)) break;
            uint32_t f = 0;
            if (lane == 0) f = atomicAdd(&c.sched[STAGE], 1u);
            f = __shfl_sync(0xffffffffu, f, 0);
            if (f < count) {
                node = c.lists[base + f];
                owner = true;
                if (lane == 0) c.slots[gw] = node;
            } else {
                owner = false;
                if (warp_load32(found) >= count) break;  // every node of the stage has a seed
                rng = rng * 1664525u + 1013904223u;
                node = find_help(c, rng);
                if (node == kEmpty) break;
            }
            const uint32_t start = c.nodes.start[node];
            m = c.nodes.size[node];
            const uint64_t k = lane < (int)m ? c.keys[start + lane] : 0;
            __syncwarp();
            if (ROT) {
                // phase-A half first: the larger one (see leaf_check)
                const unsigned even = __ballot_sync(0xffffffffu, lane < (int)m && (k & 1) == 0);
                const unsigned odd = __ballot_sync(0xffffffffu, lane < (int)m && (k & 1) == 1);
                odd_first = __popc(odd) > __popc(even);
                const unsigned first = odd_first ? odd : even, second = odd_first ? even : odd;
                na = __popc(first);
                const unsigned below = (1u << lane) - 1;
                const bool in_first = lane < (int)m && ((k & 1) != 0) == odd_first;
                if (lane < (int)m) sk[in_first ? __popc(first & below) : na + __popc(second & below)] = k;
            } else {
                if (lane < (int)m) sk[lane] = k;
            }
            __syncwarp();
            budget = budget_for(c, m);
            qn = 0;
            keep = search_eagerly(c, m, (uint64_t)W * LEAF) ? 0 : 31;
            ckeep = (1ull << (c.tab.memo[m] >> 27)) <= (uint64_t)W * LEAF ? 0 : 31;
        }
        uint32_t w = 0;
        if (lane == 0) w = atomicAdd(&c.nodes.next_win[node], 1u);
        w = __shfl_sync(0xffffffffu, w, 0);
        const uint64_t x0 = (uint64_t)w * W;                   // first base (ROT) or seed of the window
        const uint64_t enc0 = ROT ? x0 * LEAF : x0;            // first encoded seed of the window
        const uint64_t best = warp_load64(&c.nodes.seed[node]);
        if (enc0 >= best || enc0 >= budget) {
            if (ROT) leaf_phase_bc<LEAF>(sk, na, odd_first, qb, qm, qn, 0, ckeep, seed, cb, cm, &c.nodes.seed[node], found);
            if (enc0 < warp_load64(&c.nodes.seed[node]) && lane == 0) merge_seed(&c.nodes.seed[node], kSeedFailed, found);
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
            left_masks<LEAF, S>(sk, na, seed + x0 * LEAF, pk, ml);
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint64_t b = x0 + lane + 32u * s;
                const uint32_t mk = left_mask_of<LEAF>(ml[s], na);
                const bool pass = mk != ~0u;
                const unsigned bal = __ballot_sync(0xffffffffu, pass);
                if (pass) {
                    qb[qn + __popc(bal & below)] = b;
                    qm[qn + __popc(bal & below)] = mk;
                }
                qn += __popc(bal);
            }
            __syncwarp();
            const bool done =
                leaf_phase_bc<LEAF>(sk, na, odd_first, qb, qm, qn, keep, ckeep, seed, cb, cm, &c.nodes.seed[node], found);
            __syncwarp();  // qb/qm are appended to by the next window
            if (done) {  // every later window starts above the leaf's seed: leave without taking one
                if (owner && lane == 0) c.slots[gw] = kEmpty;
                node = kEmpty;
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
        if (off != 0xFFFFFFFFu) {  // this window holds the seed: leave without taking another one
            if (lane == 0) {
                merge_seed(&c.nodes.seed[node], enc0 + off, found);
                if (owner) c.slots[gw] = kEmpty;
            }
            node = kEmpty;
        }
    }
}


}  // namespace

namespace search_impl {

// Launches the persistent search kernel `k` with `smem` bytes of dynamic shared memory at the
// schedule's share of the engine's occupancy.
template <typename K>
void launch_persistent(K k, const SearchCtx &c, size_t smem, const StageSchedule &s, cudaStream_t st) {
    if (smem) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    use_max_smem(k);  // before the occupancy query, which follows the kernel's carveout preference
    const int pct = std::max(1, c.occupancy_pct * s.occupancy_pct / 100);
    int g = persistent_grid(k, smem, c.num_sms, kThreads, pct);
    g = min(g, (int)(c.nslots / kWarpsPerCta));
    SearchCtx cc = c;
    cc.nslots = g * kWarpsPerCta;
    k<<<g, kThreads, smem, st>>>(cc);
}

// The same for a kernel that also takes the pipeline state.
template <typename K>
void launch_persistent_with(K k, const SearchCtx &c, const PipeCtx &p, size_t smem, const StageSchedule &s,
                            cudaStream_t st) {
    if (smem) cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    use_max_smem(k);  // before the occupancy query, which follows the kernel's carveout preference
    const int pct = std::max(1, c.occupancy_pct * s.occupancy_pct / 100);
    int g = persistent_grid(k, smem, c.num_sms, kThreads, pct);
    g = min(g, (int)(c.nslots / kWarpsPerCta));
    SearchCtx cc = c;
    cc.nslots = g * kWarpsPerCta;
    k<<<g, kThreads, smem, st>>>(cc, p);
}

template <int LEAF, int STAGE, int S>
void launch_aggr(const SearchCtx &c, const StageSchedule &s, cudaStream_t st) {
    using C = AggrCfg<LEAF, STAGE, S>;
    launch_persistent(k_search_aggr<LEAF, STAGE, S>, c, kWarpsPerCta * C::WARP_WORDS * sizeof(uint64_t), s, st);
}

template <int LEAF, int STAGE>
void launch_aggr_s(const SearchCtx &c, const StageSchedule &s, cudaStream_t st) {
    switch (s.seeds_per_lane) {
        case 4: launch_aggr<LEAF, STAGE, 4>(c, s, st); break;
        case 8: launch_aggr<LEAF, STAGE, 8>(c, s, st); break;
        case 16: launch_aggr<LEAF, STAGE, 16>(c, s, st); break;
        default: launch_aggr<LEAF, STAGE, 12>(c, s, st); break;
    }
}

template <int LEAF>
void run_aggr(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st) {
    if (stage == kStageUpper) launch_aggr_s<LEAF, kStageUpper>(c, s, st);
    else launch_aggr_s<LEAF, kStageLower>(c, s, st);
}

template <int LEAF>
void run_partition(const SearchCtx &c, int stage, cudaStream_t st) {
    const StageSchedule full{8, 100};
    if (stage == kStageUpper) {
        using C = AggrCfg<LEAF, kStageUpper>;
        launch_persistent(k_partition_aggr<LEAF, kStageUpper>, c, kWarpsPerCta * C::MAXM * sizeof(uint64_t), full, st);
    } else {
        using C = AggrCfg<LEAF, kStageLower>;
        launch_persistent(k_partition_aggr<LEAF, kStageLower>, c, kWarpsPerCta * C::MAXM * sizeof(uint64_t), full, st);
    }
}

template <int LEAF, bool ROT, int S>
void launch_leaf(const SearchCtx &c, const StageSchedule &s, cudaStream_t st) {
    launch_persistent(k_search_leaf<LEAF, ROT, S>, c, kWarpsPerCta * leaf_warp_bytes<LEAF, ROT, S>(), s, st);
}

template <int LEAF>
void run_leaves(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st) {
    if (stage != kStageLeafRot) {
        launch_leaf<LEAF, false, 8>(c, s, st);
        return;
    }
    switch (s.seeds_per_lane) {
        case 4: launch_leaf<LEAF, true, 4>(c, s, st); break;
        case 12: launch_leaf<LEAF, true, 12>(c, s, st); break;
        default: launch_leaf<LEAF, true, 8>(c, s, st); break;
    }
}

}  // namespace search_impl

}  // namespace rsb
