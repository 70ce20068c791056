// All aggregation and leaf searches of a build in one persistent launch, with device work
// queues (the engine's pipeline mode).
//
// The stage kernels (rsb_search_impl.cuh) run one stage at a time: every node of a stage is
// searched, then partitioned, before any node of the next stage starts, so each stage ends
// with a tail in which idle warps pile onto its last nodes. Here a node is ready as soon as
// its parent has been partitioned: four queues (upper aggregation, lower aggregation,
// rotation leaves, other leaves) start with the nodes whose parents are done before the
// launch (fanout-2 nodes and bucket roots), and the warp that completes an aggregation node
// partitions its keys and appends its children to their queues. Warps take the highest
// stage first (the longest chains of dependent work start earliest) and help unfinished nodes
// only when every queue is empty.
//
// A node is complete when its minimum seed can no longer change: a seed has been found and
// no warp is still evaluating a window of the node. Every warp counts itself in the node's
// `active` counter before taking windows and out after it has drained its queues; windows
// are handed out in ascending order, so once a seed is known every window below it has been
// taken, and a warp arriving later only takes windows above it. The warp whose decrement
// leaves the counter at zero with a seed known claims the node (a compare-and-swap on its
// state) and completes it. The searches themselves are those of the stage kernels, so the
// minimum seeds - and the function - are the same. A warp copies an aggregation node's keys
// into its shared memory when it joins the node; the completing warp partitions from its
// copy straight into the key array.
//
// Memory ordering. Every decision a whole warp takes on shared state (the status, the
// completed-node count, a node's seed, the active count) is read by lane 0 and broadcast, so
// the warp never diverges around its warp-wide operations. A warp joining a node publishes
// its active count (with a fence) before it takes a window, and fences before its exit
// decrement, so that its seed merges precede the decrement; the warp whose decrement leaves
// the count at zero fences again and reads the seed with an atomic, so it sees every merge of
// the warps that left before it. A warp that joins a node after its completion takes a window
// above the node's seed and can no longer lower it (its copy of the keys may be read while
// they are being partitioned; only windows above the seed are evaluated with it).
//
// Self-checks: a node id taken from a queue or a help slot must be a node of stages 17..20,
// a push must stay within its stage's queue, and a partition must fill every part exactly
// (the seed's split of the node's keys); otherwise the launch stops with RSB_ERR_INTERNAL
// (detail: kPipeBad* | the node id or queue) without the access.
//
// Waits are bounded in time (%globaltimer): a warp that has found no work while no node
// anywhere completed for kPipelineStallNs gives up with RSB_ERR_TIMEOUT, and so does every
// warp once the launch has run for the engine's watchdog bound. The first warp to give up
// records the state of the unfinished nodes in the queue counters (pipe_diagnose) for the
// host to report.
#pragma once

#include "rsb_search_impl.cuh"

namespace rsb {

namespace {

// No node completing anywhere for this long, while nodes remain, is a stall: searches are
// bounded by their budgets and a node's drains and partition take microseconds.
constexpr uint64_t kPipelineStallNs = 10000000000ull;
// Help slots an idle warp scans per look, and its sleep between looks (doubling from the
// first to the last while it stays idle).
constexpr uint32_t kPipeHelpScan = 512;
constexpr uint32_t kPipeIdleSleepMin = 256, kPipeIdleSleepMax = 4096;
constexpr int kPipeQueues = 4;  // stages 17, 18, 19, 20
// Warps that may work on one node at a time (owner and helpers): more only take windows past
// the node's seed.
constexpr uint32_t kPipeMaxWarpsPerNode = 16;
// RSB_ERR_INTERNAL details of the self-checks (low 32 bits: the node id or queue).
constexpr uint64_t kPipeBadNode = 1ull << 32;
constexpr uint64_t kPipeBadQueue = 2ull << 32;
constexpr uint64_t kPipeBadSplit = 3ull << 32;

__device__ __forceinline__ int queue_of(uint32_t stage) { return (int)stage - kStageUpper; }

__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool pipe_node_ok(const SearchCtx &c, uint32_t id) {
    if ((uint64_t)id >= *(const volatile uint64_t *)c.node_total) return false;
    const uint32_t st = c.nodes.stage[id];
    return st >= (uint32_t)kStageUpper && st <= (uint32_t)kStageLeafBF;
}

// Appends node `id` to its stage's queue (lane 0 of the calling warp); false (and
// RSB_ERR_INTERNAL) if the id or the queue slot is out of range.
__device__ __forceinline__ bool pipe_push(const SearchCtx &c, const PipeCtx &p, uint32_t id) {
    if (!pipe_node_ok(c, id)) {
        set_error(c.status, RSB_ERR_INTERNAL, kPipeBadNode | id);
        return false;
    }
    const uint32_t st = c.nodes.stage[id];
    const int q = queue_of(st);
    const uint32_t at = atomicAdd(&p.counts[q], 1u);
    if (at >= c.stage_info[st]) {
        set_error(c.status, RSB_ERR_INTERNAL, kPipeBadQueue | (uint32_t)q);
        return false;
    }
    __threadfence();  // the node's keys (partitioned by this warp) before its publication
    atomicExch(&p.queue[c.stage_info[kNumStages + st] + at], id);
    return true;
}

// Queue tickets. A warp takes a node by drawing a ticket - the next slot index of a queue, one
// atomicAdd on its head - and reading that slot; a slot whose node is not pushed yet stays the
// warp's ticket, and the warp reads it again at its next look (meanwhile it may help other
// nodes). Every node of a stage is pushed exactly once, so a ticket below the stage's node
// count is filled eventually and a ticket at or past it is dead. A warp draws a new ticket
// only when it holds none for that queue and the queue's reserved tail is ahead of its head,
// so each push costs one atomic of the warps waiting for it, not a retry of every idle warp.
constexpr uint32_t kNoTicket = 0xFFFFFFFFu;
constexpr uint32_t kDeadTicket = 0xFFFFFFFEu;

// Takes a ready node, highest queue first; kEmpty when none is ready. Lane 0; tk holds the
// warp's tickets.
__device__ uint32_t pipe_pop(const SearchCtx &c, const PipeCtx &p, uint32_t (&tk)[kPipeQueues]) {
#pragma unroll
    for (int q = 0; q < kPipeQueues; ++q) {
        const int st = kStageUpper + q;
        if (tk[q] == kDeadTicket) continue;
        if (tk[q] == kNoTicket) {
            if (vload32(&p.counts[kPipeQueues + q]) >= vload32(&p.counts[q])) continue;
            const uint32_t t = atomicAdd(&p.counts[kPipeQueues + q], 1u);
            tk[q] = t < c.stage_info[st] ? t : kDeadTicket;
            if (tk[q] == kDeadTicket) continue;
        }
        const uint32_t id = vload32(&p.queue[c.stage_info[kNumStages + st] + tk[q]]);
        if (id == kEmpty) continue;  // not pushed yet: the ticket stays
        __threadfence();              // the node's keys, published before its id, are read after it
        tk[q] = kNoTicket;
        return id;
    }
    return kEmpty;
}

// Scans kPipeHelpScan help slots from `start` (four per lane per step) for a node whose seed
// is unknown and that fewer than kPipeMaxWarpsPerNode warps work on; kEmpty if none.
// Warp-uniform result.
__device__ uint32_t pipe_find_help(const SearchCtx &c, const PipeCtx &p, uint32_t start) {
    constexpr uint32_t U = 4;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t nw = min(c.nslots, gridDim.x * (uint32_t)kWarpsPerCta);
    const uint32_t span = min(nw, kPipeHelpScan);
    start %= nw;
    for (uint32_t k = 0; k < span; k += 32 * U) {
        uint32_t pick = kEmpty;
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) {
            const uint32_t off = k + j * 32 + lane;
            uint32_t idx = start + off;
            if (idx >= nw) idx -= nw;
            const uint32_t nd = off < span ? vload32(&c.slots[idx]) : kEmpty;
            if (pick == kEmpty && nd != kEmpty && vload64(&c.nodes.seed[nd]) == kSeedNotFound &&
                vload32(&p.active[nd]) < kPipeMaxWarpsPerNode)
                pick = nd;
        }
        const unsigned b = __ballot_sync(0xffffffffu, pick != kEmpty);
        if (b) return __shfl_sync(0xffffffffu, pick, __ffs(b) - 1);
    }
    return kEmpty;
}

// Stable fanout-way partition of an aggregation node's keys, from the completing warp's
// shared-memory copy (sk) into the key array, then its children (DFS order: the first child
// follows the node, each next one follows the previous child's subtree) go to their queues.
// The seed splits the keys exactly, so every part fills its range; a partition that does not
// (a seed that was not the node's) writes nothing outside the node, stops the launch and
// pushes no child.
template <int LEAF, int STAGE>
__device__ void pipe_complete_aggr(const SearchCtx &c, const PipeCtx &p, uint32_t id, uint64_t x,
                                   const uint64_t *sk) {
    using C = AggrCfg<LEAF, STAGE>;
    const int lane = threadIdx.x & 31;
    const uint32_t start = c.nodes.start[id];
    const uint32_t m = c.nodes.size[id];
    const uint32_t fan = uint16_t(m + C::SPLIT - 1) / C::SPLIT;
    const uint64_t sx = start_seed(C::SEED_INDEX) + x;
    uint32_t cur[C::MAXF];
#pragma unroll
    for (uint32_t j = 0; j < C::MAXF; ++j) cur[j] = j * C::SPLIT;
    bool bad = false;
    for (uint32_t c0 = 0; c0 < m; c0 += 32) {
        const uint32_t i = c0 + lane;
        const bool valid = i < m;
        const uint64_t k = valid ? sk[i] : 0;
        const uint32_t part = valid ? remap16(k + sx, m) / C::SPLIT : 0xFFu;
        uint32_t dst = 0xFFFFFFFFu;
#pragma unroll
        for (uint32_t j = 0; j < C::MAXF; ++j) {
            if (j < fan) {
                const unsigned b = __ballot_sync(0xffffffffu, part == j);
                if (part == j) dst = cur[j] + __popc(b & ((1u << lane) - 1));
                cur[j] += __popc(b);
            }
        }
        if (valid && dst < m) __stcg(&c.keys[start + dst], k);
        bad |= valid && dst >= m;
    }
#pragma unroll
    for (uint32_t j = 0; j < C::MAXF; ++j)
        if (j < fan) bad |= cur[j] != (j + 1 < fan ? (j + 1) * C::SPLIT : m);
    if (__any_sync(0xffffffffu, bad)) {
        if (lane == 0) set_error(c.status, RSB_ERR_INTERNAL, kPipeBadSplit | id);
        return;
    }
    __threadfence();  // every lane's keys before lane 0 publishes the children
    __syncwarp();
    if (lane == 0) {
        uint32_t child = id + 1;
        for (uint32_t j = 0; j < fan; ++j) {
            const uint32_t cm = j + 1 < fan ? C::SPLIT : m - (fan - 1) * C::SPLIT;
            if (cm <= 1) continue;
            if (!pipe_push(c, p, child)) break;
            child += c.tab.nodes[cm];
        }
    }
    __syncwarp();
}

// Per-node search state of a warp.
struct PipeNode {
    uint32_t id, stage, m, fan, tlo, thi, t1, mult, na, qn, keep, ckeep;
    bool full, owner, odd_first;
    uint64_t budget;
};

template <int LEAF, int STAGE>
__device__ __forceinline__ void aggr_setup(const SearchCtx &c, PipeNode &s) {
    using C = AggrCfg<LEAF, STAGE>;
    s.fan = uint16_t(s.m + C::SPLIT - 1) / C::SPLIT;
    s.full = s.m == s.fan * C::SPLIT;
    s.tlo = s.thi = 0;
    for (uint32_t j = 0; j < 8 && j < s.fan; ++j) {
        const uint32_t t = j + 1 < s.fan ? C::SPLIT : s.m - (s.fan - 1) * C::SPLIT;
        if (j < 4) s.tlo |= t << (8 * j);
        else s.thi |= t << (8 * (j - 4));
    }
    s.mult = (uint32_t)((((uint64_t)s.m << 28) + C::SPLIT - 1) / C::SPLIT);
    s.t1 = s.full ? kAccF0 + 128u * s.fan * s.m : 0u;
    for (uint32_t j = 1; j < s.fan; ++j) s.t1 += j * (j + 1 < s.fan ? C::SPLIT : s.m - (s.fan - 1) * C::SPLIT);
}

// One window of an aggregation node (phase A, then phase B of its survivors): returns false
// when the warp leaves the node.
template <int LEAF, int STAGE, int S>
__device__ bool aggr_window(const SearchCtx &c, PipeNode &s, const uint64_t *sk, uint64_t *q, uint2 *pk,
                            uint32_t *found) {
    using C = AggrCfg<LEAF, STAGE, S>;
    constexpr uint32_t W = C::W;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1;
    const uint64_t seed = start_seed(C::SEED_INDEX);
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(&c.nodes.next_win[s.id], 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    const uint64_t x0 = (uint64_t)w * W;
    const uint64_t best = warp_load64(&c.nodes.seed[s.id]);
    if (x0 >= best || x0 >= s.budget) {
        aggr_phase_b<LEAF, STAGE>(sk, q, s.qn, 0, s.m, s.fan, s.full, seed, s.tlo, s.thi, &c.nodes.seed[s.id], found);
        if (x0 < warp_load64(&c.nodes.seed[s.id]) && lane == 0) merge_seed(&c.nodes.seed[s.id], kSeedFailed, found);
        return false;
    }
    uint32_t cnt[S];
#pragma unroll
    for (int k = 0; k < S; ++k) cnt[k] = s.full ? kAccF0 : 0u;
    for (uint32_t i0 = 0; i0 < s.m; i0 += kAbortChunk) {
        const uint32_t len = min(kAbortChunk, s.m - i0);
        if (s.full) moment_sums<S, true>(sk + i0, len, seed + x0, s.fan, pk, cnt);
        else moment_sums<S, false>(sk + i0, len, seed + x0, s.mult, pk, cnt);
        if (i0 + len < s.m) {
            uint64_t b = 0;
            if (lane == 0) b = vload64(&c.nodes.seed[s.id]);
            if (__shfl_sync(0xffffffffu, b, 0) <= x0) return true;  // abandoned: a lower seed was found
        }
    }
#pragma unroll
    for (int k = 0; k < S; ++k) {
        const bool pass = cnt[k] == s.t1;
        const unsigned b = __ballot_sync(0xffffffffu, pass);
        if (pass) q[s.qn + __popc(b & below)] = x0 + lane + 32u * k;
        s.qn += __popc(b);
    }
    __syncwarp();
    aggr_phase_b<LEAF, STAGE>(sk, q, s.qn, s.keep, s.m, s.fan, s.full, seed, s.tlo, s.thi, &c.nodes.seed[s.id],
                              found);
    __syncwarp();  // q is appended to by the next window
    return true;
}

// One window of a leaf: returns false when the warp leaves the node.
template <int LEAF, bool ROT, int S>
__device__ bool leaf_window(const SearchCtx &c, PipeNode &s, const uint64_t *sk, uint2 *pk, uint64_t *qb,
                            uint32_t *qm, uint64_t *cb, uint2 *cm, uint32_t *found) {
    constexpr uint32_t W = 32 * S;
    const int lane = threadIdx.x & 31;
    const uint64_t seed = start_seed(kNumStartSeeds - 1);
    uint64_t *node_seed = &c.nodes.seed[s.id];
    uint32_t w = 0;
    if (lane == 0) w = atomicAdd(&c.nodes.next_win[s.id], 1u);
    w = __shfl_sync(0xffffffffu, w, 0);
    const uint64_t x0 = (uint64_t)w * W;
    const uint64_t enc0 = ROT ? x0 * LEAF : x0;
    const uint64_t best = warp_load64(node_seed);
    if (enc0 >= best || enc0 >= s.budget) {
        if (ROT) leaf_phase_bc<LEAF>(sk, s.na, s.odd_first, qb, qm, s.qn, 0, s.ckeep, seed, cb, cm, node_seed, found);
        if (enc0 < warp_load64(node_seed) && lane == 0) merge_seed(node_seed, kSeedFailed, found);
        return false;
    }
    if (ROT) {
        const unsigned below = (1u << lane) - 1;
        uint32_t ml[S];
#pragma unroll
        for (int k = 0; k < S; ++k) ml[k] = 0;
        left_masks<LEAF, S>(sk, s.na, seed + x0 * LEAF, pk, ml);
#pragma unroll
        for (int k = 0; k < S; ++k) {
            const uint64_t b = x0 + lane + 32u * k;
            const uint32_t mk = left_mask_of<LEAF>(ml[k], s.na);
            const bool pass = mk != ~0u;
            const unsigned bal = __ballot_sync(0xffffffffu, pass);
            if (pass) {
                qb[s.qn + __popc(bal & below)] = b;
                qm[s.qn + __popc(bal & below)] = mk;
            }
            s.qn += __popc(bal);
        }
        __syncwarp();
        leaf_phase_bc<LEAF>(sk, s.na, s.odd_first, qb, qm, s.qn, s.keep, s.ckeep, seed, cb, cm, node_seed, found);
        __syncwarp();  // qb/qm are appended to by the next window
    } else {
        const uint32_t full = (1u << s.m) - 1;
        uint32_t off = 0xFFFFFFFFu;
#pragma unroll
        for (int k = S - 1; k >= 0; --k) {
            const uint64_t bx = seed + x0 + lane + 32u * k;
            uint32_t mask = 0;
            for (uint32_t i = 0; i < s.m; ++i) mask |= 1u << remap16(sk[i] + bx, s.m);
            if (mask == full) off = lane + 32u * k;
        }
        off = __reduce_min_sync(0xffffffffu, off);
        if (off != 0xFFFFFFFFu && lane == 0) merge_seed(node_seed, enc0 + off, found);
    }
    return true;
}

// Per-warp shared memory of the pipeline kernel: the larger of the aggregation layout (the
// keys of the largest aggregation node, the phase-B queue of the window and the per-key
// terms) and the leaf layout.
template <int LEAF, int SA, int SL>
__host__ __device__ constexpr size_t pipe_warp_bytes() {
    constexpr size_t aggr = 8 * (size_t)(upper_of(LEAF) + 32 + 32 * SA) + 8 * (size_t)kAbortChunk;
    constexpr size_t leaf = leaf_warp_bytes<LEAF, true, SL>() + 8 * LEAF;
    return aggr > leaf ? aggr : leaf;
}

// Called by every warp that leaves the launch on RSB_ERR_TIMEOUT; the first records, in
// counts[10..28), a snapshot of the nodes of stages 17..20 that are not complete:
//   [10] 1 once recorded  [11] the status detail (1 stall, 3 watchdog)
//   [12] unfinished nodes, of them [13] with warps active, [14] with a seed known,
//   [15] queued by their parent, [16] with no window handed out yet
//   [17] the first unfinished node, [18] its stage | size << 8, [19] [20] its seed (low and
//   high word), [21] its active warps, [22] its windows handed out, [23] its queued-by-parent
//   flag; [24, 28) the slot at each queue's head (kEmpty when the queue is drained).
__device__ void pipe_diagnose(const SearchCtx &c, const PipeCtx &p) {
    const int lane = threadIdx.x & 31;
    uint32_t first = 0;
    if (lane == 0) first = atomicCAS(&p.counts[10], 0u, 1u) == 0u;
    if (!__shfl_sync(0xffffffffu, first, 0)) return;
    const uint32_t base = c.stage_info[kNumStages + kStageUpper];
    const uint32_t cnt = c.stage_info[kStageUpper] + c.stage_info[kStageLower] + c.stage_info[kStageLeafRot] +
                         c.stage_info[kStageLeafBF];
    uint32_t n = 0, act = 0, known = 0, blk = 0, never = 0, fid = kEmpty;
    for (uint32_t i = lane; i < cnt; i += 32) {
        const uint32_t id = c.lists[base + i];
        if (vload32(&p.claimed[id])) continue;
        ++n;
        act += vload32(&p.active[id]) != 0;
        known += vload64(&c.nodes.seed[id]) != kSeedNotFound;
        blk += p.blocked[id] != 0;
        never += vload32(&c.nodes.next_win[id]) == 0;
        fid = min(fid, id);
    }
    n = __reduce_add_sync(0xffffffffu, n);
    act = __reduce_add_sync(0xffffffffu, act);
    known = __reduce_add_sync(0xffffffffu, known);
    blk = __reduce_add_sync(0xffffffffu, blk);
    never = __reduce_add_sync(0xffffffffu, never);
    fid = __reduce_min_sync(0xffffffffu, fid);
    if (lane == 0) {
        uint32_t *d = p.counts;
        d[11] = (uint32_t)*(const volatile uint64_t *)&c.status->detail;
        d[12] = n;
        d[13] = act;
        d[14] = known;
        d[15] = blk;
        d[16] = never;
        d[17] = fid;
        if (fid != kEmpty) {
            const uint64_t x = vload64(&c.nodes.seed[fid]);
            d[18] = c.nodes.stage[fid] | (uint32_t)c.nodes.size[fid] << 8;
            d[19] = (uint32_t)x;
            d[20] = (uint32_t)(x >> 32);
            d[21] = vload32(&p.active[fid]);
            d[22] = vload32(&c.nodes.next_win[fid]);
            d[23] = p.blocked[fid];
        }
        for (int q = 0; q < kPipeQueues; ++q) {
            const uint32_t h = vload32(&p.counts[kPipeQueues + q]);
            d[24 + q] = h < vload32(&p.counts[q]) ? vload32(&p.queue[c.stage_info[kNumStages + kStageUpper + q] + h])
                                                  : kEmpty;
        }
        __threadfence();
    }
    __syncwarp();
}

template <int LEAF, int SA, int SL>
__global__ void __launch_bounds__(kThreads) k_pipeline(SearchCtx c, PipeCtx p) {
    extern __shared__ uint64_t smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint8_t *wbase = reinterpret_cast<uint8_t *>(smem) + warp * pipe_warp_bytes<LEAF, SA, SL>();
    // aggregation layout: the node's keys, phase-B queue, per-key terms
    uint64_t *ask = reinterpret_cast<uint64_t *>(wbase);
    uint64_t *aq = ask + upper_of(LEAF);
    uint2 *apk = reinterpret_cast<uint2 *>(aq + 32 + 32 * SA);
    // leaf layout: keys, per-key terms, phase-A queue (bases, masks), rotation queue (bases, masks)
    uint64_t *lsk = reinterpret_cast<uint64_t *>(wbase);
    uint2 *lpk = reinterpret_cast<uint2 *>(lsk + LEAF);
    uint64_t *qb = lsk + 2 * LEAF;
    uint32_t *qm = reinterpret_cast<uint32_t *>(qb + leaf_queue_cap<SL>());
    uint64_t *cb = reinterpret_cast<uint64_t *>(qm + leaf_queue_cap<SL>());
    uint2 *cm = reinterpret_cast<uint2 *>(cb + kRotQueueCap);
    const uint32_t gw = blockIdx.x * kWarpsPerCta + warp;
    uint32_t rng = gw * 2654435761u + 4242u;
    // lane 0: queue tickets; the completed-node count seen and when it last changed while
    // this warp was idle (0: not idle); the idle sleep
    uint32_t tk[kPipeQueues];
#pragma unroll
    for (int q = 0; q < kPipeQueues; ++q) tk[q] = kNoTicket;
    uint32_t seen_done = 0, sleep_ns = kPipeIdleSleepMin;
    uint64_t idle_since = 0;
    const uint64_t t_start = globaltimer_ns();
    PipeNode s{};
    s.id = kEmpty;
    for (;;) {
        if (c.watchdog_ns) {  // optional bound on the whole launch (rsb_engine_set_watchdog)
            uint32_t late = 0;
            if (lane == 0) late = globaltimer_ns() - t_start > c.watchdog_ns;
            if (__shfl_sync(0xffffffffu, late, 0)) {
                if (lane == 0) set_error(c.status, RSB_ERR_TIMEOUT, 3);
                break;
            }
        }
        if (s.id == kEmpty) {
            uint32_t id = kEmpty, stop = 0;
            if (lane == 0) {
                stop = status_code(c.status) != 0;
                if (!stop) id = pipe_pop(c, p, tk);
            }
            if (__shfl_sync(0xffffffffu, stop, 0)) break;
            id = __shfl_sync(0xffffffffu, id, 0);
            s.owner = id != kEmpty;
            if (id == kEmpty) {
                uint32_t done = 0, now_done = 0;
                if (lane == 0) {
                    now_done = vload32(&p.counts[2 * kPipeQueues]);
                    done = now_done >= p.counts[2 * kPipeQueues + 1];
                }
                if (__shfl_sync(0xffffffffu, done, 0)) break;  // every node is complete
                rng = rng * 1664525u + 1013904223u;
                id = pipe_find_help(c, p, rng);
                if (id == kEmpty) {
                    uint32_t give_up = 0;
                    if (lane == 0) {
                        const uint64_t now = globaltimer_ns();
                        if (idle_since == 0 || now_done != seen_done) {
                            idle_since = now;
                            seen_done = now_done;
                        }
                        give_up = now - idle_since > kPipelineStallNs;
                        if (give_up) set_error(c.status, RSB_ERR_TIMEOUT, 1);
                    }
                    if (__shfl_sync(0xffffffffu, give_up, 0)) break;
                    __nanosleep(sleep_ns);
                    sleep_ns = min(2 * sleep_ns, kPipeIdleSleepMax);
                    continue;
                }
            }
            idle_since = 0;
            sleep_ns = kPipeIdleSleepMin;
            uint32_t ok = 0;
            if (lane == 0) {
                ok = pipe_node_ok(c, id);
                if (!ok) {
                    set_error(c.status, RSB_ERR_INTERNAL, kPipeBadNode | id);
                } else {
                    atomicAdd(&p.active[id], 1u);
                    __threadfence();  // counted in before this warp takes a window of the node
                    if (s.owner) c.slots[gw] = id;
                }
            }
            if (!__shfl_sync(0xffffffffu, ok, 0)) break;
            s.id = id;
            __threadfence();  // the node's keys, published before its id, are read after it
            s.stage = c.nodes.stage[id];
            s.m = c.nodes.size[id];
            s.budget = budget_for(c, s.m);
            s.qn = 0;
            if (s.stage == kStageUpper || s.stage == kStageLower) {
                const uint32_t start = c.nodes.start[id];
                for (uint32_t i = lane; i < s.m; i += 32) ask[i] = __ldcg(&c.keys[start + i]);
                __syncwarp();
                if (s.stage == kStageUpper) aggr_setup<LEAF, kStageUpper>(c, s);
                else aggr_setup<LEAF, kStageLower>(c, s);
                s.keep = search_eagerly(c, s.m, 32u * SA) ? 0 : 31;
            } else {
                const uint32_t start = c.nodes.start[id];
                const uint64_t k = lane < (int)s.m ? __ldcg(&c.keys[start + lane]) : 0;
                s.keep = search_eagerly(c, s.m, (uint64_t)32 * SL * LEAF) ? 0 : 31;
                s.ckeep = (1ull << (c.tab.memo[s.m] >> 27)) <= (uint64_t)32 * SL * LEAF ? 0 : 31;
                if (s.stage == kStageLeafRot) {  // phase-A half first, as in k_search_leaf
                    const unsigned even = __ballot_sync(0xffffffffu, lane < (int)s.m && (k & 1) == 0);
                    const unsigned odd = __ballot_sync(0xffffffffu, lane < (int)s.m && (k & 1) == 1);
                    s.odd_first = __popc(odd) > __popc(even);
                    const unsigned first = s.odd_first ? odd : even, second = s.odd_first ? even : odd;
                    s.na = __popc(first);
                    const unsigned below = (1u << lane) - 1;
                    const bool in_first = lane < (int)s.m && ((k & 1) != 0) == s.odd_first;
                    if (lane < (int)s.m) lsk[in_first ? __popc(first & below) : s.na + __popc(second & below)] = k;
                } else if (lane < (int)s.m) {
                    lsk[lane] = k;
                }
                __syncwarp();
            }
        }
        uint32_t *found = &c.sched[kNumStages + s.stage];
        bool stay;
        switch (s.stage) {
            case kStageUpper: stay = aggr_window<LEAF, kStageUpper, SA>(c, s, ask, aq, apk, found); break;
            case kStageLower: stay = aggr_window<LEAF, kStageLower, SA>(c, s, ask, aq, apk, found); break;
            case kStageLeafRot: stay = leaf_window<LEAF, true, SL>(c, s, lsk, lpk, qb, qm, cb, cm, found); break;
            default: stay = leaf_window<LEAF, false, 8>(c, s, lsk, lpk, qb, qm, cb, cm, found); break;
        }
        if (stay) continue;
        // leaving the node: the last warp out completes it once its seed is known
        uint32_t left = 0;
        uint64_t x = 0;
        if (lane == 0) {
            if (s.owner) c.slots[gw] = kEmpty;
            __threadfence();  // this warp's seed merges before its exit
            left = atomicSub(&p.active[s.id], 1u);
            __threadfence();  // the merges of the warps that left before it, before the seed is read
            x = atomicMin((unsigned long long *)&c.nodes.seed[s.id], ~0ull);  // an atomic read
        }
        left = __shfl_sync(0xffffffffu, left, 0);
        x = __shfl_sync(0xffffffffu, x, 0);
        if (left == 1 && x != kSeedNotFound) {
            uint32_t won = 0;
            if (lane == 0) won = atomicCAS(&p.claimed[s.id], 0u, 1u) == 0u;
            won = __shfl_sync(0xffffffffu, won, 0);
            if (won) {
                __threadfence();
                if (x >= kSeedFailed) {
                    if (lane == 0) set_error(c.status, RSB_ERR_SEARCH_BUDGET, s.id);
                } else if (s.stage == kStageUpper) {
                    pipe_complete_aggr<LEAF, kStageUpper>(c, p, s.id, x, ask);
                } else if (s.stage == kStageLower) {
                    pipe_complete_aggr<LEAF, kStageLower>(c, p, s.id, x, ask);
                }
                if (lane == 0) atomicAdd(&p.counts[2 * kPipeQueues], 1u);
            }
        }
        s.id = kEmpty;
    }
    uint32_t timed_out = 0;
    if (lane == 0) timed_out = status_code(c.status) == RSB_ERR_TIMEOUT;
    if (__shfl_sync(0xffffffffu, timed_out, 0)) pipe_diagnose(c, p);
}

}  // namespace

namespace search_impl {

template <int LEAF, int SA, int SL>
void launch_pipeline_s(const SearchCtx &c, const PipeCtx &p, const StageSchedule &s, cudaStream_t st) {
    const size_t smem = kWarpsPerCta * pipe_warp_bytes<LEAF, SA, SL>();
    launch_persistent_with(k_pipeline<LEAF, SA, SL>, c, p, smem, s, st);
}

template <int LEAF>
void run_pipeline(const SearchCtx &c, const PipeCtx &p, const StageSchedule &aggr, const StageSchedule &leaf,
                  cudaStream_t st) {
    const bool a8 = aggr.seeds_per_lane == 8;
    switch (leaf.seeds_per_lane) {
        case 4: a8 ? launch_pipeline_s<LEAF, 8, 4>(c, p, aggr, st) : launch_pipeline_s<LEAF, 12, 4>(c, p, aggr, st); break;
        case 12: a8 ? launch_pipeline_s<LEAF, 8, 12>(c, p, aggr, st) : launch_pipeline_s<LEAF, 12, 12>(c, p, aggr, st); break;
        default: a8 ? launch_pipeline_s<LEAF, 8, 8>(c, p, aggr, st) : launch_pipeline_s<LEAF, 12, 8>(c, p, aggr, st); break;
    }
}

}  // namespace search_impl

}  // namespace rsb
