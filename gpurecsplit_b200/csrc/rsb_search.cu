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
//
// Files: rsb_search_common.cuh (helpers and launch sizing), rsb_search_impl.cuh (aggregation
// and leaf kernels, instantiated per leaf size in rsb_search_inst_*.cu), this file (fanout-2
// searches, stage dispatch with the engine's schedule, the evaluation probe).
#include "rsb_search_common.cuh"
#include "rsb_search_stages.h"

namespace rsb {

namespace {

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


}  // namespace

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

uint32_t search_slots_needed(int num_sms) { return (uint32_t)num_sms * 64u; }  // 64 resident warps per SM at most

bool shape_matches_kernels(const Shape &s) { return s.lower == lower_of((int)s.leaf) && s.upper == upper_of((int)s.leaf); }

// ---- stage schedules ------------------------------------------------------------------
// The built-in schedule of every (leaf size, stage, size class): the table that
// gpurecsplit_b200/tune.py measured and wrote (rsb_schedules.inc); entries not in it take
// 12 candidates per lane for aggregation at l >= 12 and 8 otherwise, 8 bases per lane for
// rotation leaves, at full occupancy.
namespace {
struct ScheduleEntry {
    uint8_t leaf, stage, size_class, seeds_per_lane, occupancy_pct;
};
constexpr ScheduleEntry kTunedSchedules[] = {
#include "rsb_schedules.inc"
    {0, 0, 0, 0, 0},  // end (no leaf size 0)
};
}  // namespace

int schedule_size_class(uint64_t keys) { return keys >= (1ull << 24) ? 2 : keys >= (1ull << 20) ? 1 : 0; }

bool schedule_valid(int stage, const StageSchedule &s) {
    if (s.occupancy_pct < 1 || s.occupancy_pct > 100) return false;
    if (stage == kStageUpper || stage == kStageLower)
        return s.seeds_per_lane == 4 || s.seeds_per_lane == 8 || s.seeds_per_lane == 12 || s.seeds_per_lane == 16;
    if (stage == kStageLeafRot) return s.seeds_per_lane == 4 || s.seeds_per_lane == 8 || s.seeds_per_lane == 12;
    return false;
}

StageSchedule default_schedule(int leaf, int stage, int size_class) {
    for (const ScheduleEntry &t : kTunedSchedules)
        if (t.leaf == leaf && t.stage == stage && t.size_class == size_class) return {t.seeds_per_lane, t.occupancy_pct};
    if (stage == kStageUpper || stage == kStageLower) return {leaf >= 12 ? 12 : 8, 100};
    return {8, 100};
}

// ---- pipeline mode: set-up of the work queues --------------------------------------------
namespace {
// Children of aggregation nodes are queued by their parent when it completes.
__global__ void k_pipe_mark(const SearchCtx c, PipeCtx p) {
    const uint32_t base = c.stage_info[kNumStages + kStageUpper];
    const uint32_t cnt = c.stage_info[kStageUpper] + c.stage_info[kStageLower];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint32_t id = c.lists[base + i];  // the lists of stages 17 and 18 are adjacent
        const uint32_t m = c.nodes.size[id];
        const uint32_t split = c.nodes.stage[id] == kStageUpper ? c.sh.lower : c.sh.leaf;
        const uint32_t fan = uint16_t(m + split - 1) / split;
        uint32_t child = id + 1;
        for (uint32_t j = 0; j < fan; ++j) {
            const uint32_t cm = j + 1 < fan ? split : m - (fan - 1) * split;
            if (cm <= 1) continue;
            p.blocked[child] = 1;
            child += c.tab.nodes[cm];
        }
    }
}

// Every other node of stages 17..20 is ready at the launch.
__global__ void k_pipe_fill(const SearchCtx c, PipeCtx p) {
    const uint32_t base = c.stage_info[kNumStages + kStageUpper];
    const uint32_t cnt = c.stage_info[kStageUpper] + c.stage_info[kStageLower] + c.stage_info[kStageLeafRot] +
                         c.stage_info[kStageLeafBF];
    if (blockIdx.x == 0 && threadIdx.x == 0) p.counts[9] = cnt;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const uint32_t id = c.lists[base + i];
        if (p.blocked[id]) continue;
        const uint32_t st = c.nodes.stage[id];
        const uint32_t at = atomicAdd(&p.counts[st - kStageUpper], 1u);
        p.queue[c.stage_info[kNumStages + st] + at] = id;
    }
}
}  // namespace

void search_pipeline(const SearchCtx &c, const PipeCtx &p, uint32_t max_nodes, const StageSchedule &aggr,
                     const StageSchedule &leaf, cudaStream_t st) {
    cudaMemsetAsync(p.queue, 0xFF, (size_t)max_nodes * sizeof(uint32_t), st);
    cudaMemsetAsync(p.counts, 0, kPipeCounters * sizeof(uint32_t), st);
    cudaMemsetAsync(p.active, 0, (size_t)max_nodes * sizeof(uint32_t), st);
    cudaMemsetAsync(p.claimed, 0, (size_t)max_nodes * sizeof(uint32_t), st);
    cudaMemsetAsync(p.blocked, 0, max_nodes, st);
    const int g = std::max(1, std::min<int>(c.num_sms * 8, (int)((max_nodes + 255) / 256)));
    use_max_smem(k_pipe_mark);
    k_pipe_mark<<<g, 256, 0, st>>>(c, p);
    use_max_smem(k_pipe_fill);
    k_pipe_fill<<<g, 256, 0, st>>>(c, p);
    RSB_LEAF_SWITCH(c.sh.leaf, search_impl::run_pipeline, c, p, aggr, leaf, st);
    count_launches(3);
}

void search_higher(const SearchCtx &c, int depth, cudaStream_t st) {
    const size_t smem = kMaxBucketSize * sizeof(uint64_t);
    cudaFuncSetAttribute(k_search_higher, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    use_max_smem(k_search_higher);
    k_search_higher<<<persistent_grid(k_search_higher, smem, c.num_sms, kHigherThreads, c.occupancy_pct), kHigherThreads,
                      smem, st>>>(c, depth);
    count_launches(1);
}

void search_aggr(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st) {
    RSB_LEAF_SWITCH(c.sh.leaf, search_impl::run_aggr, c, stage, s, st);
    count_launches(1);
}
void partition_aggr(const SearchCtx &c, int stage, cudaStream_t st) {
    RSB_LEAF_SWITCH(c.sh.leaf, search_impl::run_partition, c, stage, st);
    count_launches(1);
}
void search_leaves(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st) {
    RSB_LEAF_SWITCH(c.sh.leaf, search_impl::run_leaves, c, stage, s, st);
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
