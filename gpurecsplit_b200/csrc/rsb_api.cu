// C ABI of the construction engine: engine lifetime, the device build pipeline, handles,
// serialization and host/device queries. See include/rsb.h for the contract of each call.
//
// Build pipeline (one CUDA stream, no host synchronisation until the end):
//   keys -> hash128 -> bucket histogram -> scan -> scatter -> per-bucket sort/dup check
//   -> node counts -> scan -> tree emission -> stage lists
//   -> fanout-2 depths (CTA per node) -> upper aggr -> partition -> lower aggr -> partition
//   -> rotation leaves -> brute-force leaves
//   -> bucket bit lengths -> scan -> Rice writer + sentinel -> double Elias-Fano
// It replaces GPURecSplit::hash_gen (GPURecSplit.cuh:637-815), which runs the sort,
// grouping, unpacking and encoding on the host and calls cudaDeviceReset at the end.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "rsb_kernels.cuh"
#include "rsb_query.cuh"
#include "rsb_spooky.cuh"
#include "rsb_tables.h"

using namespace rsb;

namespace {

thread_local cudaError_t g_last_cuda = cudaSuccess;

#define RSB_CK(call)                           \
    do {                                       \
        cudaError_t e_ = (call);               \
        if (e_ != cudaSuccess) {               \
            g_last_cuda = e_;                  \
            return RSB_ERR_CUDA;               \
        }                                      \
    } while (0)

template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t cap = 0;
};

template <typename T>
rsb_status ensure(DBuf<T> &b, size_t n) {
    if (n == 0) n = 1;
    if (b.p && n <= b.cap) return RSB_OK;
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
    const size_t want = n + n / 8;  // headroom against frequent regrowth
    cudaError_t e = cudaMalloc((void **)&b.p, want * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        b.p = nullptr;
        return RSB_ERR_OOM;
    }
    b.cap = want;
    return RSB_OK;
}

template <typename T>
void release(DBuf<T> &b) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.cap = 0;
}

constexpr int kNumEvents = 6 + kNumStages;  // start, hashed/partitioned, stage boundaries, encoded

}  // namespace

struct rsb_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 0;
    int occupancy_pct = 100;
    uint32_t budget_shift = 10;
    uint64_t budget_min = 1ull << 16;
    std::map<uint32_t, std::pair<uint32_t *, uint32_t *>> tables;  // (leaf, rotate) -> device memo, nodes
    std::map<uint32_t, StageSchedule> schedules;  // (leaf, stage, size class) -> rsb_engine_set_schedule
    bool pipeline = false;                         // stages 17..20 in one persistent launch (rsb_engine_set_pipeline)
    uint64_t watchdog_ns = 0;                      // bound on a pipeline launch (rsb_engine_set_watchdog), 0: none
    DBuf<uint32_t> pq, pcounts, pactive, pclaimed;
    DBuf<uint8_t> pblocked;
    int last_seeds_per_lane[kNumStages] = {};      // schedules of the last build's stages (rsb_stats)
    DBuf<uint64_t> keys128, raw_u64, offsets, sorted, acc, node_base, scan_tmp, pos_acc, seed;
    DBuf<uint32_t> counts, node_count, lists, stage_info, sched, slots, bits, fixed_bits, nstart, nwin;
    DBuf<uint16_t> nsize;
    DBuf<uint8_t> nstage, bytes;
    DBuf<DevStatus> status;
    DBuf<EfParams> efp;
    DBuf<uint64_t> windows;  // candidate windows per search stage (rsb_stats)
    DBuf<uint32_t> verify_seen;  // RSB_VERIFY: one bit per value of the function
    // batched construction
    DBuf<uint64_t> set_key, set_bucket, set_bits, word_base, ef_base, out_block;
    DBuf<uint32_t> set_nb, bucket_id, set_words, ef_words;
    DBuf<EfParams> set_ef;
    cudaEvent_t ev[kNumEvents] = {};
};

struct rsb_mphf {
    uint32_t leaf = 0;
    bool rotate = true;
    uint64_t bucket_size = 0, keys_count = 0, nbuckets = 0;
    EfParams ef{};
    int device = -1;
    uint64_t *d_block = nullptr;  // desc | lower | upper_cum | upper_pos | jump (device copy)
    uint64_t desc_cap = 0, lower_cap = 0, cum_cap = 0, pos_cap = 0, jump_cap = 0;
    bool host_valid = false;
    std::vector<uint64_t> desc, lower, upper_cum, upper_pos, jump;
    std::vector<uint64_t> seeds;
    std::vector<uint32_t> sizes;
    // part builds (rsb_build_part_hash128): the range of the whole function's buckets and the
    // per-bucket key and descriptor-bit offsets of the part
    uint64_t part_lo = 0, part_hi = 0, part_nb_total = 0;
    std::vector<uint64_t> bucket_acc, bucket_pos;
    rsb_stats stats{};
    const LeafTables *tab = nullptr;

    uint64_t *d_desc() const { return d_block; }
    uint64_t *d_lower() const { return d_block + desc_cap; }
    uint64_t *d_cum() const { return d_lower() + lower_cap; }
    uint64_t *d_pos() const { return d_cum() + cum_cap; }
    uint64_t *d_jump() const { return d_pos() + pos_cap; }

    MphfView host_view() const {
        MphfView v{};
        v.sh = tab->shape;
        v.nbuckets = nbuckets;
        v.desc = desc.data();
        v.desc_words = desc.size();
        v.u_cum_keys = ef.u_cum_keys;
        v.u_position = ef.u_position;
        v.l_cum_keys = ef.l_cum_keys;
        v.l_position = ef.l_position;
        v.cum_keys_min_delta = ef.cum_keys_min_delta;
        v.min_diff = ef.min_diff;
        v.bits_per_key_fixed_point = ef.bits_per_key_fixed_point;
        v.lower = lower.data();
        v.upper_cum = upper_cum.data();
        v.upper_pos = upper_pos.data();
        v.jump = jump.data();
        v.lower_words = lower.size();
        v.cum_words = upper_cum.size();
        v.pos_words = upper_pos.size();
        v.jump_words = jump.size();
        v.memo = tab->memo.data();
        return v;
    }
};

namespace {

rsb_status get_device_tables(rsb_engine *e, const LeafTables &t, uint32_t leaf, bool rotate, DevTables &out) {
    const uint32_t key = leaf * 2 + (rotate ? 1 : 0);
    auto it = e->tables.find(key);
    if (it == e->tables.end()) {
        uint32_t *d = nullptr;
        if (cudaMalloc((void **)&d, 2 * kMaxBucketSize * sizeof(uint32_t)) != cudaSuccess) {
            cudaGetLastError();
            return RSB_ERR_OOM;
        }
        RSB_CK(cudaMemcpy(d, t.memo.data(), kMaxBucketSize * sizeof(uint32_t), cudaMemcpyHostToDevice));
        RSB_CK(cudaMemcpy(d + kMaxBucketSize, t.nodes.data(), kMaxBucketSize * sizeof(uint32_t), cudaMemcpyHostToDevice));
        it = e->tables.emplace(key, std::make_pair(d, d + kMaxBucketSize)).first;
    }
    out.memo = it->second.first;
    out.nodes = it->second.second;
    return RSB_OK;
}

float elapsed(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return ms;
}

uint64_t jump_words_for(uint64_t nb) {
    constexpr uint64_t q = 256, super_q = 1 << 14, sqs = 1 + (super_q / q) / 4;
    uint64_t jw = (nb / super_q) * sqs * 2;
    if (nb % super_q != 0) jw += (1 + ((nb % super_q + q - 1) / q + 3) / 4) * 2;
    return jw;
}

rsb_status copy_to_host(rsb_mphf *h, cudaStream_t st) {
    if (h->host_valid) return RSB_OK;
    if (!h->d_block) return RSB_ERR_INTERNAL;
    h->desc.resize(h->ef.desc_words);
    h->lower.resize(h->ef.lower_words);
    h->upper_cum.resize(h->ef.cum_words);
    h->upper_pos.resize(h->ef.pos_words);
    h->jump.resize(h->ef.jump_words);
    RSB_CK(cudaMemcpyAsync(h->desc.data(), h->d_desc(), h->desc.size() * 8, cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaMemcpyAsync(h->lower.data(), h->d_lower(), h->lower.size() * 8, cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaMemcpyAsync(h->upper_cum.data(), h->d_cum(), h->upper_cum.size() * 8, cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaMemcpyAsync(h->upper_pos.data(), h->d_pos(), h->upper_pos.size() * 8, cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaMemcpyAsync(h->jump.data(), h->d_jump(), h->jump.size() * 8, cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaStreamSynchronize(st));
    h->host_valid = true;
    return RSB_OK;
}

// Every search stage in dependency order: fanout-2 depths, then each aggregation level
// followed by its partition, then the leaves. Records the stage-boundary events.
uint32_t schedule_key(uint32_t leaf, int stage, int size_class) { return leaf * 256u + (uint32_t)stage * 4u + size_class; }

// The engine's schedule of one stage: a rsb_engine_set_schedule override or the built-in table.
StageSchedule engine_schedule(const rsb_engine *e, uint32_t leaf, int stage, uint64_t keys) {
    const int sc = schedule_size_class(keys);
    auto it = e->schedules.find(schedule_key(leaf, stage, sc));
    return it != e->schedules.end() ? it->second : default_schedule((int)leaf, stage, sc);
}

// After a failed pipeline-mode build: with RSB_DEBUG set in the environment, prints the
// queue counters and, when a bounded wait gave up, the kernel's snapshot of the unfinished
// nodes (pipe_diagnose in rsb_pipeline_impl.cuh) to stderr.
void report_pipeline_state(rsb_engine *e, int code, uint64_t detail, cudaStream_t st) {
    if (!e->pipeline || !e->pcounts.p || !std::getenv("RSB_DEBUG")) return;
    uint32_t d[kPipeCounters];
    if (cudaMemcpyAsync(d, e->pcounts.p, sizeof(d), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return;
    std::fprintf(stderr,
                 "rsb pipeline failed (status %d, detail %llu): why=%u tails=%u,%u,%u,%u heads=%u,%u,%u,%u "
                 "done=%u/%u unfinished=%u active=%u seed_known=%u parent_queued=%u never_joined=%u first=%u "
                 "stage=%u size=%u seed=%016llx first_active=%u first_windows=%u first_parent_queued=%u "
                 "head_slots=%x,%x,%x,%x\n",
                 code, (unsigned long long)detail, d[11], d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9],
                 d[12], d[13], d[14], d[15], d[16], d[17], d[18] & 0xFF, d[18] >> 8,
                 (unsigned long long)d[19] | (unsigned long long)d[20] << 32, d[21], d[22], d[23], d[24], d[25], d[26],
                 d[27]);
}

cudaError_t enqueue_searches(rsb_engine *e, const SearchCtx &sc, const LeafTables &lt, uint64_t keys, cudaStream_t st) {
    cudaError_t err;
    const uint32_t leaf = sc.sh.leaf;
    for (int s = 0; s < kNumStages; ++s) e->last_seeds_per_lane[s] = 0;
    for (uint32_t d = 0; d < lt.max_higher_depth && d < (uint32_t)kMaxHigherDepth; ++d) {
        search_higher(sc, (int)d, st);
        if ((err = cudaEventRecord(e->ev[2 + d], st)) != cudaSuccess) return err;
    }
    if (e->pipeline) {
        // one launch for stages 17..20; its time is reported as stage 17's
        const uint64_t max_nodes = keys + 1;
        if (ensure(e->pq, max_nodes) != RSB_OK || ensure(e->pcounts, kPipeCounters) != RSB_OK ||
            ensure(e->pactive, max_nodes) != RSB_OK || ensure(e->pclaimed, max_nodes) != RSB_OK ||
            ensure(e->pblocked, max_nodes) != RSB_OK)
            return cudaErrorMemoryAllocation;
        if ((err = cudaMemsetAsync(sc.slots, 0xFF, sc.nslots * sizeof(uint32_t), st)) != cudaSuccess) return err;
        const StageSchedule sa = engine_schedule(e, leaf, kStageLower, keys);
        const StageSchedule sl = engine_schedule(e, leaf, kStageLeafRot, keys);
        const StageSchedule aggr{sa.seeds_per_lane <= 8 ? 8 : 12, sa.occupancy_pct};
        const StageSchedule lf{sl.seeds_per_lane, 100};
        e->last_seeds_per_lane[kStageUpper] = e->last_seeds_per_lane[kStageLower] = aggr.seeds_per_lane;
        e->last_seeds_per_lane[kStageLeafRot] = lf.seeds_per_lane;
        e->last_seeds_per_lane[kStageLeafBF] = 8;
        PipeCtx p{e->pq.p, e->pcounts.p, e->pactive.p, e->pclaimed.p, e->pblocked.p};
        search_pipeline(sc, p, (uint32_t)max_nodes, aggr, lf, st);
        for (int stage = kStageUpper; stage <= kStageLeafBF; ++stage)
            if ((err = cudaEventRecord(e->ev[2 + stage], st)) != cudaSuccess) return err;
        return cudaGetLastError();
    }
    for (int stage : {kStageUpper, kStageLower}) {
        if ((err = cudaMemsetAsync(sc.slots, 0xFF, sc.nslots * sizeof(uint32_t), st)) != cudaSuccess) return err;
        const StageSchedule s = engine_schedule(e, leaf, stage, keys);
        e->last_seeds_per_lane[stage] = s.seeds_per_lane;
        search_aggr(sc, stage, s, st);
        partition_aggr(sc, stage, st);
        if ((err = cudaEventRecord(e->ev[2 + stage], st)) != cudaSuccess) return err;
    }
    for (int stage : {kStageLeafRot, kStageLeafBF}) {
        if ((err = cudaMemsetAsync(sc.slots, 0xFF, sc.nslots * sizeof(uint32_t), st)) != cudaSuccess) return err;
        const StageSchedule s = stage == kStageLeafRot ? engine_schedule(e, leaf, stage, keys) : StageSchedule{8, 100};
        e->last_seeds_per_lane[stage] = s.seeds_per_lane;
        search_leaves(sc, stage, s, st);
        if ((err = cudaEventRecord(e->ev[2 + stage], st)) != cudaSuccess) return err;
    }
    return cudaGetLastError();
}

// Per-stage device times of the last build from the engine's events.
void fill_stage_times(rsb_engine *e, const LeafTables &lt, rsb_stats &S) {
    S.ms_total = elapsed(e->ev[0], e->ev[kNumEvents - 1]);
    S.ms_partition = elapsed(e->ev[0], e->ev[1]);
    cudaEvent_t prev = e->ev[1];
    for (int s = 0; s < kNumStages; ++s) {
        const bool recorded = (s < (int)lt.max_higher_depth && s < kMaxHigherDepth) || s >= kStageUpper;
        if (!recorded) continue;
        S.ms_search[s] = elapsed(prev, e->ev[2 + s]);
        prev = e->ev[2 + s];
    }
    S.ms_encode = elapsed(prev, e->ev[kNumEvents - 1]);
}

// View of a function's device copy for device queries.
MphfView device_view(const rsb_mphf *h, const DevTables &tab) {
    MphfView v{};
    v.sh = h->tab->shape;
    v.nbuckets = h->nbuckets;
    v.desc = h->d_desc();
    v.desc_words = h->ef.desc_words;
    v.u_cum_keys = h->ef.u_cum_keys;
    v.u_position = h->ef.u_position;
    v.l_cum_keys = h->ef.l_cum_keys;
    v.l_position = h->ef.l_position;
    v.cum_keys_min_delta = h->ef.cum_keys_min_delta;
    v.min_diff = h->ef.min_diff;
    v.bits_per_key_fixed_point = h->ef.bits_per_key_fixed_point;
    v.lower = h->d_lower();
    v.upper_cum = h->d_cum();
    v.upper_pos = h->d_pos();
    v.jump = h->d_jump();
    v.lower_words = h->ef.lower_words;
    v.cum_words = h->ef.cum_words;
    v.pos_words = h->ef.pos_words;
    v.jump_words = h->ef.jump_words;
    v.memo = tab.memo;
    return v;
}

// The build proper. keys128 is device memory holding n (first, second) pairs.
// `hash_keys` (optional) enqueues the key-hashing kernel that produces keys128; it runs
// after the build's start event so that hashing is part of the measured build.
// `nb_override` (part builds) sets the bucket count instead of ceil(n / bucket_size), and
// `keep_buckets` keeps the per-bucket key and bit offsets on the host (rsb_part_export).
rsb_status build_device(rsb_engine *e, const uint64_t *keys128, uint64_t n, uint64_t bucket_size, uint32_t leaf,
                        uint32_t flags, rsb_mphf **out, bool keep_seeds,
                        const std::function<void()> &hash_keys = std::function<void()>(), uint64_t nb_override = 0,
                        bool keep_buckets = false) {
    const bool rotate = (flags & RSB_ROTATE) != 0;
    const LeafTables &lt = leaf_tables(leaf, rotate);
    if (!shape_matches_kernels(lt.shape)) return RSB_ERR_INTERNAL;
    DevTables tab;
    rsb_status rs = get_device_tables(e, lt, leaf, rotate, tab);
    if (rs != RSB_OK) return rs;
    cudaStream_t st = e->stream;
    const uint64_t nb = nb_override ? nb_override : std::max<uint64_t>(1, (n + bucket_size - 1) / bucket_size);
    const uint64_t max_nodes = n + 1;
    const uint32_t nslots = search_slots_needed(e->num_sms);

#define RSB_ENSURE(buf, cnt)                    \
    do {                                        \
        rsb_status s_ = ensure(buf, cnt);       \
        if (s_ != RSB_OK) return s_;            \
    } while (0)
    RSB_ENSURE(e->sorted, n);
    RSB_ENSURE(e->counts, nb);
    RSB_ENSURE(e->acc, nb + 1);
    RSB_ENSURE(e->node_count, nb);
    RSB_ENSURE(e->node_base, nb + 1);
    RSB_ENSURE(e->scan_tmp, scan_blocks(nb + 1) + 8);
    RSB_ENSURE(e->nstart, max_nodes);
    RSB_ENSURE(e->nsize, max_nodes);
    RSB_ENSURE(e->nstage, max_nodes);
    RSB_ENSURE(e->seed, max_nodes);
    RSB_ENSURE(e->nwin, max_nodes);
    RSB_ENSURE(e->lists, max_nodes);
    RSB_ENSURE(e->stage_info, 3 * kNumStages);
    RSB_ENSURE(e->sched, 2 * kNumStages);
    RSB_ENSURE(e->slots, nslots);
    RSB_ENSURE(e->bits, nb);
    RSB_ENSURE(e->fixed_bits, nb);
    RSB_ENSURE(e->pos_acc, nb + 1);
    RSB_ENSURE(e->status, 1);
    RSB_ENSURE(e->efp, 1);
    RSB_ENSURE(e->windows, kNumStages);

    auto *h = new (std::nothrow) rsb_mphf;
    if (!h) return RSB_ERR_OOM;
    h->leaf = leaf;
    h->rotate = rotate;
    h->bucket_size = bucket_size;
    h->keys_count = n;
    h->nbuckets = nb;
    h->tab = &lt;
    h->device = e->device;
    // Output capacities (upper bounds; the encoder reports the exact sizes).
    h->desc_cap = (8 * n + 65536) / 64 + 16;
    h->lower_cap = ((nb + 1) * 56 + 63) / 64 + 2;
    h->cum_cap = (3 * (nb + 1) + 63) / 64 + 2;
    h->pos_cap = h->cum_cap;
    h->jump_cap = jump_words_for(nb) + 2;
    const uint64_t block_words = h->desc_cap + h->lower_cap + h->cum_cap + h->pos_cap + h->jump_cap;
    if (cudaMallocAsync((void **)&h->d_block, block_words * 8, st) != cudaSuccess) {
        cudaGetLastError();
        delete h;
        return RSB_ERR_OOM;
    }
    auto fail = [&](rsb_status s) {
        if (h->d_block) cudaFreeAsync(h->d_block, st);
        cudaStreamSynchronize(st);
        delete h;
        return s;
    };
#define RSB_CKH(call)                         \
    do {                                      \
        cudaError_t e_ = (call);              \
        if (e_ != cudaSuccess) {              \
            g_last_cuda = e_;                 \
            return fail(RSB_ERR_CUDA);        \
        }                                     \
    } while (0)

    NodeArrays nodes{e->nstart.p, e->nsize.p, e->nstage.p, e->seed.p, e->nwin.p};
    ScanTmp stmp{e->scan_tmp.p, e->scan_tmp.cap};
    const uint64_t *node_total = e->node_base.p + nb;
    const uint64_t launches0 = launches_so_far();

    RSB_CKH(cudaEventRecord(e->ev[0], st));
    if (hash_keys) hash_keys();
    RSB_CKH(cudaMemsetAsync(e->status.p, 0, sizeof(DevStatus), st));
    RSB_CKH(cudaMemsetAsync(e->efp.p, 0, sizeof(EfParams), st));
    RSB_CKH(cudaMemsetAsync(e->windows.p, 0, kNumStages * sizeof(uint64_t), st));
    RSB_CKH(cudaMemsetAsync(e->sched.p, 0, 2 * kNumStages * sizeof(uint32_t), st));

    // ---- buckets ----
    launch_bucket_count(keys128, n, nb, e->counts.p, st);
    launch_bucket_check(e->counts.p, nb, e->status.p, st);
    exclusive_scan_u32(e->counts.p, e->acc.p, nb, stmp, st);
    launch_bucket_scatter(keys128, n, nb, e->acc.p, e->counts.p, e->sorted.p, st);
    launch_bucket_dupcheck(e->sorted.p, e->acc.p, nb, e->status.p, st);
    // ---- tree ----
    launch_bucket_nodes(e->acc.p, nb, tab, e->node_count.p, st);
    exclusive_scan_u32(e->node_count.p, e->node_base.p, nb, stmp, st);
    RSB_CKH(cudaMemsetAsync(e->seed.p, 0xFF, max_nodes * sizeof(uint64_t), st));
    RSB_CKH(cudaMemsetAsync(e->nwin.p, 0, max_nodes * sizeof(uint32_t), st));
    launch_tree_emit(e->acc.p, nb, e->node_base.p, lt.shape, nodes, st);
    launch_stage_lists(e->nstage.p, node_total, (uint32_t)max_nodes, e->stage_info.p, e->lists.p, st);
    RSB_CKH(cudaGetLastError());
    RSB_CKH(cudaEventRecord(e->ev[1], st));

    // ---- searches ----
    SearchCtx sc{};
    sc.sh = lt.shape;
    sc.node_total = node_total;
    sc.stage_info = e->stage_info.p;
    sc.lists = e->lists.p;
    sc.nodes = nodes;
    sc.keys = e->sorted.p;
    sc.tab = tab;
    sc.status = e->status.p;
    sc.sched = e->sched.p;
    sc.slots = e->slots.p;
    sc.nslots = nslots;
    sc.budget_shift = e->budget_shift;
    sc.budget_min = e->budget_min;
    sc.num_sms = e->num_sms;
    sc.occupancy_pct = e->occupancy_pct;
    sc.watchdog_ns = e->watchdog_ns;
    RSB_CKH(enqueue_searches(e, sc, lt, n, st));

    // ---- encoding ----
    launch_bucket_bits(e->node_base.p, nb, nodes, tab, e->bits.p, e->fixed_bits.p, e->status.p, st);
    exclusive_scan_u32(e->bits.p, e->pos_acc.p, nb, stmp, st);
    RSB_CKH(cudaMemsetAsync(h->d_block, 0, block_words * 8, st));
    launch_write_rice(e->node_base.p, nb, nodes, tab, e->pos_acc.p, e->fixed_bits.p, h->d_desc(), h->desc_cap, e->efp.p,
                      e->status.p, st);
    launch_ef_build(e->acc.p, e->pos_acc.p, nb, n, e->efp.p, h->d_lower(), h->lower_cap, h->d_cum(), h->cum_cap,
                    h->d_pos(), h->pos_cap, h->d_jump(), h->jump_cap, e->status.p, st);
    launch_evals(node_total, nodes, leaf, rotate ? 1 : 0, e->efp.p, e->windows.p, st);
    RSB_CKH(cudaGetLastError());
    RSB_CKH(cudaEventRecord(e->ev[kNumEvents - 1], st));
    // Wait for the build before the pageable copies below: a device-to-host copy into pageable
    // memory holds the calling thread inside the driver until its stream reaches it, which
    // would also hold back other threads' pageable copies (another engine's build) for the
    // whole duration of this build.
    RSB_CKH(cudaEventSynchronize(e->ev[kNumEvents - 1]));

    DevStatus dst{};
    uint32_t stage_counts[kNumStages];
    RSB_CKH(cudaMemcpyAsync(&dst, e->status.p, sizeof(dst), cudaMemcpyDeviceToHost, st));
    uint64_t windows[kNumStages];
    RSB_CKH(cudaMemcpyAsync(&h->ef, e->efp.p, sizeof(EfParams), cudaMemcpyDeviceToHost, st));
    RSB_CKH(cudaMemcpyAsync(windows, e->windows.p, sizeof(windows), cudaMemcpyDeviceToHost, st));
    RSB_CKH(cudaMemcpyAsync(stage_counts, e->stage_info.p, sizeof(stage_counts), cudaMemcpyDeviceToHost, st));
    RSB_CKH(cudaStreamSynchronize(st));
    if (dst.code != 0) report_pipeline_state(e, dst.code, dst.detail, st);
    if (dst.code != 0) return fail((rsb_status)dst.code);

    // stats
    rsb_stats &S = h->stats;
    S.keys = n;
    S.buckets = nb;
    S.evals_alg = h->ef.evals_alg;
    for (int s = 0; s < kNumStages; ++s) {
        S.evals_stage[s] = h->ef.evals_stage[s];
        S.windows_stage[s] = windows[s];
        S.window_candidates[s] = 32u * (uint32_t)e->last_seeds_per_lane[s];
    }
    S.kernel_launches = launches_so_far() - launches0;
    S.descriptor_bits = h->ef.total_bits;
    uint64_t tot = 0;
    for (int s = 0; s < kNumStages; ++s) {
        S.nodes_per_stage[s] = stage_counts[s];
        tot += stage_counts[s];
    }
    S.nodes = tot;
    fill_stage_times(e, lt, S);

    if (keep_seeds) {
        h->seeds.resize(tot);
        h->sizes.resize(tot);
        std::vector<uint16_t> sz(tot);
        if (tot) {
            RSB_CKH(cudaMemcpy(h->seeds.data(), e->seed.p, tot * 8, cudaMemcpyDeviceToHost));
            RSB_CKH(cudaMemcpy(sz.data(), e->nsize.p, tot * 2, cudaMemcpyDeviceToHost));
        }
        for (uint64_t i = 0; i < tot; ++i) h->sizes[i] = sz[i];
    }
    if (flags & RSB_VERIFY) {
        RSB_CKH(ensure(e->verify_seen, (n + 31) / 32 + 1) == RSB_OK ? cudaSuccess : cudaErrorMemoryAllocation);
        RSB_CKH(cudaMemsetAsync(e->status.p, 0, sizeof(DevStatus), st));
        launch_verify(device_view(h, tab), keys128, n, e->acc.p, e->pos_acc.p, nb, e->verify_seen.p, e->status.p, st);
        RSB_CKH(cudaGetLastError());
        DevStatus vst{};
        RSB_CKH(cudaMemcpyAsync(&vst, e->status.p, sizeof(vst), cudaMemcpyDeviceToHost, st));
        RSB_CKH(cudaStreamSynchronize(st));
        if (vst.code != 0) return fail(RSB_ERR_INTERNAL);
    }
    if (keep_buckets) {
        h->bucket_acc.resize(nb + 1);
        h->bucket_pos.resize(nb + 1);
        RSB_CKH(cudaMemcpy(h->bucket_acc.data(), e->acc.p, (nb + 1) * 8, cudaMemcpyDeviceToHost));
        RSB_CKH(cudaMemcpy(h->bucket_pos.data(), e->pos_acc.p, (nb + 1) * 8, cudaMemcpyDeviceToHost));
    }
    if (!(flags & RSB_DEVICE_ONLY)) {
        rsb_status s = copy_to_host(h, st);
        if (s != RSB_OK) return fail(s);
    }
    *out = h;
    return RSB_OK;
}

// Device scratch of a batched build of n keys in nsets sets and nb_total buckets whose
// encoded output takes block_words words (also used to pre-size an engine).
rsb_status ensure_batch_buffers(rsb_engine *e, uint64_t n, uint64_t nb_total, uint32_t nsets, uint64_t block_words) {
    const uint64_t max_nodes = n + 1;
    const uint32_t nslots = search_slots_needed(e->num_sms);
    RSB_ENSURE(e->sorted, n);
    RSB_ENSURE(e->set_key, nsets + 1);
    RSB_ENSURE(e->set_nb, nsets);
    RSB_ENSURE(e->set_bucket, nsets + 1);
    RSB_ENSURE(e->bucket_id, n);
    RSB_ENSURE(e->counts, nb_total);
    RSB_ENSURE(e->acc, nb_total + 1);
    RSB_ENSURE(e->node_count, nb_total);
    RSB_ENSURE(e->node_base, nb_total + 1);
    RSB_ENSURE(e->scan_tmp, scan_blocks(std::max<uint64_t>(nb_total, nsets) + 1) + 8);
    RSB_ENSURE(e->nstart, max_nodes);
    RSB_ENSURE(e->nsize, max_nodes);
    RSB_ENSURE(e->nstage, max_nodes);
    RSB_ENSURE(e->seed, max_nodes);
    RSB_ENSURE(e->nwin, max_nodes);
    RSB_ENSURE(e->lists, max_nodes);
    RSB_ENSURE(e->stage_info, 3 * kNumStages);
    RSB_ENSURE(e->sched, 2 * kNumStages);
    RSB_ENSURE(e->slots, nslots);
    RSB_ENSURE(e->bits, nb_total);
    RSB_ENSURE(e->fixed_bits, nb_total);
    RSB_ENSURE(e->pos_acc, nb_total + 1);
    RSB_ENSURE(e->status, 1);
    RSB_ENSURE(e->efp, 1);
    RSB_ENSURE(e->windows, kNumStages);
    RSB_ENSURE(e->set_words, nsets);
    RSB_ENSURE(e->set_bits, nsets);
    RSB_ENSURE(e->word_base, nsets + 1);
    RSB_ENSURE(e->ef_words, 4 * (uint64_t)nsets);
    RSB_ENSURE(e->ef_base, 4 * ((uint64_t)nsets + 1));
    RSB_ENSURE(e->set_ef, nsets);
    RSB_ENSURE(e->out_block, block_words);
    return RSB_OK;
}

// Batched construction: nsets independent key sets (set s = keys [h_off[s], h_off[s+1]))
// in one device pipeline. Sets share the global bucket space, so the tree, the stage lists
// and every search kernel run once for all sets; bucket assignment and the encoders are
// set-aware. outs[s] receives a host-side function identical to the plain build of set s.
rsb_status build_batch_device(rsb_engine *e, const uint64_t *keys128, const uint64_t *h_off, uint32_t nsets,
                              uint64_t bucket_size, uint32_t leaf, uint32_t flags, rsb_mphf **outs, rsb_stats *stats,
                              const std::function<void()> &hash_keys) {
    const bool rotate = (flags & RSB_ROTATE) != 0;
    const LeafTables &lt = leaf_tables(leaf, rotate);
    if (!shape_matches_kernels(lt.shape)) return RSB_ERR_INTERNAL;
    DevTables tab;
    rsb_status rs = get_device_tables(e, lt, leaf, rotate, tab);
    if (rs != RSB_OK) return rs;
    cudaStream_t st = e->stream;
    const uint64_t n = h_off[nsets];
    std::vector<uint64_t> set_nb(nsets);
    uint64_t nb_total = 0, lower_cap = 0, cum_cap = 0, jump_cap = 0;
    for (uint32_t s = 0; s < nsets; ++s) {
        const uint64_t ns = h_off[s + 1] - h_off[s];
        const uint64_t nb = std::max<uint64_t>(1, (ns + bucket_size - 1) / bucket_size);
        set_nb[s] = nb;
        nb_total += nb;
        lower_cap += ((nb + 1) * 56 + 63) / 64 + 2;
        cum_cap += (3 * (nb + 1) + 63) / 64 + 2;
        jump_cap += jump_words_for(nb) + 2;
    }
    if (nb_total >= (1ull << 32) - 1) return RSB_ERR_BAD_ARG;
    const uint64_t desc_cap = (8 * n) / 64 + 3 * (uint64_t)nsets + 16;
    const uint64_t block_words = desc_cap + lower_cap + 2 * cum_cap + jump_cap;
    rs = ensure_batch_buffers(e, n, nb_total, nsets, block_words);
    if (rs != RSB_OK) return rs;
    const uint64_t max_nodes = n + 1;
    const uint32_t nslots = search_slots_needed(e->num_sms);

    NodeArrays nodes{e->nstart.p, e->nsize.p, e->nstage.p, e->seed.p, e->nwin.p};
    ScanTmp stmp{e->scan_tmp.p, e->scan_tmp.cap};
    const uint64_t *node_total = e->node_base.p + nb_total;
    const uint64_t launches0 = launches_so_far();
    uint64_t *desc = e->out_block.p, *lower = desc + desc_cap, *ucum = lower + lower_cap, *upos = ucum + cum_cap,
             *jump = upos + cum_cap;
    uint32_t *lw = e->ef_words.p, *cw = lw + nsets, *pw = cw + nsets, *jw = pw + nsets;
    uint64_t *lb = e->ef_base.p, *cb = lb + nsets + 1, *pb = cb + nsets + 1, *jb = pb + nsets + 1;

    RSB_CK(cudaEventRecord(e->ev[0], st));
    if (hash_keys) hash_keys();
    RSB_CK(cudaMemsetAsync(e->status.p, 0, sizeof(DevStatus), st));
    RSB_CK(cudaMemsetAsync(e->efp.p, 0, sizeof(EfParams), st));
    RSB_CK(cudaMemsetAsync(e->windows.p, 0, kNumStages * sizeof(uint64_t), st));
    RSB_CK(cudaMemsetAsync(e->sched.p, 0, 2 * kNumStages * sizeof(uint32_t), st));
    RSB_CK(cudaMemcpyAsync(e->set_key.p, h_off, (nsets + 1) * 8, cudaMemcpyHostToDevice, st));
    // ---- buckets of all sets ----
    launch_set_nbuckets(e->set_key.p, nsets, bucket_size, e->set_nb.p, st);
    exclusive_scan_u32(e->set_nb.p, e->set_bucket.p, nsets, stmp, st);
    launch_set_bucket_ids(keys128, n, e->set_key.p, e->set_bucket.p, nsets, nb_total, e->bucket_id.p, e->counts.p, st);
    launch_bucket_check(e->counts.p, nb_total, e->status.p, st);
    exclusive_scan_u32(e->counts.p, e->acc.p, nb_total, stmp, st);
    launch_set_scatter(keys128, n, e->set_key.p, e->set_bucket.p, nsets, e->bucket_id.p, e->acc.p, e->counts.p, nb_total,
                       e->sorted.p, st);
    launch_bucket_dupcheck(e->sorted.p, e->acc.p, nb_total, e->status.p, st);
    // ---- tree ----
    launch_bucket_nodes(e->acc.p, nb_total, tab, e->node_count.p, st);
    exclusive_scan_u32(e->node_count.p, e->node_base.p, nb_total, stmp, st);
    RSB_CK(cudaMemsetAsync(e->seed.p, 0xFF, max_nodes * sizeof(uint64_t), st));
    RSB_CK(cudaMemsetAsync(e->nwin.p, 0, max_nodes * sizeof(uint32_t), st));
    launch_tree_emit(e->acc.p, nb_total, e->node_base.p, lt.shape, nodes, st);
    launch_stage_lists(e->nstage.p, node_total, (uint32_t)max_nodes, e->stage_info.p, e->lists.p, st);
    RSB_CK(cudaGetLastError());
    RSB_CK(cudaEventRecord(e->ev[1], st));
    // ---- searches (all sets at once) ----
    SearchCtx sc{};
    sc.sh = lt.shape;
    sc.node_total = node_total;
    sc.stage_info = e->stage_info.p;
    sc.lists = e->lists.p;
    sc.nodes = nodes;
    sc.keys = e->sorted.p;
    sc.tab = tab;
    sc.status = e->status.p;
    sc.sched = e->sched.p;
    sc.slots = e->slots.p;
    sc.nslots = nslots;
    sc.budget_shift = e->budget_shift;
    sc.budget_min = e->budget_min;
    sc.num_sms = e->num_sms;
    sc.occupancy_pct = e->occupancy_pct;
    sc.watchdog_ns = e->watchdog_ns;
    RSB_CK(enqueue_searches(e, sc, lt, n, st));
    // ---- per-set encoding ----
    launch_bucket_bits(e->node_base.p, nb_total, nodes, tab, e->bits.p, e->fixed_bits.p, e->status.p, st);
    exclusive_scan_u32(e->bits.p, e->pos_acc.p, nb_total, stmp, st);
    launch_set_desc_words(e->pos_acc.p, e->set_bucket.p, nsets, e->set_words.p, e->set_bits.p, st);
    exclusive_scan_u32(e->set_words.p, e->word_base.p, nsets, stmp, st);
    RSB_CK(cudaMemsetAsync(e->out_block.p, 0, block_words * 8, st));
    launch_set_write_rice(e->node_base.p, nb_total, nodes, tab, e->pos_acc.p, e->fixed_bits.p, e->set_bucket.p, nsets,
                          e->word_base.p, e->set_bits.p, desc, desc_cap, e->status.p, st);
    launch_set_ef_params(e->acc.p, e->pos_acc.p, e->set_bucket.p, nsets, e->set_ef.p, lw, cw, pw, jw, st);
    exclusive_scan_u32(lw, lb, nsets, stmp, st);
    exclusive_scan_u32(cw, cb, nsets, stmp, st);
    exclusive_scan_u32(pw, pb, nsets, stmp, st);
    exclusive_scan_u32(jw, jb, nsets, stmp, st);
    launch_set_ef_fill(e->acc.p, e->pos_acc.p, e->set_bucket.p, nsets, e->set_ef.p, lb, cb, pb, jb, lower, ucum, upos,
                       jump, st);
    launch_evals(node_total, nodes, leaf, rotate ? 1 : 0, e->efp.p, e->windows.p, st);
    RSB_CK(cudaGetLastError());
    RSB_CK(cudaEventRecord(e->ev[kNumEvents - 1], st));
    // Wait for the build before the pageable copies below: a device-to-host copy into pageable
    // memory holds the calling thread inside the driver until its stream reaches it, which
    // would also hold back other threads' pageable copies (another engine's build) for the
    // whole duration of this build.
    RSB_CK(cudaEventSynchronize(e->ev[kNumEvents - 1]));

    DevStatus dst{};
    EfParams totals{};
    uint32_t stage_counts[kNumStages];
    std::vector<EfParams> sef(nsets);
    std::vector<uint64_t> bases(4 * ((uint64_t)nsets + 1)), wbase(nsets + 1);
    RSB_CK(cudaMemcpyAsync(&dst, e->status.p, sizeof(dst), cudaMemcpyDeviceToHost, st));
    uint64_t windows[kNumStages];
    RSB_CK(cudaMemcpyAsync(&totals, e->efp.p, sizeof(totals), cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaMemcpyAsync(windows, e->windows.p, sizeof(windows), cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaMemcpyAsync(stage_counts, e->stage_info.p, sizeof(stage_counts), cudaMemcpyDeviceToHost, st));
    if (nsets) {
        RSB_CK(cudaMemcpyAsync(sef.data(), e->set_ef.p, nsets * sizeof(EfParams), cudaMemcpyDeviceToHost, st));
        RSB_CK(cudaMemcpyAsync(bases.data(), e->ef_base.p, bases.size() * 8, cudaMemcpyDeviceToHost, st));
        RSB_CK(cudaMemcpyAsync(wbase.data(), e->word_base.p, wbase.size() * 8, cudaMemcpyDeviceToHost, st));
    }
    RSB_CK(cudaStreamSynchronize(st));
    if (dst.code != 0) report_pipeline_state(e, dst.code, dst.detail, st);
    if (dst.code != 0) return (rsb_status)dst.code;
    // the used part of each output array, then one function per set
    std::vector<uint64_t> hdesc(nsets ? wbase[nsets] : 0), hlower(nsets ? bases[nsets] : 0),
        hcum(nsets ? bases[2 * (nsets + 1) - 1] : 0), hpos(nsets ? bases[3 * (nsets + 1) - 1] : 0),
        hjump(nsets ? bases[4 * (nsets + 1) - 1] : 0);
    if (!hdesc.empty()) RSB_CK(cudaMemcpyAsync(hdesc.data(), desc, hdesc.size() * 8, cudaMemcpyDeviceToHost, st));
    if (!hlower.empty()) RSB_CK(cudaMemcpyAsync(hlower.data(), lower, hlower.size() * 8, cudaMemcpyDeviceToHost, st));
    if (!hcum.empty()) RSB_CK(cudaMemcpyAsync(hcum.data(), ucum, hcum.size() * 8, cudaMemcpyDeviceToHost, st));
    if (!hpos.empty()) RSB_CK(cudaMemcpyAsync(hpos.data(), upos, hpos.size() * 8, cudaMemcpyDeviceToHost, st));
    if (!hjump.empty()) RSB_CK(cudaMemcpyAsync(hjump.data(), jump, hjump.size() * 8, cudaMemcpyDeviceToHost, st));
    RSB_CK(cudaStreamSynchronize(st));
    const uint64_t *hlb = bases.data(), *hcb = hlb + nsets + 1, *hpb = hcb + nsets + 1, *hjb = hpb + nsets + 1;
    for (uint32_t s = 0; s < nsets; ++s) {
        auto *h = new (std::nothrow) rsb_mphf;
        if (!h) {
            for (uint32_t t = 0; t < s; ++t) rsb_free(outs[t]);
            return RSB_ERR_OOM;
        }
        h->leaf = leaf;
        h->rotate = rotate;
        h->bucket_size = bucket_size;
        h->keys_count = h_off[s + 1] - h_off[s];
        h->nbuckets = set_nb[s];
        h->tab = &lt;
        h->ef = sef[s];
        h->desc.assign(hdesc.begin() + wbase[s], hdesc.begin() + wbase[s + 1]);
        h->lower.assign(hlower.begin() + hlb[s], hlower.begin() + hlb[s + 1]);
        h->upper_cum.assign(hcum.begin() + hcb[s], hcum.begin() + hcb[s + 1]);
        h->upper_pos.assign(hpos.begin() + hpb[s], hpos.begin() + hpb[s + 1]);
        h->jump.assign(hjump.begin() + hjb[s], hjump.begin() + hjb[s + 1]);
        h->host_valid = true;
        h->stats.keys = h->keys_count;
        h->stats.buckets = set_nb[s];
        h->stats.descriptor_bits = sef[s].total_bits;
        outs[s] = h;
    }
    if (stats) {
        rsb_stats &S = *stats;
        S = rsb_stats{};
        S.keys = n;
        S.buckets = nb_total;
        S.evals_alg = totals.evals_alg;
        for (int s = 0; s < kNumStages; ++s) {
            S.evals_stage[s] = totals.evals_stage[s];
            S.windows_stage[s] = windows[s];
            S.window_candidates[s] = 32u * (uint32_t)e->last_seeds_per_lane[s];
            S.nodes_per_stage[s] = stage_counts[s];
            S.nodes += stage_counts[s];
        }
        S.kernel_launches = launches_so_far() - launches0;
        for (uint32_t s = 0; s < nsets; ++s) S.descriptor_bits += sef[s].total_bits;
        fill_stage_times(e, lt, S);
    }
    return RSB_OK;
}

rsb_status check_common(rsb_engine *e, uint64_t n, uint64_t bucket_size, uint32_t leaf, rsb_mphf **out) {
    if (!e || !out) return RSB_ERR_BAD_ARG;
    if (leaf < 2 || leaf > (uint32_t)kMaxLeafSize || bucket_size == 0) return RSB_ERR_BAD_ARG;
    if (n >= (1ull << 32) - 1) return RSB_ERR_BAD_ARG;
    if (cudaSetDevice(e->device) != cudaSuccess) {
        cudaGetLastError();
        return RSB_ERR_CUDA;
    }
    return RSB_OK;
}

constexpr uint32_t kKeepSeeds = RSB_KEEP_SEEDS;

}  // namespace

extern "C" {

const char *rsb_version(void) { return "rsb 0.1 (sm_100a)"; }

rsb_status rsb_probe_eval_rate(rsb_engine *e, double *evals_per_second, double *ms) {
    if (!e || !evals_per_second) return RSB_ERR_BAD_ARG;
    RSB_CK(cudaSetDevice(e->device));
    uint64_t evals = 0;
    RSB_CK(cudaEventRecord(e->ev[0], e->stream));
    probe_eval_rate(e->num_sms, &evals, e->stream);
    RSB_CK(cudaGetLastError());
    RSB_CK(cudaEventRecord(e->ev[1], e->stream));
    RSB_CK(cudaEventSynchronize(e->ev[1]));
    const double t = elapsed(e->ev[0], e->ev[1]);
    if (t <= 0) return RSB_ERR_INTERNAL;
    *evals_per_second = (double)evals / (t * 1e-3);
    if (ms) *ms = t;
    return RSB_OK;
}

rsb_status rsb_golomb_memo(uint32_t leaf, uint32_t *out) {
    if (leaf < 2 || leaf > (uint32_t)kMaxLeafSize || !out) return RSB_ERR_BAD_ARG;
    const LeafTables &t = leaf_tables(leaf, true);
    std::memcpy(out, t.memo.data(), kMaxBucketSize * sizeof(uint32_t));
    return RSB_OK;
}

const char *rsb_strerror(rsb_status s) {
    switch (s) {
        case RSB_OK: return "ok";
        case RSB_ERR_BAD_ARG: return "invalid argument";
        case RSB_ERR_CUDA: return cudaGetErrorString(g_last_cuda);
        case RSB_ERR_OOM: return "out of memory";
        case RSB_ERR_DUPLICATE_KEY: return "duplicate key (two keys share a bucket and their second hash half)";
        case RSB_ERR_SEARCH_BUDGET: return "seed search exceeded its candidate budget";
        case RSB_ERR_BUCKET_TOO_LARGE: return "bucket with 3000 or more keys";
        case RSB_ERR_TIMEOUT: return "bounded device wait timed out";
        case RSB_ERR_FORMAT: return "malformed serialized function or leaf size mismatch";
        case RSB_ERR_INTERNAL: return "internal error";
        case RSB_ERR_NO_DEVICE: return "no usable CUDA device";
    }
    return "unknown status";
}

rsb_status rsb_engine_create(int device, void *stream, rsb_engine **out) {
    if (!out) return RSB_ERR_BAD_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) {
        cudaGetLastError();
        return RSB_ERR_NO_DEVICE;
    }
    RSB_CK(cudaSetDevice(device));
    cudaDeviceProp prop{};
    RSB_CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) return RSB_ERR_NO_DEVICE;  // kernels are built for sm_100a only
    auto *e = new (std::nothrow) rsb_engine;
    if (!e) return RSB_ERR_OOM;
    e->device = device;
    e->num_sms = prop.multiProcessorCount;
    if (stream) {
        e->stream = (cudaStream_t)stream;
    } else {
        if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
            delete e;
            return RSB_ERR_CUDA;
        }
        e->own_stream = true;
    }
    for (auto &ev : e->ev) cudaEventCreate(&ev);
    // Keep freed pool memory cached: handles are allocated stream-ordered on every build.
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    cudaGetLastError();
    *out = e;
    return RSB_OK;
}

rsb_status rsb_engine_destroy(rsb_engine *e) {
    if (!e) return RSB_ERR_BAD_ARG;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    release(e->keys128); release(e->raw_u64); release(e->offsets); release(e->sorted); release(e->acc);
    release(e->node_base); release(e->scan_tmp); release(e->pos_acc); release(e->seed); release(e->counts);
    release(e->node_count); release(e->lists); release(e->stage_info); release(e->sched); release(e->slots);
    release(e->bits); release(e->fixed_bits); release(e->nstart); release(e->nwin); release(e->nsize);
    release(e->nstage); release(e->bytes); release(e->status); release(e->efp); release(e->windows);
    release(e->verify_seen);
    release(e->pq); release(e->pcounts); release(e->pactive); release(e->pclaimed); release(e->pblocked);
    release(e->set_key); release(e->set_bucket); release(e->set_bits); release(e->word_base); release(e->ef_base);
    release(e->out_block); release(e->set_nb); release(e->bucket_id); release(e->set_words); release(e->ef_words);
    release(e->set_ef);
    for (auto &kv : e->tables) cudaFree(kv.second.first);
    for (auto &ev : e->ev) cudaEventDestroy(ev);
    if (e->own_stream) cudaStreamDestroy(e->stream);
    delete e;
    return RSB_OK;
}

rsb_status rsb_engine_set_budget(rsb_engine *e, uint32_t shift, uint64_t min_candidates) {
    if (!e || shift > 62) return RSB_ERR_BAD_ARG;
    e->budget_shift = shift;
    e->budget_min = min_candidates;
    return RSB_OK;
}

rsb_status rsb_engine_reserve(rsb_engine *e, uint64_t keys, uint64_t bucket_size, uint64_t string_bytes,
                              uint32_t sets) {
    if (!e || bucket_size == 0 || sets == 0) return RSB_ERR_BAD_ARG;
    RSB_CK(cudaSetDevice(e->device));
    const uint64_t nb = keys / bucket_size + sets;
    if (nb >= (1ull << 32) - 1) return RSB_ERR_BAD_ARG;
    // Output block of the batched encoders: descriptors, EF lower bits, two upper-bit
    // arrays and the jump table, with the per-set slack of build_batch_device.
    const uint64_t block_words = (8 * keys) / 64 + 3 * (uint64_t)sets + 16 + ((nb + sets) * 56 + 63) / 64 +
                                 2 * ((3 * (nb + sets) + 63) / 64) + jump_words_for(nb) + 24 * (uint64_t)sets;
    rsb_status s = ensure_batch_buffers(e, keys, nb, sets, block_words);
    if (s == RSB_OK) s = ensure(e->keys128, 2 * keys);
    if (s == RSB_OK && string_bytes) s = ensure(e->bytes, string_bytes);
    if (s == RSB_OK && string_bytes) s = ensure(e->offsets, keys + 1);
    return s;
}

rsb_status rsb_engine_set_occupancy(rsb_engine *e, uint32_t percent) {
    if (!e || percent == 0 || percent > 100) return RSB_ERR_BAD_ARG;
    e->occupancy_pct = (int)percent;
    return RSB_OK;
}

rsb_status rsb_engine_set_watchdog(rsb_engine *e, double seconds) {
    if (!e || !(seconds >= 0) || seconds > 1e6) return RSB_ERR_BAD_ARG;
    e->watchdog_ns = (uint64_t)(seconds * 1e9);
    return RSB_OK;
}

rsb_status rsb_engine_set_pipeline(rsb_engine *e, uint32_t on) {
    if (!e || on > 1) return RSB_ERR_BAD_ARG;
    e->pipeline = on != 0;
    return RSB_OK;
}

rsb_status rsb_engine_set_schedule(rsb_engine *e, uint32_t leaf, uint32_t stage, uint32_t size_class,
                                   uint32_t seeds_per_lane, uint32_t occupancy_pct) {
    if (!e || leaf < 2 || leaf > (uint32_t)kMaxLeafSize || size_class >= (uint32_t)kScheduleSizeClasses ||
        (stage != (uint32_t)kStageUpper && stage != (uint32_t)kStageLower && stage != (uint32_t)kStageLeafRot))
        return RSB_ERR_BAD_ARG;
    const uint32_t key = schedule_key(leaf, (int)stage, (int)size_class);
    if (seeds_per_lane == 0) {
        e->schedules.erase(key);
        return RSB_OK;
    }
    const StageSchedule s{(int)seeds_per_lane, (int)occupancy_pct};
    if (!schedule_valid((int)stage, s)) return RSB_ERR_BAD_ARG;
    e->schedules[key] = s;
    return RSB_OK;
}

rsb_status rsb_engine_get_schedule(rsb_engine *e, uint32_t leaf, uint32_t stage, uint32_t size_class,
                                   uint32_t *seeds_per_lane, uint32_t *occupancy_pct) {
    if (!e || !seeds_per_lane || !occupancy_pct || leaf < 2 || leaf > (uint32_t)kMaxLeafSize ||
        size_class >= (uint32_t)kScheduleSizeClasses ||
        (stage != (uint32_t)kStageUpper && stage != (uint32_t)kStageLower && stage != (uint32_t)kStageLeafRot))
        return RSB_ERR_BAD_ARG;
    auto it = e->schedules.find(schedule_key(leaf, (int)stage, (int)size_class));
    const StageSchedule s = it != e->schedules.end() ? it->second : default_schedule((int)leaf, (int)stage, (int)size_class);
    *seeds_per_lane = (uint32_t)s.seeds_per_lane;
    *occupancy_pct = (uint32_t)s.occupancy_pct;
    return RSB_OK;
}

static rsb_status stage_keys128(rsb_engine *e, const rsb_hash128 *keys, uint64_t n, uint32_t flags, const uint64_t **dk) {
    if (flags & RSB_KEYS_ON_DEVICE) {
        *dk = (const uint64_t *)keys;
        return RSB_OK;
    }
    rsb_status s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    if (n) RSB_CK(cudaMemcpyAsync(e->keys128.p, keys, n * 16, cudaMemcpyHostToDevice, e->stream));
    *dk = e->keys128.p;
    return RSB_OK;
}

rsb_status rsb_build_hash128(rsb_engine *e, const rsb_hash128 *keys, uint64_t n, uint64_t bucket_size, uint32_t leaf,
                             uint32_t flags, rsb_mphf **out) {
    rsb_status s = check_common(e, n, bucket_size, leaf, out);
    if (s != RSB_OK) return s;
    if (n && !keys) return RSB_ERR_BAD_ARG;
    const uint64_t *dk = nullptr;
    s = stage_keys128(e, keys, n, flags, &dk);
    if (s != RSB_OK) return s;
    return build_device(e, dk, n, bucket_size, leaf, flags, out, (flags & kKeepSeeds) != 0);
}

rsb_status rsb_build_u64(rsb_engine *e, const uint64_t *keys, uint64_t n, uint64_t bucket_size, uint32_t leaf,
                         uint32_t flags, rsb_mphf **out) {
    rsb_status s = check_common(e, n, bucket_size, leaf, out);
    if (s != RSB_OK) return s;
    if (n && !keys) return RSB_ERR_BAD_ARG;
    const uint64_t *dk = keys;
    if (!(flags & RSB_KEYS_ON_DEVICE)) {
        s = ensure(e->raw_u64, n);
        if (s != RSB_OK) return s;
        if (n) RSB_CK(cudaMemcpyAsync(e->raw_u64.p, keys, n * 8, cudaMemcpyHostToDevice, e->stream));
        dk = e->raw_u64.p;
    }
    s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    uint64_t *k128 = e->keys128.p;
    cudaStream_t st = e->stream;
    return build_device(e, k128, n, bucket_size, leaf, flags, out, (flags & kKeepSeeds) != 0,
                        [=] { launch_hash_u64(dk, n, k128, st); });
}

// Host string keys: only the referenced bytes [offsets[0], offsets[n]) go to the device, and
// the hash kernel subtracts offsets[0] (*base) from every offset.
static rsb_status stage_strings(rsb_engine *e, const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint32_t flags,
                                const uint8_t **db, const uint64_t **doff, uint64_t *base) {
    if (flags & RSB_KEYS_ON_DEVICE) {
        *db = bytes;
        *doff = offsets;
        *base = 0;
        return RSB_OK;
    }
    if (offsets[n] < offsets[0]) return RSB_ERR_BAD_ARG;
    const uint64_t nbytes = offsets[n] - offsets[0];
    rsb_status s = ensure(e->bytes, nbytes);
    if (s != RSB_OK) return s;
    s = ensure(e->offsets, n + 1);
    if (s != RSB_OK) return s;
    if (nbytes) RSB_CK(cudaMemcpyAsync(e->bytes.p, bytes + offsets[0], nbytes, cudaMemcpyHostToDevice, e->stream));
    RSB_CK(cudaMemcpyAsync(e->offsets.p, offsets, (n + 1) * 8, cudaMemcpyHostToDevice, e->stream));
    *db = e->bytes.p;
    *doff = e->offsets.p;
    *base = offsets[0];
    return RSB_OK;
}

rsb_status rsb_build_strings(rsb_engine *e, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                             uint64_t bucket_size, uint32_t leaf, uint32_t flags, rsb_mphf **out) {
    rsb_status s = check_common(e, n, bucket_size, leaf, out);
    if (s != RSB_OK) return s;
    if (!offsets) return RSB_ERR_BAD_ARG;
    const uint8_t *db;
    const uint64_t *doff;
    uint64_t sbase = 0;
    s = stage_strings(e, bytes, offsets, n, flags, &db, &doff, &sbase);
    if (s != RSB_OK) return s;
    s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    uint64_t *k128 = e->keys128.p;
    cudaStream_t st = e->stream;
    return build_device(e, k128, n, bucket_size, leaf, flags, out, (flags & kKeepSeeds) != 0,
                        [=] { launch_hash_strings(db, doff, n, sbase, k128, st); });
}

static rsb_status check_batch(rsb_engine *e, const uint64_t *set_offsets, uint32_t nsets, uint64_t bucket_size,
                              uint32_t leaf, rsb_mphf **outs) {
    if (!e || !set_offsets || (nsets && !outs)) return RSB_ERR_BAD_ARG;
    if (leaf < 2 || leaf > (uint32_t)kMaxLeafSize || bucket_size == 0) return RSB_ERR_BAD_ARG;
    if (set_offsets[0] != 0) return RSB_ERR_BAD_ARG;
    for (uint32_t s = 0; s < nsets; ++s)
        if (set_offsets[s + 1] < set_offsets[s]) return RSB_ERR_BAD_ARG;
    if (set_offsets[nsets] >= (1ull << 32) - 1) return RSB_ERR_BAD_ARG;
    if (cudaSetDevice(e->device) != cudaSuccess) {
        cudaGetLastError();
        return RSB_ERR_CUDA;
    }
    return RSB_OK;
}

rsb_status rsb_build_batch_hash128(rsb_engine *e, const rsb_hash128 *keys, const uint64_t *set_offsets, uint32_t nsets,
                                   uint64_t bucket_size, uint32_t leaf, uint32_t flags, rsb_mphf **outs,
                                   rsb_stats *stats) {
    rsb_status s = check_batch(e, set_offsets, nsets, bucket_size, leaf, outs);
    if (s != RSB_OK) return s;
    const uint64_t n = set_offsets[nsets];
    if (n && !keys) return RSB_ERR_BAD_ARG;
    const uint64_t *dk = nullptr;
    s = stage_keys128(e, keys, n, flags, &dk);
    if (s != RSB_OK) return s;
    return build_batch_device(e, dk, set_offsets, nsets, bucket_size, leaf, flags, outs, stats, std::function<void()>());
}

rsb_status rsb_build_batch_u64(rsb_engine *e, const uint64_t *keys, const uint64_t *set_offsets, uint32_t nsets,
                               uint64_t bucket_size, uint32_t leaf, uint32_t flags, rsb_mphf **outs, rsb_stats *stats) {
    rsb_status s = check_batch(e, set_offsets, nsets, bucket_size, leaf, outs);
    if (s != RSB_OK) return s;
    const uint64_t n = set_offsets[nsets];
    if (n && !keys) return RSB_ERR_BAD_ARG;
    const uint64_t *dk = keys;
    if (!(flags & RSB_KEYS_ON_DEVICE)) {
        s = ensure(e->raw_u64, n);
        if (s != RSB_OK) return s;
        if (n) RSB_CK(cudaMemcpyAsync(e->raw_u64.p, keys, n * 8, cudaMemcpyHostToDevice, e->stream));
        dk = e->raw_u64.p;
    }
    s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    uint64_t *k128 = e->keys128.p;
    cudaStream_t st = e->stream;
    return build_batch_device(e, k128, set_offsets, nsets, bucket_size, leaf, flags, outs, stats,
                              [=] { launch_hash_u64(dk, n, k128, st); });
}

rsb_status rsb_build_batch_strings(rsb_engine *e, const uint8_t *bytes, const uint64_t *offsets,
                                   const uint64_t *set_offsets, uint32_t nsets, uint64_t bucket_size, uint32_t leaf,
                                   uint32_t flags, rsb_mphf **outs, rsb_stats *stats) {
    rsb_status s = check_batch(e, set_offsets, nsets, bucket_size, leaf, outs);
    if (s != RSB_OK) return s;
    if (!offsets) return RSB_ERR_BAD_ARG;
    const uint64_t n = set_offsets[nsets];
    const uint8_t *db;
    const uint64_t *doff;
    uint64_t sbase = 0;
    s = stage_strings(e, bytes, offsets, n, flags, &db, &doff, &sbase);
    if (s != RSB_OK) return s;
    s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    uint64_t *k128 = e->keys128.p;
    cudaStream_t st = e->stream;
    return build_batch_device(e, k128, set_offsets, nsets, bucket_size, leaf, flags, outs, stats,
                              [=] { launch_hash_strings(db, doff, n, sbase, k128, st); });
}

// ---- sharded construction: parts over bucket ranges, merged into one function ----------
//
// The reference's compute_thread splits the buckets into contiguous ranges, builds each
// range's Rice stream separately and appends the streams in bucket order
// (SIMDRecSplit.hpp:695-745); bucket ranges on several GPUs work the same way. A part is
// built like a plain function whose buckets are the range's (k_part_first re-maps the first
// halves; the second halves, which decide every seed, are unchanged); its export carries the
// per-bucket key and bit offsets and its Rice bits; the merge concatenates the bits in bucket
// order, appends the sentinel and builds the double Elias-Fano index over all buckets.

static constexpr uint64_t kPartMagic = 0x3154524150425352ull;  // "RSBPART1"
static rsb_status ensure_host(rsb_mphf *h);

rsb_status rsb_build_part_hash128(rsb_engine *e, const rsb_hash128 *keys, uint64_t n, uint64_t nbuckets_total,
                                  uint64_t bucket_lo, uint64_t bucket_hi, uint64_t bucket_size, uint32_t leaf,
                                  uint32_t flags, rsb_mphf **out) {
    rsb_status s = check_common(e, n, bucket_size, leaf, out);
    if (s != RSB_OK) return s;
    if ((n && !keys) || nbuckets_total == 0 || bucket_lo >= bucket_hi || bucket_hi > nbuckets_total ||
        bucket_hi - bucket_lo >= (1ull << 32))
        return RSB_ERR_BAD_ARG;
    const uint64_t nbp = bucket_hi - bucket_lo;
    s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    s = ensure(e->status, 1);
    if (s != RSB_OK) return s;
    cudaStream_t st = e->stream;
    if (n) {
        RSB_CK(cudaMemcpyAsync(e->keys128.p, keys, n * 16,
                               (flags & RSB_KEYS_ON_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
        RSB_CK(cudaMemsetAsync(e->status.p, 0, sizeof(DevStatus), st));
        launch_part_first(e->keys128.p, n, nbuckets_total, bucket_lo, nbp, e->status.p, st);
        RSB_CK(cudaGetLastError());
        DevStatus dst{};
        RSB_CK(cudaMemcpyAsync(&dst, e->status.p, sizeof(dst), cudaMemcpyDeviceToHost, st));
        RSB_CK(cudaStreamSynchronize(st));
        if (dst.code != 0) return (rsb_status)dst.code;  // a key outside the bucket range
    }
    rsb_mphf *h = nullptr;
    s = build_device(e, e->keys128.p, n, bucket_size, leaf, flags & ~(uint32_t)RSB_DEVICE_ONLY, &h,
                     (flags & kKeepSeeds) != 0, std::function<void()>(), nbp, true);
    if (s != RSB_OK) return s;
    h->part_lo = bucket_lo;
    h->part_hi = bucket_hi;
    h->part_nb_total = nbuckets_total;
    *out = h;
    return RSB_OK;
}

rsb_status rsb_part_export(rsb_mphf *h, uint8_t *buf, size_t *len) {
    if (!h || !len || h->part_hi == 0 || h->bucket_acc.size() != h->nbuckets + 1) return RSB_ERR_BAD_ARG;
    rsb_status s = ensure_host(h);
    if (s != RSB_OK) return s;
    const uint64_t nb = h->nbuckets, bits = h->bucket_pos[nb], words = (bits + 63) / 64;
    const size_t need = 8 * (9 + 2 * (nb + 1) + words);
    if (!buf) {
        *len = need;
        return RSB_OK;
    }
    if (*len < need || words > h->desc.size()) return RSB_ERR_BAD_ARG;
    uint64_t *o = (uint64_t *)buf;  // caller's buffer: written with memcpy, no alignment needed
    const uint64_t head[9] = {kPartMagic, h->leaf, h->rotate ? 1u : 0u, h->part_nb_total, h->part_lo, h->part_hi,
                              h->keys_count, bits, h->bucket_size};
    std::memcpy(o, head, sizeof(head));
    std::memcpy(buf + 8 * 9, h->bucket_acc.data(), 8 * (nb + 1));
    std::memcpy(buf + 8 * (9 + nb + 1), h->bucket_pos.data(), 8 * (nb + 1));
    std::vector<uint64_t> d(h->desc.begin(), h->desc.begin() + words);
    if (bits % 64) d[words - 1] &= (1ull << (bits % 64)) - 1;  // the part's sentinel is not part of it
    std::memcpy(buf + 8 * (9 + 2 * (nb + 1)), d.data(), 8 * words);
    *len = need;
    return RSB_OK;
}

rsb_status rsb_merge_parts(rsb_engine *e, const uint8_t *const *parts, const size_t *lens, uint32_t nparts,
                           uint32_t leaf_size, uint32_t flags, rsb_mphf **out) {
    if (!e || !parts || !lens || !out || nparts == 0) return RSB_ERR_BAD_ARG;
    struct Part {
        uint64_t leaf, rotate, nb_total, lo, hi, keys, bits, bucket_size;
        const uint8_t *acc, *pos, *desc;
    };
    std::vector<Part> ps(nparts);
    for (uint32_t i = 0; i < nparts; ++i) {
        if (!parts[i] || lens[i] < 8 * 9) return RSB_ERR_FORMAT;
        uint64_t head[9];
        std::memcpy(head, parts[i], sizeof(head));
        Part &p = ps[i];
        p = Part{head[1], head[2], head[3], head[4], head[5], head[6], head[7], head[8], nullptr, nullptr, nullptr};
        if (head[0] != kPartMagic || p.lo >= p.hi || p.hi > p.nb_total || p.bits > 8 * (uint64_t)lens[i])
            return RSB_ERR_FORMAT;
        const uint64_t nb = p.hi - p.lo, words = (p.bits + 63) / 64;
        if (nb > lens[i] / 16 || lens[i] != 8 * (9 + 2 * (nb + 1) + words)) return RSB_ERR_FORMAT;
        p.acc = parts[i] + 8 * 9;
        p.pos = p.acc + 8 * (nb + 1);
        p.desc = p.pos + 8 * (nb + 1);
        // offsets start at 0, never decrease and end at the part's key and bit counts
        uint64_t a0 = 0, b0 = 0;
        for (uint64_t j = 0; j <= nb; ++j) {
            uint64_t a, b;
            std::memcpy(&a, p.acc + 8 * j, 8);
            std::memcpy(&b, p.pos + 8 * j, 8);
            if ((j == 0 && (a | b)) || a < a0 || b < b0) return RSB_ERR_FORMAT;
            a0 = a;
            b0 = b;
        }
        if (a0 != p.keys || b0 != p.bits) return RSB_ERR_FORMAT;
    }
    // the parts must tile the buckets of one function in order
    const Part &p0 = ps[0];
    uint64_t n = 0, total_bits = 0;
    for (uint32_t i = 0; i < nparts; ++i) {
        const Part &p = ps[i];
        if (p.leaf != p0.leaf || p.rotate != p0.rotate || p.nb_total != p0.nb_total || p.bucket_size != p0.bucket_size ||
            p.lo != (i ? ps[i - 1].hi : 0))
            return RSB_ERR_BAD_ARG;
        n += p.keys;
        total_bits += p.bits;
    }
    const uint64_t nb = p0.nb_total;
    if (ps[nparts - 1].hi != nb || nb != std::max<uint64_t>(1, (n + p0.bucket_size - 1) / p0.bucket_size))
        return RSB_ERR_BAD_ARG;
    const uint32_t leaf = (uint32_t)p0.leaf;
    const bool rotate = p0.rotate != 0;
    if (leaf < 2 || leaf > (uint32_t)kMaxLeafSize || leaf != leaf_size || (((flags & RSB_ROTATE) != 0) != rotate))
        return RSB_ERR_BAD_ARG;
    RSB_CK(cudaSetDevice(e->device));

    // global bucket offsets and the concatenated Rice stream, then the sentinel appendFixed(1, 1)
    std::vector<uint64_t> acc(nb + 1), pos(nb + 1);
    const uint64_t desc_words = (((total_bits + 1 + 7) / 8) + 7 + 7) / 8;  // RiceBitVector.hpp:77
    std::vector<uint64_t> desc(desc_words + 1, 0);
    uint64_t kbase = 0, bbase = 0;
    for (const Part &p : ps) {
        const uint64_t pnb = p.hi - p.lo;
        for (uint64_t j = 0; j < pnb; ++j) {
            uint64_t a, b;
            std::memcpy(&a, p.acc + 8 * j, 8);
            std::memcpy(&b, p.pos + 8 * j, 8);
            acc[p.lo + j] = kbase + a;
            pos[p.lo + j] = bbase + b;
        }
        const uint64_t words = (p.bits + 63) / 64, sh = bbase % 64, w0 = bbase / 64;
        for (uint64_t k = 0; k < words; ++k) {
            uint64_t v;
            std::memcpy(&v, p.desc + 8 * k, 8);
            desc[w0 + k] |= v << sh;
            if (sh && w0 + k + 1 < desc.size()) desc[w0 + k + 1] |= v >> (64 - sh);
        }
        kbase += p.keys;
        bbase += p.bits;
    }
    acc[nb] = kbase;
    pos[nb] = bbase;
    desc[total_bits / 64] |= 1ull << (total_bits % 64);
    desc.resize(desc_words);

    const LeafTables &lt = leaf_tables(leaf, rotate);
    cudaStream_t st = e->stream;
    rsb_status s = ensure(e->acc, nb + 1);
    if (s == RSB_OK) s = ensure(e->pos_acc, nb + 1);
    if (s == RSB_OK) s = ensure(e->status, 1);
    if (s == RSB_OK) s = ensure(e->efp, 1);
    if (s != RSB_OK) return s;
    auto *h = new (std::nothrow) rsb_mphf;
    if (!h) return RSB_ERR_OOM;
    h->leaf = leaf;
    h->rotate = rotate;
    h->bucket_size = p0.bucket_size;
    h->keys_count = n;
    h->nbuckets = nb;
    h->tab = &lt;
    h->device = e->device;
    h->desc_cap = desc_words;
    h->lower_cap = ((nb + 1) * 56 + 63) / 64 + 2;
    h->cum_cap = (3 * (nb + 1) + 63) / 64 + 2;
    h->pos_cap = h->cum_cap;
    h->jump_cap = jump_words_for(nb) + 2;
    const uint64_t block_words = h->desc_cap + h->lower_cap + h->cum_cap + h->pos_cap + h->jump_cap;
    auto fail = [&](rsb_status r) {
        if (h->d_block) cudaFree(h->d_block);
        delete h;
        return r;
    };
    if (cudaMalloc((void **)&h->d_block, block_words * 8) != cudaSuccess) {
        cudaGetLastError();
        return fail(RSB_ERR_OOM);
    }
#define RSB_CKM(call)                  \
    do {                               \
        cudaError_t e_ = (call);       \
        if (e_ != cudaSuccess) {       \
            g_last_cuda = e_;          \
            cudaStreamSynchronize(st); \
            return fail(RSB_ERR_CUDA); \
        }                              \
    } while (0)
    RSB_CKM(cudaMemsetAsync(h->d_block, 0, block_words * 8, st));
    RSB_CKM(cudaMemcpyAsync(h->d_desc(), desc.data(), desc_words * 8, cudaMemcpyHostToDevice, st));
    RSB_CKM(cudaMemcpyAsync(e->acc.p, acc.data(), (nb + 1) * 8, cudaMemcpyHostToDevice, st));
    RSB_CKM(cudaMemcpyAsync(e->pos_acc.p, pos.data(), (nb + 1) * 8, cudaMemcpyHostToDevice, st));
    RSB_CKM(cudaMemsetAsync(e->status.p, 0, sizeof(DevStatus), st));
    RSB_CKM(cudaMemsetAsync(e->efp.p, 0, sizeof(EfParams), st));
    launch_ef_build(e->acc.p, e->pos_acc.p, nb, n, e->efp.p, h->d_lower(), h->lower_cap, h->d_cum(), h->cum_cap,
                    h->d_pos(), h->pos_cap, h->d_jump(), h->jump_cap, e->status.p, st);
    RSB_CKM(cudaGetLastError());
    DevStatus dst{};
    RSB_CKM(cudaMemcpyAsync(&dst, e->status.p, sizeof(dst), cudaMemcpyDeviceToHost, st));
    RSB_CKM(cudaMemcpyAsync(&h->ef, e->efp.p, sizeof(EfParams), cudaMemcpyDeviceToHost, st));
    RSB_CKM(cudaStreamSynchronize(st));
#undef RSB_CKM
    if (dst.code != 0) return fail((rsb_status)dst.code);
    h->ef.total_bits = total_bits;
    h->ef.desc_words = desc_words;
    h->stats.keys = n;
    h->stats.buckets = nb;
    h->stats.descriptor_bits = total_bits;
    s = copy_to_host(h, st);
    if (s != RSB_OK) return fail(s);
    *out = h;
    return RSB_OK;
}

rsb_status rsb_hash_strings(rsb_engine *e, const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint32_t flags,
                            rsb_hash128 *out) {
    if (!e || !offsets || !out) return RSB_ERR_BAD_ARG;
    RSB_CK(cudaSetDevice(e->device));
    const uint8_t *db;
    const uint64_t *doff;
    uint64_t sbase = 0;
    rsb_status s = stage_strings(e, bytes, offsets, n, flags, &db, &doff, &sbase);
    if (s != RSB_OK) return s;
    s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    launch_hash_strings(db, doff, n, sbase, e->keys128.p, e->stream);
    RSB_CK(cudaGetLastError());
    RSB_CK(cudaStreamSynchronize(e->stream));  // before a pageable copy (see the build paths)
    RSB_CK(cudaMemcpyAsync(out, e->keys128.p, n * 16, (flags & RSB_KEYS_ON_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                           e->stream));
    RSB_CK(cudaStreamSynchronize(e->stream));
    return RSB_OK;
}

rsb_status rsb_hash_u64(rsb_engine *e, const uint64_t *keys, uint64_t n, uint32_t flags, rsb_hash128 *out) {
    if (!e || (n && (!keys || !out))) return RSB_ERR_BAD_ARG;
    RSB_CK(cudaSetDevice(e->device));
    const uint64_t *dk = keys;
    if (!(flags & RSB_KEYS_ON_DEVICE)) {
        rsb_status s = ensure(e->raw_u64, n);
        if (s != RSB_OK) return s;
        if (n) RSB_CK(cudaMemcpyAsync(e->raw_u64.p, keys, n * 8, cudaMemcpyHostToDevice, e->stream));
        dk = e->raw_u64.p;
    }
    rsb_status s = ensure(e->keys128, 2 * n);
    if (s != RSB_OK) return s;
    launch_hash_u64(dk, n, e->keys128.p, e->stream);
    RSB_CK(cudaGetLastError());
    if (n)
        RSB_CK(cudaStreamSynchronize(e->stream));  // before a pageable copy (see the build paths)
    RSB_CK(cudaMemcpyAsync(out, e->keys128.p, n * 16, (flags & RSB_KEYS_ON_DEVICE) ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                               e->stream));
    RSB_CK(cudaStreamSynchronize(e->stream));
    return RSB_OK;
}

static rsb_status ensure_host(rsb_mphf *h) {
    if (h->host_valid) return RSB_OK;
    cudaStream_t st = nullptr;
    if (h->device >= 0) cudaSetDevice(h->device);
    return copy_to_host(h, st);
}

rsb_status rsb_query_hash128(rsb_mphf *h, const rsb_hash128 *keys, uint64_t n, uint64_t *out) {
    if (!h || (n && (!keys || !out))) return RSB_ERR_BAD_ARG;
    rsb_status s = ensure_host(h);
    if (s != RSB_OK) return s;
    const MphfView v = h->host_view();
    for (uint64_t i = 0; i < n; ++i) out[i] = mphf_query(v, keys[i].first, keys[i].second);
    return RSB_OK;
}

rsb_status rsb_query_strings(rsb_mphf *h, const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out) {
    if (!h || !offsets || (n && !out)) return RSB_ERR_BAD_ARG;
    rsb_status s = ensure_host(h);
    if (s != RSB_OK) return s;
    const MphfView v = h->host_view();
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t h0 = 0, h1 = 0;
        spooky128(bytes + offsets[i], offsets[i + 1] - offsets[i], h0, h1);
        out[i] = mphf_query(v, h1, h0);
    }
    return RSB_OK;
}

rsb_status rsb_query_device(rsb_engine *e, rsb_mphf *h, const rsb_hash128 *keys, uint64_t n, uint64_t *out) {
    if (!e || !h || (n && (!keys || !out))) return RSB_ERR_BAD_ARG;
    RSB_CK(cudaSetDevice(e->device));
    if (!h->d_block || h->device != e->device) {
        // upload a host-side (e.g. deserialized) function
        rsb_status s = ensure_host(h);
        if (s != RSB_OK) return s;
        if (h->d_block) cudaFree(h->d_block);
        h->desc_cap = h->desc.size();
        h->lower_cap = h->lower.size();
        h->cum_cap = h->upper_cum.size();
        h->pos_cap = h->upper_pos.size();
        h->jump_cap = h->jump.size();
        const uint64_t words = h->desc_cap + h->lower_cap + h->cum_cap + h->pos_cap + h->jump_cap + 1;
        RSB_CK(cudaMalloc((void **)&h->d_block, words * 8));
        RSB_CK(cudaMemcpy(h->d_desc(), h->desc.data(), h->desc.size() * 8, cudaMemcpyHostToDevice));
        RSB_CK(cudaMemcpy(h->d_lower(), h->lower.data(), h->lower.size() * 8, cudaMemcpyHostToDevice));
        RSB_CK(cudaMemcpy(h->d_cum(), h->upper_cum.data(), h->upper_cum.size() * 8, cudaMemcpyHostToDevice));
        RSB_CK(cudaMemcpy(h->d_pos(), h->upper_pos.data(), h->upper_pos.size() * 8, cudaMemcpyHostToDevice));
        RSB_CK(cudaMemcpy(h->d_jump(), h->jump.data(), h->jump.size() * 8, cudaMemcpyHostToDevice));
        h->device = e->device;
    }
    DevTables tab;
    rsb_status s = get_device_tables(e, *h->tab, h->leaf, h->rotate, tab);
    if (s != RSB_OK) return s;
    const MphfView v = device_view(h, tab);
    launch_query_view(v, (const uint64_t *)keys, n, out, e->stream);
    RSB_CK(cudaGetLastError());
    RSB_CK(cudaStreamSynchronize(e->stream));
    return RSB_OK;
}

// bitCountCumKeys + bitCountPosition (DoubleEF.hpp:435-437) + descriptors.getBits()
// (RiceBitVector.hpp:152); the C++ wrapper adds 8 * sizeof(*this) like getBits() does.
rsb_status rsb_get_bits(rsb_mphf *h, uint64_t *bits) {
    if (!h || !bits) return RSB_ERR_BAD_ARG;
    const EfParams &f = h->ef;
    const uint64_t nb = f.num_buckets;
    const uint64_t jh = f.jump_words / 2;
    const uint64_t cum = (nb + 1) * f.l_cum_keys + nb + 1 + (f.u_cum_keys >> f.l_cum_keys) + jh;
    const uint64_t pos = (nb + 1) * f.l_position + nb + 1 + (f.u_position >> f.l_position) + jh;
    *bits = cum + pos + f.desc_words * 64;
    return RSB_OK;
}

static void put64(std::vector<uint8_t> &o, uint64_t v) {
    uint8_t b[8];
    std::memcpy(b, &v, 8);
    o.insert(o.end(), b, b + 8);
}
static void put_vec(std::vector<uint8_t> &o, const std::vector<uint64_t> &v) {
    put64(o, v.size());
    const uint8_t *p = (const uint8_t *)v.data();
    o.insert(o.end(), p, p + v.size() * 8);
}

// Layout of operator<< (GPURecSplit.cuh:817-825, DoubleEF.hpp:100-113); a word vector is
// written as a uint64 element count followed by its words.
rsb_status rsb_serialize(rsb_mphf *h, uint8_t *buf, size_t *len) {
    if (!h || !len) return RSB_ERR_BAD_ARG;
    rsb_status s = ensure_host(h);
    if (s != RSB_OK) return s;
    const size_t need = 8 * (3 + 1 + h->desc.size() + 6 + 4 + h->lower.size() + h->upper_cum.size() + h->upper_pos.size() +
                             h->jump.size());
    if (!buf) {
        *len = need;
        return RSB_OK;
    }
    if (*len < need) {
        *len = need;
        return RSB_ERR_BAD_ARG;
    }
    std::vector<uint8_t> o;
    o.reserve(need);
    put64(o, h->leaf);
    put64(o, h->bucket_size);
    put64(o, h->keys_count);
    put_vec(o, h->desc);
    put64(o, h->ef.num_buckets);
    put64(o, h->ef.u_cum_keys);
    put64(o, h->ef.u_position);
    put64(o, (uint64_t)h->ef.cum_keys_min_delta);
    put64(o, (uint64_t)h->ef.min_diff);
    put64(o, h->ef.bits_per_key_fixed_point);
    put_vec(o, h->lower);
    put_vec(o, h->upper_cum);
    put_vec(o, h->upper_pos);
    put_vec(o, h->jump);
    std::memcpy(buf, o.data(), o.size());
    *len = o.size();
    return RSB_OK;
}

rsb_status rsb_deserialize(const uint8_t *buf, size_t len, uint32_t leaf, uint32_t flags, rsb_mphf **out) {
    if (!buf || !out) return RSB_ERR_BAD_ARG;
    size_t off = 0;
    bool ok = true;
    auto get64 = [&]() -> uint64_t {
        if (len - off < 8 || off > len) {
            ok = false;
            return 0;
        }
        uint64_t v;
        std::memcpy(&v, buf + off, 8);
        off += 8;
        return v;
    };
    auto get_vec = [&](std::vector<uint64_t> &v) {
        const uint64_t n = get64();
        if (!ok || (len - off) / 8 < n) {
            ok = false;
            return;
        }
        v.resize(n);
        std::memcpy(v.data(), buf + off, n * 8);
        off += n * 8;
    };
    const uint64_t l = get64();
    if (!ok || l != leaf || leaf < 2 || leaf > (uint32_t)kMaxLeafSize) return RSB_ERR_FORMAT;
    auto *h = new (std::nothrow) rsb_mphf;
    if (!h) return RSB_ERR_OOM;
    h->leaf = leaf;
    h->rotate = (flags & RSB_ROTATE) != 0;
    h->bucket_size = get64();
    h->keys_count = get64();
    if (!ok || h->bucket_size == 0) {
        delete h;
        return RSB_ERR_FORMAT;
    }
    h->nbuckets = std::max<uint64_t>(1, (h->keys_count + h->bucket_size - 1) / h->bucket_size);  // :499
    get_vec(h->desc);
    EfParams &f = h->ef;
    f.num_buckets = get64();
    f.u_cum_keys = get64();
    f.u_position = get64();
    f.cum_keys_min_delta = (int64_t)get64();
    f.min_diff = (int64_t)get64();
    f.bits_per_key_fixed_point = get64();
    get_vec(h->lower);
    get_vec(h->upper_cum);
    get_vec(h->upper_pos);
    get_vec(h->jump);
    if (!ok) {
        delete h;
        return RSB_ERR_FORMAT;
    }
    const uint64_t nb = f.num_buckets;
    f.l_position = f.u_position / (nb + 1) == 0 ? 0 : 63 - __builtin_clzll(f.u_position / (nb + 1));  // DoubleEF.hpp:123
    f.l_cum_keys = f.u_cum_keys / (nb + 1) == 0 ? 0 : 63 - __builtin_clzll(f.u_cum_keys / (nb + 1));
    f.desc_words = h->desc.size();
    f.lower_words = h->lower.size();
    f.cum_words = h->upper_cum.size();
    f.pos_words = h->upper_pos.size();
    f.jump_words = h->jump.size();
    h->tab = &leaf_tables(leaf, h->rotate);
    h->host_valid = true;
    *out = h;
    return RSB_OK;
}

rsb_status rsb_seeds(rsb_mphf *h, uint64_t *seeds, uint32_t *sizes, size_t *count) {
    if (!h || !count) return RSB_ERR_BAD_ARG;
    if (!seeds) {
        *count = h->seeds.size();
        return RSB_OK;
    }
    const size_t n = std::min(*count, h->seeds.size());
    std::memcpy(seeds, h->seeds.data(), n * 8);
    if (sizes) std::memcpy(sizes, h->sizes.data(), n * 4);
    *count = n;
    return RSB_OK;
}

rsb_status rsb_get_stats(rsb_mphf *h, rsb_stats *s) {
    if (!h || !s) return RSB_ERR_BAD_ARG;
    *s = h->stats;
    return RSB_OK;
}

rsb_status rsb_free(rsb_mphf *h) {
    if (!h) return RSB_ERR_BAD_ARG;
    if (h->d_block) {
        cudaSetDevice(h->device);
        cudaFree(h->d_block);
    }
    delete h;
    return RSB_OK;
}

}  // extern "C"
