// Launchers of the engine's kernels (implemented in rsb_prep.cu, rsb_search.cu, rsb_encode.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rsb_common.cuh"

namespace rsb {

// Every kernel of the engine asks for the largest shared-memory carveout of the SM (once per
// kernel and device). An SM keeps one L1/shared split while CTAs are resident, so kernels of
// two engines can only share SMs (a build service runs a small request beside a large one)
// if neither kernel has the SMs configured with less shared memory than the other needs.
// The kernels keep their working sets in shared memory and registers; L1 matters little.
void prefer_shared_memory(const void *func);
// Streaming multiprocessors of the current device (queried once per device); grid caps of
// the non-persistent kernels are multiples of it.
int device_sm_count();
template <typename K>
inline void use_max_smem(K kernel) {
    prefer_shared_memory((const void *)kernel);
}


// Device-side per-leaf constants (uploaded once per engine and leaf size).
struct DevTables {
    const uint32_t *memo;   // kMaxBucketSize
    const uint32_t *nodes;  // kMaxBucketSize
};

// Scratch of a plain exclusive scan.
struct ScanTmp {
    uint64_t *block_sums;
    size_t blocks_cap;
};

size_t scan_blocks(size_t n);
// out[i] = sum_{j<i} in[i] for i <= n (out has n+1 entries); in is u32.
void exclusive_scan_u32(const uint32_t *in, uint64_t *out, size_t n, ScanTmp tmp, cudaStream_t st);

// ---- preparation (rsb_prep.cu) ----
void launch_hash_u64(const uint64_t *keys, uint64_t n, uint64_t *out128, cudaStream_t st);
void launch_part_first(uint64_t *keys128, uint64_t n, uint64_t nb_total, uint64_t lo, uint64_t nbp, DevStatus *status,
                       cudaStream_t st);
// Key i occupies bytes[offsets[i] - base, offsets[i + 1] - base).
void launch_hash_strings(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t base, uint64_t *out128,
                         cudaStream_t st);
void launch_bucket_count(const uint64_t *keys128, uint64_t n, uint64_t nbuckets, uint32_t *counts, cudaStream_t st);
void launch_bucket_check(const uint32_t *counts, uint64_t nbuckets, DevStatus *status, cudaStream_t st);
void launch_bucket_scatter(const uint64_t *keys128, uint64_t n, uint64_t nbuckets, const uint64_t *acc,
                           uint32_t *cursor, uint64_t *sorted, cudaStream_t st);
// Fails the build with RSB_ERR_DUPLICATE_KEY if a bucket holds two equal second halves.
void launch_bucket_dupcheck(const uint64_t *sorted, const uint64_t *acc, uint64_t nbuckets, DevStatus *status,
                            cudaStream_t st);
void launch_bucket_nodes(const uint64_t *acc, uint64_t nbuckets, DevTables tab, uint32_t *node_count, cudaStream_t st);
void launch_tree_emit(const uint64_t *acc, uint64_t nbuckets, const uint64_t *node_base, Shape sh, NodeArrays nodes,
                      cudaStream_t st);
// Stage lists: counting sort of node ids by stage. stage_info holds [kNumStages] counts
// followed by [kNumStages] bases; lists receives the node ids.
void launch_stage_lists(const uint8_t *stage, const uint64_t *total_nodes, uint32_t max_nodes, uint32_t *stage_info,
                        uint32_t *lists, cudaStream_t st);

// ---- search (rsb_search.cu) ----
struct SearchCtx {
    Shape sh;
    const uint64_t *node_total;  // device: number of nodes
    const uint32_t *stage_info;  // device: counts[kNumStages], bases[kNumStages]
    const uint32_t *lists;
    NodeArrays nodes;
    uint64_t *keys;              // bucket-partitioned key seconds
    DevTables tab;
    DevStatus *status;
    uint32_t *sched;             // per stage: fresh-node counter [0, kNumStages), finished nodes [kNumStages, 2*kNumStages)
    uint32_t *slots;             // help slots
    uint32_t nslots;
    uint32_t budget_shift;
    uint64_t budget_min;
    int num_sms;
    int occupancy_pct;           // persistent kernels keep this percentage of full occupancy
    uint64_t watchdog_ns;        // pipeline kernel: give up with RSB_ERR_TIMEOUT after this long (0: never)
};
// Launch schedule of one persistent search stage: candidates (seeds, or bases for rotation
// leaves) per lane of a window, and the percentage of full occupancy its grid keeps. Any
// valid schedule finds the same minimum seeds; only the speed differs.
struct StageSchedule {
    int seeds_per_lane;
    int occupancy_pct;
};
// Size class of a build for the schedule table: 0 below 2^20 keys, 1 from 2^20, 2 from 2^24.
constexpr int kScheduleSizeClasses = 3;
int schedule_size_class(uint64_t keys);
bool schedule_valid(int stage, const StageSchedule &s);
// The built-in (tuned) schedule; brute-force leaves always take 8 seeds per lane.
StageSchedule default_schedule(int leaf, int stage, int size_class);
// Device state of a pipeline launch (all aggregation and leaf searches in one persistent
// kernel with work queues; rsb_pipeline_impl.cuh).
// counts: [0,4) reserved tails, [4,8) heads, [8] completed nodes, [9] nodes of stages 17..20;
// when a bounded wait gives up, [10..32) describe the unfinished nodes (pipe_diagnose).
constexpr int kPipeCounters = 32;
struct PipeCtx {
    uint32_t *queue;    // node ids, one queue per stage 17..20 at that stage's list offset (kEmpty = not yet written)
    uint32_t *counts;   // kPipeCounters words, see above
    uint32_t *active;   // per node: warps working on it
    uint32_t *claimed;  // per node: 1 once completed
    uint8_t *blocked;   // per node: its parent is an aggregation node (it is queued by that parent)
};
// The searches of stages 17..20 in one launch (after the fanout-2 stages). Same seeds as the
// stage kernels. max_nodes bounds the node ids.
void search_pipeline(const SearchCtx &c, const PipeCtx &p, uint32_t max_nodes, const StageSchedule &aggr,
                     const StageSchedule &leaf, cudaStream_t st);
void search_higher(const SearchCtx &c, int depth, cudaStream_t st);
void search_aggr(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st);
void partition_aggr(const SearchCtx &c, int stage, cudaStream_t st);
void search_leaves(const SearchCtx &c, int stage, const StageSchedule &s, cudaStream_t st);
uint32_t search_slots_needed(int num_sms);

// ---- encoding (rsb_encode.cu) ----
struct EfParams {
    uint64_t num_buckets, u_cum_keys, u_position, l_cum_keys, l_position;
    int64_t cum_keys_min_delta, min_diff;
    uint64_t bits_per_key_fixed_point;
    uint64_t lower_words, cum_words, pos_words, jump_words;
    uint64_t total_bits;       // descriptor bits before the sentinel
    uint64_t desc_words;       // descriptor words incl. the sentinel
    uint64_t evals_alg;
    uint64_t evals_stage[kNumStages];
};

// Kernels launched by this library (all threads), for the launch accounting of rsb_stats.
void count_launches(uint64_t k);
uint64_t launches_so_far();
void probe_eval_rate(int num_sms, uint64_t *out_evals, cudaStream_t st);
void launch_bucket_bits(const uint64_t *node_base, uint64_t nbuckets, NodeArrays nodes, DevTables tab,
                        uint32_t *bits, uint32_t *fixed_bits, DevStatus *status, cudaStream_t st);
void launch_write_rice(const uint64_t *node_base, uint64_t nbuckets, NodeArrays nodes, DevTables tab,
                       const uint64_t *pos_acc, const uint32_t *fixed_bits, uint64_t *desc, uint64_t desc_cap_words,
                       EfParams *ef, DevStatus *status, cudaStream_t st);
void launch_ef_build(const uint64_t *cum, const uint64_t *pos, uint64_t nbuckets, uint64_t keys, EfParams *ef,
                     uint64_t *lower, uint64_t lower_cap, uint64_t *upper_cum, uint64_t cum_cap, uint64_t *upper_pos,
                     uint64_t pos_cap, uint64_t *jump, uint64_t jump_cap, DevStatus *status, cudaStream_t st);
// Also adds the candidate windows handed out by the persistent searches, per stage, to
// windows[0, kNumStages).
void launch_evals(const uint64_t *node_total, NodeArrays nodes, uint32_t leaf, uint32_t rotate, EfParams *ef,
                  uint64_t *windows, cudaStream_t st);

// ---- batched construction (rsb_batch.cu) ----
void launch_set_nbuckets(const uint64_t *set_key, uint32_t nsets, uint64_t bucket_size, uint32_t *nb, cudaStream_t st);
void launch_set_bucket_ids(const uint64_t *keys128, uint64_t n, const uint64_t *set_key, const uint64_t *set_bucket,
                           uint32_t nsets, uint64_t nb_total, uint32_t *bucket_id, uint32_t *counts, cudaStream_t st);
void launch_set_scatter(const uint64_t *keys128, uint64_t n, const uint64_t *set_key, const uint64_t *set_bucket,
                        uint32_t nsets, const uint32_t *bucket_id, const uint64_t *acc, uint32_t *cursor,
                        uint64_t nb_total, uint64_t *sorted, cudaStream_t st);
void launch_set_desc_words(const uint64_t *pos_acc, const uint64_t *set_bucket, uint32_t nsets, uint32_t *words,
                           uint64_t *set_bits, cudaStream_t st);
void launch_set_write_rice(const uint64_t *node_base, uint64_t nb_total, NodeArrays nodes, DevTables tab,
                           const uint64_t *pos_acc, const uint32_t *fixed_bits, const uint64_t *set_bucket,
                           uint32_t nsets, const uint64_t *word_base, const uint64_t *set_bits, uint64_t *desc,
                           uint64_t cap_words, DevStatus *status, cudaStream_t st);
void launch_set_ef_params(const uint64_t *acc, const uint64_t *pos, const uint64_t *set_bucket, uint32_t nsets,
                          EfParams *ef, uint32_t *lower_w, uint32_t *cum_w, uint32_t *pos_w, uint32_t *jump_w,
                          cudaStream_t st);
void launch_set_ef_fill(const uint64_t *acc, const uint64_t *pos, const uint64_t *set_bucket, uint32_t nsets,
                        const EfParams *ef, const uint64_t *lower_base, const uint64_t *cum_base, const uint64_t *pos_base,
                        const uint64_t *jump_base, uint64_t *lower, uint64_t *upper_cum, uint64_t *upper_pos,
                        uint64_t *jump, cudaStream_t st);

// ---- queries (rsb_query.cu) ----
struct MphfView;
void launch_query_view(const MphfView &f, const uint64_t *keys128, uint64_t n, uint64_t *out, cudaStream_t st);
// Device self-verification of a built function (RSB_VERIFY): every bucket's Elias-Fano entry
// against acc/pos, and every key to a distinct value below n (seen: (n + 31) / 32 words).
void launch_verify(const MphfView &f, const uint64_t *keys128, uint64_t n, const uint64_t *acc, const uint64_t *pos,
                   uint64_t nb, uint32_t *seen, DevStatus *status, cudaStream_t st);
bool shape_matches_kernels(const Shape &s);

}  // namespace rsb
