/*
 * rsb.h — C ABI of the B200-native RecSplit construction engine (librsb.so).
 *
 * This is the drop-in boundary for the construction path of ByteHamster/GpuRecSplit.
 * Every entry point takes plain pointers and sizes; no C++ or CUDA types cross it
 * (streams are passed as void*). The C++ class in include/rsb/GPURecSplit.hpp wraps
 * these calls behind the reference's GPURecSplit<LEAF_SIZE, AT, ROTATE> interface.
 *
 * Reference interfaces are cited as path:line within the GpuRecSplit project.
 *
 * Ownership: the caller owns every input buffer; the library owns engines and handles
 * and frees them in rsb_engine_destroy / rsb_free. The library never calls exit(),
 * abort() or cudaDeviceReset(); every failure is returned as an rsb_status.
 * Threading: an engine may be used by one host thread at a time; handles are immutable
 * after construction and may be queried concurrently.
 */
#ifndef RSB_H_
#define RSB_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum rsb_status {
    RSB_OK = 0,
    RSB_ERR_BAD_ARG = 1,          /* invalid leaf size, bucket size, pointer or flag */
    RSB_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    RSB_ERR_OOM = 3,              /* device or host allocation failed */
    RSB_ERR_DUPLICATE_KEY = 4,    /* two keys share a bucket and the same second half; the
                                     reference loops forever here (GPURecSplit.cuh:436) */
    RSB_ERR_SEARCH_BUDGET = 5,    /* a seed search exceeded its candidate budget */
    RSB_ERR_BUCKET_TOO_LARGE = 6, /* a bucket holds >= 3000 keys (AbstractParallelRecSplit.hpp:60;
                                     the reference throws std::out_of_range, GPURecSplit.cuh:682) */
    RSB_ERR_TIMEOUT = 7,          /* a bounded device wait gave up */
    RSB_ERR_FORMAT = 8,           /* malformed serialized input or leaf-size mismatch
                                     (the reference abort()s, GPURecSplit.cuh:831-833) */
    RSB_ERR_INTERNAL = 9,
    RSB_ERR_NO_DEVICE = 10        /* no CUDA device or the kernels do not match it */
} rsb_status;

/* Build flags. */
#define RSB_ROTATE 1u          /* USE_BIJECTIONS_ROTATE template parameter (reference default true) */
#define RSB_KEYS_ON_DEVICE 2u  /* key pointers are device memory; otherwise host memory */
#define RSB_DEVICE_ONLY 4u     /* keep the result on the device; the host copy is made lazily */
#define RSB_KEEP_SEEDS 8u      /* keep the DFS seed stream for rsb_seeds() */
#define RSB_VERIFY 16u         /* plain builds: verify the result on the device before returning - every
                                  bucket's Elias-Fano entry decodes to its offsets (the check the
                                  reference's debug builds run, DoubleEF.hpp:351-364) and every key maps
                                  to a distinct value in [0, n); a failure returns RSB_ERR_INTERNAL */

/* 128-bit key hash: util/Hash128.h:14-23 (hash128_t{first, second}). */
typedef struct rsb_hash128 {
    uint64_t first, second;
} rsb_hash128;

typedef struct rsb_engine rsb_engine; /* device context: stream, cached scratch, tables */
typedef struct rsb_mphf rsb_mphf;     /* one built minimal perfect hash function */

/* Per-build measurements (device time from CUDA events on the engine stream). */
typedef struct rsb_stats {
    uint64_t keys;
    uint64_t buckets;
    uint64_t nodes;                /* seeds in the descriptor stream */
    uint64_t nodes_per_stage[21];  /* 0..16 fanout-2 depth d, 17 upper aggr, 18 lower aggr, 19 rotation leaves, 20 other leaves */
    uint64_t evals_alg;            /* sum over nodes of (trials up to the found seed) * node size */
    uint64_t descriptor_bits;      /* Golomb-Rice stream length without the sentinel */
    double ms_total;               /* whole build on the device */
    double ms_partition;           /* hashing, bucket histogram/scan/scatter, per-bucket sort */
    double ms_search[21];          /* per search stage */
    double ms_encode;              /* Rice + Elias-Fano */
    uint64_t evals_stage[21];      /* evals_alg split by search stage */
    uint64_t kernel_launches;      /* kernels this build launched */
    uint64_t windows_stage[21];    /* candidate windows handed out per persistent search stage (17..20) */
    uint64_t window_candidates[21];/* candidates (seeds; bases for rotation leaves) per window of that stage */
} rsb_stats;

/* ---- engine ------------------------------------------------------------------------ */

/* Creates an engine on `device` (an int CUDA ordinal). `stream` (a cudaStream_t, may be
 * NULL for a private stream) is where all work of this engine is enqueued. */
rsb_status rsb_engine_create(int device, void *stream, rsb_engine **out);
rsb_status rsb_engine_destroy(rsb_engine *engine);
/* Candidate budget of every seed search: 2^(g(m) + shift) seeds, at least 2^16 (default
 * shift 10). Exceeding it ends the build with RSB_ERR_SEARCH_BUDGET instead of looping. */
rsb_status rsb_engine_set_budget(rsb_engine *engine, uint32_t shift, uint64_t min_candidates);
/* Pre-sizes the engine's cached device scratch (no reference counterpart) for builds, plain
 * or batched, of up to `keys` keys in up to `sets` sets, with buckets of at least
 * `bucket_size` keys and up to `string_bytes` bytes of host string keys, so that such builds
 * allocate no scratch (growing scratch frees and reallocates, which waits for the device).
 * Returns RSB_ERR_OOM, leaving the engine usable, if the device cannot hold it. */
rsb_status rsb_engine_reserve(rsb_engine *engine, uint64_t keys, uint64_t bucket_size, uint64_t string_bytes,
                              uint32_t sets);
/* Limits the engine's persistent seed-search kernels to `percent` (1..100, default 100) of
 * their full occupancy on every SM (no reference counterpart), leaving room on each SM for
 * kernels of other streams - e.g. small requests of a build service running beside a large
 * build. Results do not change; only scheduling does. */
rsb_status rsb_engine_set_occupancy(rsb_engine *engine, uint32_t percent);
/* Pipeline mode (no reference counterpart; off by default): the aggregation and leaf searches
 * of every build run as one persistent launch with device work queues - a node is searched as
 * soon as its parent has been partitioned, instead of stage after stage with a barrier
 * between stages. The function is the same. on: 0 or 1. */
rsb_status rsb_engine_set_pipeline(rsb_engine *engine, uint32_t on);
/* Upper bound on one pipeline-mode launch in seconds (0, the default: none). A launch that
 * runs longer stops and the build returns RSB_ERR_TIMEOUT; the engine stays usable. A guard
 * for callers that prefer an error to an unexpectedly long build. */
rsb_status rsb_engine_set_watchdog(rsb_engine *engine, double seconds);
/* Schedule of one persistent search stage (no reference counterpart: the reference's launch
 * constants are fixed, GPURecSplit.cuh:420-425): candidates per lane of a search window and
 * the percentage of the engine's occupancy the stage's grid keeps, for builds of `leaf_size`
 * in size class `size_class` (0: fewer than 2^20 keys, 1: 2^20 to 2^24, 2: at least 2^24).
 * `stage`: 17 upper aggregation (seeds_per_lane 4, 8, 12 or 16), 18 lower aggregation (4, 8, 12 or 16), 19 rotation
 * leaves (bases per lane 4, 8 or 12); occupancy 1..100. seeds_per_lane 0 restores the
 * built-in schedule (the table gpurecsplit_b200/tune.py measured). Every schedule finds the
 * same minimum seeds: results never change, only speed. */
rsb_status rsb_engine_set_schedule(rsb_engine *engine, uint32_t leaf_size, uint32_t stage, uint32_t size_class,
                                   uint32_t seeds_per_lane, uint32_t occupancy_pct);
rsb_status rsb_engine_get_schedule(rsb_engine *engine, uint32_t leaf_size, uint32_t stage, uint32_t size_class,
                                   uint32_t *seeds_per_lane, uint32_t *occupancy_pct);

/* ---- construction ------------------------------------------------------------------ */

/* Replaces GPURecSplit(vector<hash128_t>& keys, size_t bucket_size, int numThreads),
 * GPURecSplit.cuh:484-489 (same for SIMDRecSplit.hpp:228-232). The caller's keys are
 * not modified (the reference sorts them in place, AbstractParallelRecSplit.hpp:344). */
rsb_status rsb_build_hash128(rsb_engine *engine, const rsb_hash128 *keys, uint64_t n, uint64_t bucket_size,
                             uint32_t leaf_size, uint32_t flags, rsb_mphf **out);

/* Replaces GPURecSplit(const vector<string>& keys, size_t bucket_size, int numThreads),
 * GPURecSplit.cuh:443-472: key i is bytes[offsets[i] .. offsets[i+1]); hashed on the
 * device with SpookyHash V2 (seed 0), first = h1, second = h0 (util/Hash128.h:32-36). */
rsb_status rsb_build_strings(rsb_engine *engine, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                             uint64_t bucket_size, uint32_t leaf_size, uint32_t flags, rsb_mphf **out);

/* 64-bit integer keys (no reference counterpart: the reference benchmarks feed random
 * hash128 values, benchmark/benchmark_construction.hpp:54-58). Each key k is mixed to
 * first = fmix64(k) (MurmurHash3), second = stafford13(k + 0x9e3779b97f4a7c15). */
rsb_status rsb_build_u64(rsb_engine *engine, const uint64_t *keys, uint64_t n, uint64_t bucket_size,
                         uint32_t leaf_size, uint32_t flags, rsb_mphf **out);

/* Batched construction (no reference counterpart: the reference builds one set per
 * constructor call). Builds nsets independent functions in one device pipeline; set s is
 * keys[set_offsets[s] .. set_offsets[s+1]) (set_offsets: host memory, nsets + 1 entries,
 * starting at 0, non-decreasing). outs[s] is identical to the plain build of set s with the
 * same bucket size, leaf size and flags; it lives on the host. `stats` (may be NULL)
 * receives the whole batch's measurements. */
rsb_status rsb_build_batch_hash128(rsb_engine *engine, const rsb_hash128 *keys, const uint64_t *set_offsets,
                                   uint32_t nsets, uint64_t bucket_size, uint32_t leaf_size, uint32_t flags,
                                   rsb_mphf **outs, rsb_stats *stats);
rsb_status rsb_build_batch_u64(rsb_engine *engine, const uint64_t *keys, const uint64_t *set_offsets, uint32_t nsets,
                               uint64_t bucket_size, uint32_t leaf_size, uint32_t flags, rsb_mphf **outs,
                               rsb_stats *stats);
/* String keys: key i is bytes[offsets[i] .. offsets[i+1]) (offsets has set_offsets[nsets] + 1
 * entries); set s is keys set_offsets[s] .. set_offsets[s+1]. */
rsb_status rsb_build_batch_strings(rsb_engine *engine, const uint8_t *bytes, const uint64_t *offsets,
                                   const uint64_t *set_offsets, uint32_t nsets, uint64_t bucket_size,
                                   uint32_t leaf_size, uint32_t flags, rsb_mphf **outs, rsb_stats *stats);

/* ---- serving: continuous batching of build requests (no reference counterpart) ---------
 * A server owns `inflight` engines on one device, each with a worker thread. At creation
 * every engine reserves scratch for its share of `hbm_budget` bytes (hbm_budget / inflight):
 * room for a fixed number of keys, string bytes and buckets. Submitted requests wait in a
 * queue; whenever a worker is free it takes the oldest request and every other queued
 * request of the same (leaf size, bucket size, flags, key kind) class, in arrival order, as
 * long as the batch fits that reservation (and `max_batch_keys`, 0 = no limit), and builds
 * them as one batch. Batches on different workers overlap on the device. A request that
 * alone exceeds a worker's reservation fails with RSB_ERR_OOM; a request whose batch fails
 * is rebuilt alone, so only a faulty request (e.g. duplicate keys) fails. Results are
 * bit-identical to plain builds of the same keys. */
typedef struct rsb_server rsb_server;
typedef struct rsb_request_info {
    double submit_s, admit_s, done_s; /* steady-clock seconds since the server was created */
    uint32_t batch_requests;          /* requests built together with this one (itself included) */
    uint64_t batch_keys;
} rsb_request_info;
rsb_status rsb_server_create(int device, uint64_t hbm_budget, uint32_t inflight, uint64_t max_batch_keys,
                             rsb_server **out);
/* Copies the keys; returns at once with the request's id. */
rsb_status rsb_server_submit_strings(rsb_server *server, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                                     uint64_t bucket_size, uint32_t leaf_size, uint32_t flags, uint64_t *id);
rsb_status rsb_server_submit_hash128(rsb_server *server, const rsb_hash128 *keys, uint64_t n, uint64_t bucket_size,
                                     uint32_t leaf_size, uint32_t flags, uint64_t *id);
/* Waits for request `id` (at most timeout_s seconds; < 0 waits without limit) and hands
 * over its function (the caller frees it with rsb_free). RSB_ERR_TIMEOUT if not done (the
 * request can be waited for again). One caller at a time may wait for a request: a second
 * concurrent wait for the same id returns RSB_ERR_BAD_ARG, as does a wait for an id whose
 * result was already handed over. */
rsb_status rsb_server_wait(rsb_server *server, uint64_t id, double timeout_s, rsb_mphf **out, rsb_request_info *info);
/* Stops accepting requests, finishes the queued ones and releases the engines. */
rsb_status rsb_server_destroy(rsb_server *server);

/* ---- sharded construction over bucket ranges (several GPUs) ---------------------------
 * No reference counterpart as an API: the reference builds contiguous bucket ranges in its
 * threads and appends their Rice streams in bucket order (SIMDRecSplit.hpp:695-745). Here a
 * range can be built on another GPU (or process) and the ranges merged into the one function
 * the plain build makes from all keys, byte for byte. */

/* Builds the part of an nbuckets_total-bucket function (nbuckets_total = ceil(n_all /
 * bucket_size) for the n_all keys of all parts) that covers buckets [bucket_lo, bucket_hi):
 * `keys` are exactly the keys whose bucket remap128(first, nbuckets_total) lies in the range,
 * in any order (a key outside it returns RSB_ERR_BAD_ARG). The handle serves rsb_part_export;
 * it is not itself a complete function. */
rsb_status rsb_build_part_hash128(rsb_engine *engine, const rsb_hash128 *keys, uint64_t n, uint64_t nbuckets_total,
                                  uint64_t bucket_lo, uint64_t bucket_hi, uint64_t bucket_size, uint32_t leaf_size,
                                  uint32_t flags, rsb_mphf **out);
/* Writes a part as bytes (its bucket range, per-bucket key and bit offsets, Rice bits) to
 * hand to the merging process. With buf == NULL only *len is set. */
rsb_status rsb_part_export(rsb_mphf *part, uint8_t *buf, size_t *len);
/* Merges exported parts that tile buckets [0, nbuckets_total) in order into the complete
 * function (host and device copies; the Elias-Fano index is built on the engine's device).
 * `leaf_size` and RSB_ROTATE in `flags` must match the parts'. RSB_ERR_FORMAT for malformed
 * parts, RSB_ERR_BAD_ARG for parts that do not tile one function. */
rsb_status rsb_merge_parts(rsb_engine *engine, const uint8_t *const *parts, const size_t *lens, uint32_t nparts,
                           uint32_t leaf_size, uint32_t flags, rsb_mphf **out);

/* ---- queries and accessors --------------------------------------------------------- */

/* Replaces size_t operator()(const hash128_t&), AbstractParallelRecSplit.hpp:409-466
 * (host evaluation; keys and out are host memory). */
rsb_status rsb_query_hash128(rsb_mphf *mphf, const rsb_hash128 *keys, uint64_t n, uint64_t *out);
/* Replaces size_t operator()(const string&), AbstractParallelRecSplit.hpp:473. */
rsb_status rsb_query_strings(rsb_mphf *mphf, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                             uint64_t *out);
/* Device evaluation of operator() for many keys (keys and out are device memory, work is
 * enqueued on the engine stream and completed before return). */
rsb_status rsb_query_device(rsb_engine *engine, rsb_mphf *mphf, const rsb_hash128 *keys, uint64_t n,
                            uint64_t *out);

/* Replaces size_t getBits(), AbstractParallelRecSplit.hpp:476-478. */
rsb_status rsb_get_bits(rsb_mphf *mphf, uint64_t *bits);
/* Replaces operator<<, GPURecSplit.cuh:817-825. With buf == NULL only *len is set. */
rsb_status rsb_serialize(rsb_mphf *mphf, uint8_t *buf, size_t *len);
/* Replaces operator>>, GPURecSplit.cuh:827-841; a leaf size other than `leaf_size`
 * returns RSB_ERR_FORMAT instead of abort(). `flags` carries RSB_ROTATE. */
rsb_status rsb_deserialize(const uint8_t *buf, size_t len, uint32_t leaf_size, uint32_t flags, rsb_mphf **out);
/* Seeds in descriptor (DFS pre-order) order with the size of each node; for parity
 * debugging (no reference counterpart). With seeds == NULL only *count is set. */
rsb_status rsb_seeds(rsb_mphf *mphf, uint64_t *seeds, uint32_t *sizes, size_t *count);
rsb_status rsb_get_stats(rsb_mphf *mphf, rsb_stats *stats);
rsb_status rsb_free(rsb_mphf *mphf);

/* ---- hashing only (parity checks of the key mixers) --------------------------------- */
rsb_status rsb_hash_strings(rsb_engine *engine, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                            uint32_t flags, rsb_hash128 *out);
rsb_status rsb_hash_u64(rsb_engine *engine, const uint64_t *keys, uint64_t n, uint32_t flags, rsb_hash128 *out);

/* rsb_hash_strings without any device allocation. No counterpart in the reference.
 * For callers that cannot allocate device memory (a plugin inside a host process that owns
 * all device memory through its own pool, or a serving thread that must not call cudaMalloc
 * because it can synchronise the device). Key i is bytes[offsets[i] .. offsets[i+1]); only
 * bytes[offsets[0] .. offsets[n]) is read, so `offsets` may index into a larger buffer.
 * bytes, offsets and out are host memory; the work runs on the current device and on
 * `stream` (a cudaStream_t, NULL for the default stream) and is complete on return. The
 * results equal rsb_hash_strings'. Staging uses one fixed array of device memory inside the
 * library (about 1.8 MiB, held by every GPU that loads the library until exit), so at most
 * 32,768 keys and 1 MiB of key bytes (offsets[n] - offsets[0]) per call: larger inputs return
 * RSB_ERR_BAD_ARG. The array is created when the library's device code is loaded on a
 * device: at the first call under lazy module loading (the CUDA 12 default) or at context
 * creation with CUDA_MODULE_LOADING=EAGER, so make one small call on each device before a
 * memory pool claims all of its memory. The first call on a device also resolves the
 * array's address (cudaGetSymbolAddress); make it before any stream capture. Each call copies
 * through pageable host memory and waits for `stream`, so a stream that is capturing is
 * refused with RSB_ERR_BAD_ARG before any work. A CUDA error already pending on the calling
 * thread is left in place and the call returns RSB_ERR_CUDA. Calls share the array; a
 * process-wide lock held until the stream finishes keeps their GPU work from overlapping. */
rsb_status rsb_hash_strings_static(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, rsb_hash128 *out,
                                   void *stream);

/* Measures the device's rate of remixAndRemap32 candidate evaluations (the primitive of
 * every seed search) with a synthetic kernel at full occupancy: the integer ceiling the
 * search kernels are compared with. No reference counterpart. */
rsb_status rsb_probe_eval_rate(rsb_engine *engine, double *evals_per_second, double *ms);

/* Golomb-Rice table of the engine for one leaf size (3000 entries), the table generated by
 * fill_golomb_rice<LEAF_SIZE>() (AbstractParallelRecSplit.hpp:191-227) and shipped as
 * golombRiceMemo.hpp. Host-only; needs no device. */
rsb_status rsb_golomb_memo(uint32_t leaf_size, uint32_t *out);

const char *rsb_strerror(rsb_status status);
/* Library version string. */
const char *rsb_version(void);

#ifdef __cplusplus
}
#endif

#endif /* RSB_H_ */
