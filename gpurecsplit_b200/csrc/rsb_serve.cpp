// Serving: continuous batching of build requests over several engines on one device.
//
// Each of `inflight` workers owns an engine (its own CUDA stream and cached scratch). A free
// worker takes the oldest queued request plus every other queued request of the same class
// (leaf size, bucket size, flags, key kind) in arrival order while their estimated device
// working set fits its share of the HBM budget, builds them as one batch
// (rsb_build_batch_*), and hands each request its own function. Requests that arrive while
// batches run join the next batch a worker forms, and batches of different workers overlap
// on the device.
//
// Budget: at creation every engine reserves scratch for a fixed capacity (keys, string
// bytes, buckets, sets) derived from its share, and a batch is admitted only while it fits
// that capacity, so engines never grow and the server holds about hbm_budget bytes of
// device memory from creation to destruction.
//
// Lanes: with two or more workers, worker 0 serves only small requests (estimated device
// time below kSmallMs) on a high-priority stream, and the other workers take any request.
// The persistent search kernels of the large lanes keep kLargeLaneOccupancy percent of full
// occupancy and those of the small lane the rest, so a small request's grid is resident
// beside a running large build instead of queueing CTAs behind it (a persistent kernel
// cannot finish before all of its CTAs have started). A small request therefore never waits
// for a multi-second batch to finish.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime.h>

#include "rsb.h"

namespace {

using Clock = std::chrono::steady_clock;

constexpr double kSmallMs = 20.0;
// 67: with 16K-register search CTAs (256 threads x 64 registers) a large lane at 75 % holds 3
// of an SM's 4 CTA slots of registers and small builds slowed down several-fold (mixed-load
// p50 139 ms); at 67 % it holds 2 and the p50 is 28 ms at the same capacity (measured on one
// B200 with the serving benchmark).
constexpr uint32_t kLargeLaneOccupancy = 67;

// Device ns per key of a build by leaf size, interpolated geometrically between rates
// measured on one B200 (l = 8: 2, 12: 5, 16: 250, 24: 1e5 ns/key); used only to route
// requests between lanes.
double est_ns_per_key(uint32_t leaf) {
    static const double L[4] = {8, 12, 16, 24}, V[4] = {2, 5, 250, 1e5};
    if (leaf <= 8) return V[0];
    for (int i = 0; i < 3; ++i)
        if (leaf <= L[i + 1]) {
            const double t = (leaf - L[i]) / (L[i + 1] - L[i]);
            return std::exp(std::log(V[i]) + t * (std::log(V[i + 1]) - std::log(V[i])));
        }
    return V[3];
}

struct Request {
    uint64_t id = 0;
    uint32_t leaf = 0, flags = 0;
    uint64_t bucket = 0;
    bool strings = false;
    uint64_t n = 0;
    std::vector<uint8_t> bytes;      // string keys, concatenated
    std::vector<uint64_t> offsets;   // n + 1 entries into bytes
    std::vector<rsb_hash128> keys;   // hash128 keys
    uint64_t buckets = 0;            // buckets of this request's function
    double est_ms = 0;               // estimated device time of a build alone
    double submit_s = 0, admit_s = 0, done_s = 0;
    uint32_t batch_requests = 0;
    uint64_t batch_keys = 0;
    bool done = false;
    bool waited = false;  // a caller is in rsb_server_wait for this request (at most one)
    rsb_status status = RSB_OK;
    rsb_mphf *result = nullptr;

    bool same_class(const Request &o) const {
        return leaf == o.leaf && bucket == o.bucket && flags == o.flags && strings == o.strings;
    }
};

// Capacity of one worker with `share` bytes: a quarter for string bytes, the rest for keys
// at ~62.5 device bytes each (hash 16, partitioned key 8, bucket id 4, node arrays 23,
// descriptor 1, string offset 8, plus 40 per bucket at >= 16 keys per bucket), all with
// the engine's 1/8 allocation headroom.
struct Capacity {
    uint64_t keys = 0, bytes = 0, buckets = 0;
    uint32_t sets = 0;
};

Capacity capacity_for(uint64_t share) {
    Capacity c;
    c.bytes = (uint64_t)(share / 4 / 1.125);
    c.keys = (uint64_t)(share * 0.75 / (1.125 * 62.5));
    c.buckets = c.keys / 16 + 1024;
    c.sets = 1u << 16;
    return c;
}

}  // namespace

struct rsb_server {
    int device = 0;
    uint64_t budget = 0, share = 0, max_batch_keys = 0;
    Capacity cap;
    Clock::time_point t0;
    std::vector<rsb_engine *> engines;
    std::vector<cudaStream_t> streams;  // streams the server created for its engines
    std::vector<std::thread> workers;
    bool lanes = false;                 // worker 0 serves small requests only
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;
    std::unordered_map<uint64_t, Request *> requests;
    uint64_t next_id = 1;
    bool stopping = false;

    double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }
};

namespace {

// Builds the requests of one batch; on a batch failure (e.g. a duplicate key in one
// request) every request is built alone so that only the faulty one fails.
void build(rsb_engine *e, std::vector<Request *> &batch) {
    const uint32_t nsets = (uint32_t)batch.size();
    const Request &r0 = *batch[0];
    std::vector<uint64_t> set_offsets(nsets + 1, 0);
    for (uint32_t s = 0; s < nsets; ++s) set_offsets[s + 1] = set_offsets[s] + batch[s]->n;
    std::vector<rsb_mphf *> outs(nsets, nullptr);
    rsb_status st;
    if (r0.strings) {
        std::vector<uint64_t> offsets(set_offsets[nsets] + 1, 0);
        uint64_t total_bytes = 0;
        for (auto *r : batch) total_bytes += r->bytes.size();
        std::vector<uint8_t> bytes(total_bytes);
        uint64_t k = 0, b = 0;
        for (auto *r : batch) {
            if (!r->bytes.empty()) std::memcpy(bytes.data() + b, r->bytes.data(), r->bytes.size());
            for (uint64_t i = 0; i < r->n; ++i) offsets[k + i] = b + r->offsets[i];
            k += r->n;
            b += r->bytes.size();
        }
        offsets[k] = b;
        st = rsb_build_batch_strings(e, bytes.data(), offsets.data(), set_offsets.data(), nsets, r0.bucket, r0.leaf,
                                     r0.flags, outs.data(), nullptr);
    } else {
        std::vector<rsb_hash128> keys(set_offsets[nsets]);
        uint64_t k = 0;
        for (auto *r : batch) {
            if (r->n) std::memcpy(keys.data() + k, r->keys.data(), r->n * sizeof(rsb_hash128));
            k += r->n;
        }
        st = rsb_build_batch_hash128(e, keys.data(), set_offsets.data(), nsets, r0.bucket, r0.leaf, r0.flags,
                                     outs.data(), nullptr);
    }
    if (st == RSB_OK) {
        for (uint32_t s = 0; s < nsets; ++s) {
            batch[s]->result = outs[s];
            batch[s]->status = RSB_OK;
        }
        return;
    }
    if (nsets == 1) {
        batch[0]->status = st;
        return;
    }
    for (auto *r : batch) {
        std::vector<Request *> one{r};
        build(e, one);
    }
}

bool may_take(const rsb_server *S, size_t w, const Request *r) {
    return !(S->lanes && w == 0) || r->est_ms < kSmallMs;
}

void worker(rsb_server *S, size_t w) {
    rsb_engine *e = S->engines[w];
    for (;;) {
        std::vector<Request *> batch;
        uint64_t keys = 0;
        {
            std::unique_lock<std::mutex> lock(S->mu);
            Request *oldest = nullptr;
            S->cv_work.wait(lock, [&] {
                oldest = nullptr;
                for (Request *r : S->pending)
                    if (may_take(S, w, r)) {
                        oldest = r;
                        break;
                    }
                return S->stopping || oldest != nullptr;
            });
            if (!oldest) return;  // stopping, and nothing left this worker may take
            const Request *first = oldest;  // stays valid: it moves from the queue into the batch
            const Capacity &cap = S->cap;
            uint64_t bytes = 0, buckets = 0;
            for (auto it = S->pending.begin(); it != S->pending.end();) {
                Request *r = *it;
                const bool fits = keys + r->n <= cap.keys && bytes + r->bytes.size() <= cap.bytes &&
                                  buckets + r->buckets <= cap.buckets && batch.size() < cap.sets &&
                                  keys + r->n <= S->max_batch_keys;
                if (r->same_class(*first) && may_take(S, w, r) && (batch.empty() || fits)) {
                    batch.push_back(r);
                    keys += r->n;
                    bytes += r->bytes.size();
                    buckets += r->buckets;
                    it = S->pending.erase(it);
                } else {
                    ++it;
                }
            }
            const double t = S->now();
            for (auto *r : batch) r->admit_s = t;
        }
        const Request &r0 = *batch[0];
        if (batch.size() == 1 &&
            (r0.n > S->cap.keys || r0.bytes.size() > S->cap.bytes || r0.buckets > S->cap.buckets)) {
            batch[0]->status = RSB_ERR_OOM;  // larger than this worker's share of the budget
        } else {
            build(e, batch);
        }
        {
            std::lock_guard<std::mutex> lock(S->mu);
            const double t = S->now();
            for (auto *r : batch) {
                r->done = true;
                r->done_s = t;
                r->batch_requests = (uint32_t)batch.size();
                r->batch_keys = keys;
                r->bytes.clear();
                r->bytes.shrink_to_fit();
                r->offsets.clear();
                r->offsets.shrink_to_fit();
                r->keys.clear();
                r->keys.shrink_to_fit();
            }
        }
        S->cv_done.notify_all();
    }
}

rsb_status enqueue(rsb_server *S, Request *r, uint64_t *id) {
    {
        std::lock_guard<std::mutex> lock(S->mu);
        if (S->stopping) {
            delete r;
            return RSB_ERR_BAD_ARG;
        }
        r->id = S->next_id++;
        r->submit_s = S->now();
        S->pending.push_back(r);
        S->requests[r->id] = r;
        *id = r->id;
    }
    S->cv_work.notify_all();  // lanes differ in what they may take
    return RSB_OK;
}

bool valid_params(uint64_t bucket, uint32_t leaf) { return bucket > 0 && leaf >= 2 && leaf <= 24; }

}  // namespace

extern "C" {

rsb_status rsb_server_create(int device, uint64_t hbm_budget, uint32_t inflight, uint64_t max_batch_keys,
                             rsb_server **out) {
    if (!out || inflight == 0 || inflight > 16 || hbm_budget == 0) return RSB_ERR_BAD_ARG;
    auto *S = new (std::nothrow) rsb_server;
    if (!S) return RSB_ERR_OOM;
    S->device = device;
    S->budget = hbm_budget;
    S->share = hbm_budget / inflight;
    S->max_batch_keys = max_batch_keys ? max_batch_keys : (uint64_t)1 << 31;
    S->cap = capacity_for(S->share);
    S->t0 = Clock::now();
    S->lanes = inflight >= 2;
    auto fail = [&](rsb_status st) {
        for (auto *x : S->engines) rsb_engine_destroy(x);
        for (auto s : S->streams) cudaStreamDestroy(s);
        delete S;
        return st;
    };
    for (uint32_t i = 0; i < inflight; ++i) {
        cudaStream_t stream = nullptr;
        if (S->lanes && i == 0) {  // the small-request lane runs on the highest stream priority
            int least = 0, greatest = 0;
            if (cudaSetDevice(device) != cudaSuccess || cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess ||
                cudaStreamCreateWithPriority(&stream, cudaStreamNonBlocking, greatest) != cudaSuccess) {
                cudaGetLastError();
                return fail(RSB_ERR_NO_DEVICE);
            }
            S->streams.push_back(stream);
        }
        rsb_engine *e = nullptr;
        rsb_status st = rsb_engine_create(device, stream, &e);
        if (st == RSB_OK && S->lanes)
            st = rsb_engine_set_occupancy(e, i == 0 ? 100 - kLargeLaneOccupancy : kLargeLaneOccupancy);
        if (st == RSB_OK) st = rsb_engine_reserve(e, S->cap.keys, 16, S->cap.bytes, S->cap.sets);
        if (st != RSB_OK) {
            if (e) rsb_engine_destroy(e);
            return fail(st);
        }
        S->engines.push_back(e);
    }
    for (size_t i = 0; i < S->engines.size(); ++i) S->workers.emplace_back(worker, S, i);
    *out = S;
    return RSB_OK;
}

rsb_status rsb_server_submit_strings(rsb_server *S, const uint8_t *bytes, const uint64_t *offsets, uint64_t n,
                                     uint64_t bucket, uint32_t leaf, uint32_t flags, uint64_t *id) {
    if (!S || !offsets || !id || !valid_params(bucket, leaf)) return RSB_ERR_BAD_ARG;
    for (uint64_t i = 0; i < n; ++i)
        if (offsets[i + 1] < offsets[i]) return RSB_ERR_BAD_ARG;
    auto *r = new (std::nothrow) Request;
    if (!r) return RSB_ERR_OOM;
    r->strings = true;
    r->leaf = leaf;
    r->bucket = bucket;
    r->flags = flags & RSB_ROTATE;
    r->n = n;
    const uint64_t b0 = offsets[0], b1 = offsets[n];
    r->bytes.assign(bytes + b0, bytes + b1);
    r->offsets.resize(n + 1);
    for (uint64_t i = 0; i <= n; ++i) r->offsets[i] = offsets[i] - b0;
    r->buckets = std::max<uint64_t>(1, (n + bucket - 1) / bucket);
    r->est_ms = n * est_ns_per_key(leaf) * 1e-6;
    return enqueue(S, r, id);
}

rsb_status rsb_server_submit_hash128(rsb_server *S, const rsb_hash128 *keys, uint64_t n, uint64_t bucket,
                                     uint32_t leaf, uint32_t flags, uint64_t *id) {
    if (!S || (n && !keys) || !id || !valid_params(bucket, leaf)) return RSB_ERR_BAD_ARG;
    auto *r = new (std::nothrow) Request;
    if (!r) return RSB_ERR_OOM;
    r->leaf = leaf;
    r->bucket = bucket;
    r->flags = flags & RSB_ROTATE;
    r->n = n;
    r->keys.assign(keys, keys + n);
    r->buckets = std::max<uint64_t>(1, (n + bucket - 1) / bucket);
    r->est_ms = n * est_ns_per_key(leaf) * 1e-6;
    return enqueue(S, r, id);
}

rsb_status rsb_server_wait(rsb_server *S, uint64_t id, double timeout_s, rsb_mphf **out, rsb_request_info *info) {
    if (!S || !out) return RSB_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lock(S->mu);
    auto it = S->requests.find(id);
    if (it == S->requests.end()) return RSB_ERR_BAD_ARG;
    Request *r = it->second;
    // One waiter per request: the waiter that returns the result frees the request, so a
    // second concurrent waiter would read freed memory. It is refused instead.
    if (r->waited) return RSB_ERR_BAD_ARG;
    r->waited = true;
    auto ready = [&] { return r->done; };
    if (timeout_s < 0) S->cv_done.wait(lock, ready);
    else if (!S->cv_done.wait_for(lock, std::chrono::duration<double>(timeout_s), ready)) {
        r->waited = false;  // the request stays; it may be waited for again
        return RSB_ERR_TIMEOUT;
    }
    if (info) {
        info->submit_s = r->submit_s;
        info->admit_s = r->admit_s;
        info->done_s = r->done_s;
        info->batch_requests = r->batch_requests;
        info->batch_keys = r->batch_keys;
    }
    const rsb_status st = r->status;
    *out = r->result;
    S->requests.erase(id);  // by key: submissions during the wait may have rehashed the map
    delete r;
    return st;
}

rsb_status rsb_server_destroy(rsb_server *S) {
    if (!S) return RSB_ERR_BAD_ARG;
    {
        std::lock_guard<std::mutex> lock(S->mu);
        S->stopping = true;
    }
    S->cv_work.notify_all();
    for (auto &t : S->workers) t.join();
    for (auto *e : S->engines) rsb_engine_destroy(e);
    for (auto s : S->streams) cudaStreamDestroy(s);
    for (auto &kv : S->requests) {
        if (kv.second->result) rsb_free(kv.second->result);
        delete kv.second;
    }
    delete S;
    return RSB_OK;
}

}  // extern "C"
