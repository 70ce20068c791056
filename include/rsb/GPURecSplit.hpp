// Drop-in C++ interface of the B200 construction engine.
//
// Source-compatible with the construction API of ByteHamster/GpuRecSplit:
//   template <size_t LEAF_SIZE, sux::util::AllocType AT = MALLOC, bool USE_BIJECTIONS_ROTATE = true>
//   class GPURecSplit / SIMDRecSplit      include/function/GPURecSplit.cuh:409-505,
//                                         include/function/SIMDRecSplit.hpp:161-247
//   size_t operator()(const hash128_t&)   include/function/AbstractParallelRecSplit.hpp:409-466
//   size_t operator()(const string&)      :473
//   size_t getBits()                      :476-478
//   operator<< / operator>>               GPURecSplit.cuh:817-841
// Both class names build the same function as the reference's SIMDRecSplit and GPURecSplit
// (16-bit remap; the reference's equivalence test holds them equal). Construction runs on
// the GPU through the C ABI of rsb.h (link with -lrsb); queries and serialization run on
// the host. Errors throw std::runtime_error instead of looping forever (duplicate keys) or
// calling exit()/abort().
#pragma once

#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <istream>
#include <mutex>
#include <ostream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../rsb.h"

#ifndef RSB_NO_SUX_ALLOCTYPE
// The reference's third template parameter is sux::util::AllocType; construction on the GPU
// does not depend on it. Define RSB_NO_SUX_ALLOCTYPE when sux's own definition is visible.
namespace sux::util {
enum AllocType { MALLOC, SMALLPAGE, TRANSHUGEPAGE, FORCEHUGEPAGE };
}
#endif

namespace bez::function {

// util/Hash128.h:14-23 — layout-compatible with rsb_hash128.
typedef struct __hash128_t {
    uint64_t first, second;
    bool operator<(const __hash128_t &o) const { return first < o.first || second < o.second; }
    __hash128_t() = default;
    __hash128_t(const uint64_t first, const uint64_t second) : first(first), second(second) {}
} hash128_t;
static_assert(sizeof(hash128_t) == sizeof(rsb_hash128), "hash128_t must match rsb_hash128");

namespace rsb_detail {

inline void check(rsb_status s, const char *what) {
    if (s != RSB_OK) throw std::runtime_error(std::string(what) + ": " + rsb_strerror(s));
}

// One engine per process on the current CUDA device (selected with RSB_DEVICE, default 0).
inline rsb_engine *engine() {
    static std::mutex mu;
    static rsb_engine *e = nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!e) {
        const char *d = std::getenv("RSB_DEVICE");
        check(rsb_engine_create(d ? std::atoi(d) : 0, nullptr, &e), "rsb_engine_create");
    }
    return e;
}

inline void read_exact(std::istream &is, void *dst, size_t n) {
    is.read((char *)dst, (std::streamsize)n);
    if (!is) throw std::runtime_error("GPURecSplit: truncated stream");
}

}  // namespace rsb_detail

template <size_t LEAF_SIZE, sux::util::AllocType AT = sux::util::AllocType::MALLOC, bool USE_BIJECTIONS_ROTATE = true>
class GPURecSplit {
    static_assert(LEAF_SIZE >= 2 && LEAF_SIZE <= 24, "LEAF_SIZE must be in [2, 24]");
    static constexpr uint32_t kFlags = USE_BIJECTIONS_ROTATE ? RSB_ROTATE : 0u;
    rsb_mphf *h_ = nullptr;

    void reset(rsb_mphf *h) {
        if (h_) rsb_free(h_);
        h_ = h;
    }

  public:
    GPURecSplit() {}

    // GPURecSplit.cuh:443-472 (string keys, hashed with SpookyHash V2 on the device).
    GPURecSplit(const std::vector<std::string> &keys, const size_t bucket_size, const int /*numThreads*/ = 1) {
        std::vector<uint64_t> offsets(keys.size() + 1, 0);
        for (size_t i = 0; i < keys.size(); ++i) offsets[i + 1] = offsets[i] + keys[i].size();
        std::vector<uint8_t> bytes(offsets.back());
        for (size_t i = 0; i < keys.size(); ++i)
            if (!keys[i].empty()) std::memcpy(bytes.data() + offsets[i], keys[i].data(), keys[i].size());
        rsb_mphf *h = nullptr;
        rsb_detail::check(rsb_build_strings(rsb_detail::engine(), bytes.data(), offsets.data(), keys.size(), bucket_size,
                                            LEAF_SIZE, kFlags, &h),
                          "GPURecSplit(strings)");
        reset(h);
    }

    // GPURecSplit.cuh:484-489. Unlike the reference, the caller's vector is not reordered.
    GPURecSplit(std::vector<hash128_t> &keys, const size_t bucket_size, const int /*numThreads*/ = 1) {
        rsb_mphf *h = nullptr;
        rsb_detail::check(rsb_build_hash128(rsb_detail::engine(), (const rsb_hash128 *)keys.data(), keys.size(),
                                            bucket_size, LEAF_SIZE, kFlags, &h),
                          "GPURecSplit(hash128)");
        reset(h);
    }

    // GPURecSplit.cuh:498-505: one key per line.
    GPURecSplit(std::ifstream &input, const size_t bucket_size, const int numThreads = 1) {
        std::vector<std::string> keys;
        for (std::string key; std::getline(input, key);) keys.push_back(key);
        *this = GPURecSplit(keys, bucket_size, numThreads);
    }

    GPURecSplit(const GPURecSplit &) = delete;
    GPURecSplit &operator=(const GPURecSplit &) = delete;
    GPURecSplit(GPURecSplit &&o) noexcept : h_(o.h_) { o.h_ = nullptr; }
    GPURecSplit &operator=(GPURecSplit &&o) noexcept {
        if (this != &o) {
            reset(o.h_);
            o.h_ = nullptr;
        }
        return *this;
    }
    ~GPURecSplit() { reset(nullptr); }

    size_t operator()(const hash128_t &hash) {
        uint64_t v = 0;
        rsb_detail::check(rsb_query_hash128(h_, (const rsb_hash128 *)&hash, 1, &v), "GPURecSplit::operator()");
        return (size_t)v;
    }

    size_t operator()(const std::string &key) {
        const uint64_t offsets[2] = {0, key.size()};
        uint64_t v = 0;
        rsb_detail::check(rsb_query_strings(h_, (const uint8_t *)key.data(), offsets, 1, &v), "GPURecSplit::operator()");
        return (size_t)v;
    }

    // Many queries at once (host evaluation).
    void operator()(const hash128_t *keys, size_t n, uint64_t *out) {
        rsb_detail::check(rsb_query_hash128(h_, (const rsb_hash128 *)keys, n, out), "GPURecSplit::operator()");
    }

    // The reference adds the size of its own object (AbstractParallelRecSplit.hpp:476-478):
    // three size_t fields, the descriptor RiceBitVector (one sux Vector), and DoubleEF (four
    // sux Vectors and ten 64-bit fields). sux's Vector is taken as three words (size,
    // capacity, data pointer), so the count equals a reference build's on the same function.
    static constexpr size_t kReferenceObjectBytes = 3 * 8 + 5 * (3 * 8) + 10 * 8;

    size_t getBits() {
        uint64_t bits = 0;
        rsb_detail::check(rsb_get_bits(h_, &bits), "GPURecSplit::getBits");
        return (size_t)bits + 8 * kReferenceObjectBytes;
    }

    rsb_mphf *handle() const { return h_; }

    friend std::ostream &operator<<(std::ostream &os, const GPURecSplit &rs) {
        size_t len = 0;
        rsb_detail::check(rsb_serialize(rs.h_, nullptr, &len), "GPURecSplit::operator<<");
        std::vector<uint8_t> buf(len);
        rsb_detail::check(rsb_serialize(rs.h_, buf.data(), &len), "GPURecSplit::operator<<");
        os.write((const char *)buf.data(), (std::streamsize)len);
        return os;
    }

    // Reads leaf size, bucket size, key count, the descriptor vector, six Elias-Fano scalars
    // and four Elias-Fano vectors (AbstractParallelRecSplit.hpp:490-504, DoubleEF.hpp:115-135).
    friend std::istream &operator>>(std::istream &is, GPURecSplit &rs) {
        std::vector<uint8_t> buf;
        auto take = [&](size_t n) {
            const size_t o = buf.size();
            buf.resize(o + n);
            rsb_detail::read_exact(is, buf.data() + o, n);
            return o;
        };
        auto take_vec = [&]() {
            uint64_t n;
            const size_t at = take(8);  // take() may reallocate buf: read the count after it
            std::memcpy(&n, buf.data() + at, 8);
            if (n > (uint64_t(1) << 40)) throw std::runtime_error("GPURecSplit: malformed stream");
            take(n * 8);
        };
        take(24);
        take_vec();
        take(48);
        for (int i = 0; i < 4; ++i) take_vec();
        rsb_mphf *h = nullptr;
        rsb_detail::check(rsb_deserialize(buf.data(), buf.size(), LEAF_SIZE, kFlags, &h), "GPURecSplit::operator>>");
        rs.reset(h);
        return is;
    }
};

// SIMDRecSplit builds the same function as GPURecSplit (SIMDRecSplit.hpp:161-163).
template <size_t LEAF_SIZE, sux::util::AllocType AT = sux::util::AllocType::MALLOC, bool USE_BIJECTIONS_ROTATE = true>
using SIMDRecSplit = GPURecSplit<LEAF_SIZE, AT, USE_BIJECTIONS_ROTATE>;

}  // namespace bez::function
