/*
 * TEST INFRASTRUCTURE ONLY — the checker and the timed CPU reference arm, never the product.
 *
 * Compiles the reference's own construction engine, unmodified, from the GpuRecSplit source
 * tree: include/function/SIMDRecSplit.hpp together with AbstractParallelRecSplit.hpp,
 * RiceBitVector.hpp, DoubleEF.hpp, golombRiceMemo.hpp, support/common.hpp, util/Hash128.h,
 * util/Sorter.hpp and util/SimdUtils.hpp. Its third-party dependencies are absent from the
 * checkout (the extlib/ submodules are empty), so oracle/_ref_shim/ supplies project-written
 * stand-ins: vectorclass (AVX-512 subset), gcem (constexpr ceil/sqrt), sux::util::Vector and
 * a declaration of SpookyHash. The ips2ra sort behind bez::sorter::sortParallel_hash128_t
 * (src/Sorter.cpp:4-5) is replaced below by a parallel sort on the same key (`first`); the
 * order of keys inside a bucket does not change any seed.
 *
 * The library (oracle/_ref/libref_simdrs.so, built by oracle/Makefile) exports:
 *   ref_build      SIMDRecSplit<L, MALLOC, ROT>(vector<hash128_t>&, b, threads)
 *                  (SIMDRecSplit.hpp:228-232) and its operator<< (AbstractParallelRecSplit.hpp:480-488)
 *   ref_query      operator>> (:490-504) then operator()(hash128_t) (:409-466) per key
 *   ref_get_bits   getBits() (:476-478) of a deserialized function
 *   ref_object_size sizeof(SIMDRecSplit<L, MALLOC, ROT>)
 *   ref_encode     the reference's RiceBitVector::Builder (RiceBitVector.hpp:58-134) and
 *                  DoubleEF<MALLOC, true> (DoubleEF.hpp:140-365) driven with given seeds, in
 *                  the order compute_thread and the searches append them
 *                  (SIMDRecSplit.hpp:293-296,415-418,600-602,707-715,802-804), then operator<<
 * Only tests/, bench.py's reference arm / cpu_baseline and __graft_entry__.smoke() load it.
 */
#ifndef SIMD
#define SIMD
#endif
#include <function/SIMDRecSplit.hpp>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

// ---- stand-in for src/Sorter.cpp (ips2ra::parallel::sort by .first) --------------------
void bez::sorter::sortParallel_hash128_t(bez::function::hash128_t *objects, size_t n, size_t numThreads) {
    using bez::function::hash128_t;
    auto by_first = [](const hash128_t &a, const hash128_t &b) { return a.first < b.first; };
    size_t t = std::max<size_t>(1, std::min<size_t>(numThreads, 64));
    if (n < (size_t(1) << 16) || t == 1) {
        std::sort(objects, objects + n, by_first);
        return;
    }
    // Split by the top bits of `first` into t ranges of equal width, then sort each range.
    const int bits = 8;
    const size_t nbin = size_t(1) << bits;
    std::vector<size_t> count(nbin + 1, 0);
    for (size_t i = 0; i < n; i++) count[(objects[i].first >> (64 - bits)) + 1]++;
    for (size_t b = 0; b < nbin; b++) count[b + 1] += count[b];
    std::vector<hash128_t> tmp(objects, objects + n);
    std::vector<size_t> pos(count.begin(), count.end() - 1);
    for (size_t i = 0; i < n; i++) objects[pos[tmp[i].first >> (64 - bits)]++] = tmp[i];
    std::vector<std::thread> th;
    for (size_t k = 0; k < t; k++) {
        th.emplace_back([&, k] {
            for (size_t b = k; b < nbin; b += t) std::sort(objects + count[b], objects + count[b + 1], by_first);
        });
    }
    for (auto &x : th) x.join();
}

namespace {

using bez::function::hash128_t;
using bez::function::SIMDRecSplit;

struct Blob {
    std::string bytes;
};

// Exposes the reference's protected fields to drive its own encoders and stream operator.
template <size_t L, bool ROT> struct Encoded : public SIMDRecSplit<L, sux::util::AllocType::MALLOC, ROT> {
    using Base = SIMDRecSplit<L, sux::util::AllocType::MALLOC, ROT>;
    int encode(const uint64_t *bucket_keys, uint64_t nbuckets, uint64_t n, uint64_t bucket_size, const uint64_t *seeds,
               const uint32_t *sizes, uint64_t nseeds) {
        this->bucket_size = bucket_size;
        this->keys_count = n;
        this->nbuckets = nbuckets;
        std::vector<uint64_t> bucket_size_acc(nbuckets + 1), bucket_pos_acc(nbuckets + 1);
        bucket_size_acc[0] = 0;
        for (uint64_t i = 0; i < nbuckets; i++) bucket_size_acc[i + 1] = bucket_size_acc[i] + bucket_keys[i];
        if (bucket_size_acc[nbuckets] != n) return 1;
        static constexpr std::array<uint32_t, 3000> memo = bez::function::get_golomb_rice_memo(L);
        typename bez::function::RiceBitVector<sux::util::AllocType::MALLOC>::Builder builder;
        std::vector<uint32_t> unary;
        uint64_t k = 0;
        bucket_pos_acc[0] = 0;
        for (uint64_t i = 0; i < nbuckets; i++) {
            const uint64_t s = bucket_keys[i];
            if (s > 1) {
                // a bucket of s keys holds skip_nodes(s) nodes (golombRiceMemo.hpp)
                const uint64_t nodes = (memo[s] >> 16) & 0x7FF;
                if (k + nodes > nseeds || sizes[k] != s) return 2;
                for (uint64_t j = 0; j < nodes; j++, k++) {
                    const int log2golomb = memo[sizes[k]] >> 27;
                    builder.appendFixed(seeds[k], log2golomb);
                    unary.push_back(seeds[k] >> log2golomb);
                }
                builder.appendUnaryAll(unary);
                unary.clear();
            }
            bucket_pos_acc[i + 1] = builder.getBits();
        }
        if (k != nseeds) return 3;
        builder.appendFixed(1, 1);
        this->descriptors = builder.build();
        this->ef = bez::function::DoubleEF<sux::util::AllocType::MALLOC, true>(bucket_size_acc, bucket_pos_acc);
        return 0;
    }
};

template <size_t L, bool ROT> Blob *build(const uint64_t *keys128, uint64_t n, uint64_t b, int threads) {
    std::vector<hash128_t> keys;
    keys.reserve(n + 1);  // parallelPartition reads one element past the last key
    for (uint64_t i = 0; i < n; i++) keys.emplace_back(keys128[2 * i], keys128[2 * i + 1]);
    SIMDRecSplit<L, sux::util::AllocType::MALLOC, ROT> rs(keys, b, threads);
    std::ostringstream os;
    os << rs;
    return new Blob{os.str()};
}

template <size_t L, bool ROT> int query(const uint8_t *bytes, uint64_t len, const uint64_t *keys128, uint64_t n,
                                        uint64_t *out) {
    std::istringstream is(std::string(reinterpret_cast<const char *>(bytes), len));
    SIMDRecSplit<L, sux::util::AllocType::MALLOC, ROT> rs;
    uint64_t leaf = 0;
    if (len < 8) return 1;
    std::memcpy(&leaf, bytes, 8);
    if (leaf != L) return 1;  // operator>> abort()s on a mismatch
    is >> rs;
    if (!is) return 1;
    for (uint64_t i = 0; i < n; i++) out[i] = rs(hash128_t(keys128[2 * i], keys128[2 * i + 1]));
    return 0;
}

template <size_t L, bool ROT> uint64_t get_bits(const uint8_t *bytes, uint64_t len) {
    std::istringstream is(std::string(reinterpret_cast<const char *>(bytes), len));
    SIMDRecSplit<L, sux::util::AllocType::MALLOC, ROT> rs;
    is >> rs;
    return rs.getBits();
}

template <size_t L, bool ROT> Blob *encode(const uint64_t *bucket_keys, uint64_t nbuckets, uint64_t n, uint64_t b,
                                           const uint64_t *seeds, const uint32_t *sizes, uint64_t nseeds, int *err) {
    Encoded<L, ROT> e;
    *err = e.encode(bucket_keys, nbuckets, n, b, seeds, sizes, nseeds);
    if (*err) return nullptr;
    std::ostringstream os;
    os << static_cast<typename Encoded<L, ROT>::Base &>(e);
    return new Blob{os.str()};
}

template <template <size_t, bool> class F, typename R, typename... A> R dispatch(uint32_t leaf, int rot, R bad, A... a) {
#define RSB_REF_CASE(L)                                          \
    case L:                                                      \
        return rot ? F<L, true>::run(a...) : F<L, false>::run(a...);
    switch (leaf) {
        RSB_REF_CASE(2) RSB_REF_CASE(3) RSB_REF_CASE(4) RSB_REF_CASE(5) RSB_REF_CASE(6) RSB_REF_CASE(7)
        RSB_REF_CASE(8) RSB_REF_CASE(9) RSB_REF_CASE(10) RSB_REF_CASE(11) RSB_REF_CASE(12) RSB_REF_CASE(13)
        RSB_REF_CASE(14) RSB_REF_CASE(15) RSB_REF_CASE(16) RSB_REF_CASE(17) RSB_REF_CASE(18) RSB_REF_CASE(19)
        RSB_REF_CASE(20) RSB_REF_CASE(21) RSB_REF_CASE(22) RSB_REF_CASE(23) RSB_REF_CASE(24)
        default:
            return bad;
    }
#undef RSB_REF_CASE
}

template <size_t L, bool R> struct BuildF {
    static Blob *run(const uint64_t *k, uint64_t n, uint64_t b, int t) { return build<L, R>(k, n, b, t); }
};
template <size_t L, bool R> struct QueryF {
    static int run(const uint8_t *p, uint64_t len, const uint64_t *k, uint64_t n, uint64_t *o) {
        return query<L, R>(p, len, k, n, o);
    }
};
template <size_t L, bool R> struct BitsF {
    static uint64_t run(const uint8_t *p, uint64_t len) { return get_bits<L, R>(p, len); }
};
template <size_t L, bool R> struct SizeF {
    static uint64_t run() { return sizeof(SIMDRecSplit<L, sux::util::AllocType::MALLOC, R>); }
};
template <size_t L, bool R> struct EncodeF {
    static Blob *run(const uint64_t *bk, uint64_t nb, uint64_t n, uint64_t b, const uint64_t *s, const uint32_t *z,
                     uint64_t ns, int *err) {
        return encode<L, R>(bk, nb, n, b, s, z, ns, err);
    }
};

}  // namespace

extern "C" {

// Builds with the reference's SIMDRecSplit; returns a handle holding the serialized bytes.
void *ref_build(const uint64_t *keys128, uint64_t n, uint32_t leaf, uint64_t bucket_size, int rotate, int threads) {
    if (bucket_size == 0 || threads < 1) return nullptr;
    return dispatch<BuildF, Blob *>(leaf, rotate, nullptr, keys128, n, bucket_size, threads);
}

// Encodes given DFS seeds and node sizes with the reference's Builder and DoubleEF.
void *ref_encode(const uint64_t *bucket_keys, uint64_t nbuckets, uint64_t n, uint64_t bucket_size, uint32_t leaf,
                 int rotate, const uint64_t *seeds, const uint32_t *sizes, uint64_t nseeds, int *err) {
    *err = 0;
    if (nbuckets == 0) {
        *err = 4;
        return nullptr;
    }
    void *r = dispatch<EncodeF, Blob *>(leaf, rotate, nullptr, bucket_keys, nbuckets, n, bucket_size, seeds, sizes,
                                        nseeds, err);
    if (r == nullptr && *err == 0) *err = 5;
    return r;
}

uint64_t ref_blob_len(void *h) { return static_cast<Blob *>(h)->bytes.size(); }
void ref_blob_copy(void *h, void *dst) {
    const std::string &s = static_cast<Blob *>(h)->bytes;
    std::memcpy(dst, s.data(), s.size());
}
void ref_blob_free(void *h) { delete static_cast<Blob *>(h); }

// Deserializes with the reference's operator>> and evaluates operator() for every key.
int ref_query(const uint8_t *bytes, uint64_t len, uint32_t leaf, int rotate, const uint64_t *keys128, uint64_t n,
              uint64_t *out) {
    return dispatch<QueryF, int>(leaf, rotate, -1, bytes, len, keys128, n, out);
}

uint64_t ref_get_bits(const uint8_t *bytes, uint64_t len, uint32_t leaf, int rotate) {
    return dispatch<BitsF, uint64_t>(leaf, rotate, 0, bytes, len);
}

uint64_t ref_object_size(uint32_t leaf, int rotate) { return dispatch<SizeF, uint64_t>(leaf, rotate, 0); }

}  // extern "C"
