/*
 * TEST INFRASTRUCTURE ONLY — the checker, never the product.
 *
 * Scalar CPU restatement of the RecSplit construction path of ByteHamster/GpuRecSplit
 * as implemented by its SIMDRecSplit engine (the semantics GPURecSplit is tested against,
 * test/GPUandSIMDequivalence.cu:13-25). Only tests/, bench.py's cpu_baseline / reference
 * arm and __graft_entry__.smoke() load this library. The CUDA product in gpurecsplit_b200/
 * never links, loads or calls it.
 *
 * Parity pins for this restatement (the reference itself cannot be compiled in this
 * container: its sux, vectorclass, gcem, ips2ra and SpookyV2 submodules are empty):
 *   - the Golomb-Rice table generated here is checked against the reference's shipped
 *     table include/function/golombRiceMemo.hpp (digests in tests/golden/memo_digests.json);
 *   - every build is checked to be a bijection onto [0,n) through the restated query
 *     (test/recsplitCorrectness.hpp:10-35) over the reference's correctness grid;
 *   - bits/key is checked against the README's published values (README.md:16-23).
 *
 * Reference files cited below are paths within the GpuRecSplit project.
 */
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>
#ifdef ORC_SIMD
#include <immintrin.h>
#endif

namespace orc {

constexpr int kMaxBucketSize = 3000;  // AbstractParallelRecSplit.hpp:60
constexpr int kMaxLeafSize = 24;      // AbstractParallelRecSplit.hpp:62
constexpr int kMaxFanout = 9;         // AbstractParallelRecSplit.hpp:63

// AbstractParallelRecSplit.hpp:95-97
constexpr uint64_t kStartSeed[20] = {
    0x106393c187cae21a, 0x6453cec3f7376937, 0x643e521ddbd2be98, 0x3740c6412f6572cb, 0x717d47562f1ce470,
    0x4cd6eb4c63befb7c, 0x9bfd8c5e18c8da73, 0x082f20e10092a9a3, 0x2ada2ce68d21defc, 0xe33cb4f3e7c6466b,
    0x3980be458c509c59, 0xc466fd9584828e8c, 0x45f0aabe1a61ede6, 0xf6e7b8b33ad9b98d, 0x4ef95e25f4b4983d,
    0x81175195173b92d3, 0x4e50927d8dd15978, 0x1ea2099d1fafae7f, 0x425c8a06fbaaa815, 0xcd4216006c74052a};
constexpr int kNumStartSeeds = 20;

// AbstractParallelRecSplit.hpp:106
constexpr uint8_t kBijMemo[25] = {0, 0, 0, 1, 3, 4, 5, 7, 8, 10, 11, 12, 14, 15, 16, 18, 19, 21, 22, 23, 25, 26, 28, 29, 30};

enum Status { OK = 0, ERR_BAD_ARG = 1, ERR_DUPLICATE_KEY = 2, ERR_BUCKET_TOO_LARGE = 3, ERR_FORMAT = 4 };

struct Shape {
    uint32_t leaf, lower, upper;
};

// SplittingStrategy::lower_aggr / upper_aggr, AbstractParallelRecSplit.hpp:133,135.
// The upper expression is a double product in the reference (int * double ternary).
static Shape make_shape(uint32_t leaf) {
    Shape s;
    s.leaf = leaf;
    const double c = std::ceil(0.35 * leaf + 1. / 2);
    const int64_t f = std::max<int64_t>(2, (int64_t)c);
    s.lower = leaf * (uint32_t)f;
    const double u = leaf < 7 ? 2.0 : std::ceil(0.21 * leaf + 9. / 10);
    s.upper = (uint32_t)((double)s.lower * u);
    return s;
}

// SplittingStrategy::split_params, AbstractParallelRecSplit.hpp:137-148 (note the uint16_t casts).
static void split_params(const Shape &s, uint32_t m, uint32_t &fanout, uint32_t &unit) {
    if (m > s.upper) {
        unit = s.upper * (uint16_t(m / 2 + s.upper - 1) / s.upper);
        fanout = 2;
    } else if (m > s.lower) {
        unit = s.lower;
        fanout = uint16_t(m + s.lower - 1) / s.lower;
    } else {
        unit = s.leaf;
        fanout = uint16_t(m + s.leaf - 1) / s.leaf;
    }
}

// fill_golomb_rice / _fill_golomb_rice, AbstractParallelRecSplit.hpp:191-227.
// Bits 27-31: Rice parameter; bits 16-26: subtree node count; bits 0-15: subtree fixed-bit sum.
static void fill_memo(const Shape &s, uint32_t *memo) {
    uint32_t m = 0;
    for (; m <= s.leaf; ++m) memo[m] = uint32_t(kBijMemo[m]) << 27 | uint32_t(m > 1) << 16 | kBijMemo[m];
    for (; m < (uint32_t)kMaxBucketSize; ++m) {
        uint32_t fanout = 0, unit = 0;
        split_params(s, m, fanout, unit);
        int k[kMaxFanout] = {0};
        k[fanout - 1] = (int)m;
        for (uint32_t i = 0; i < fanout - 1; ++i) {
            k[i] = (int)unit;
            k[fanout - 1] -= k[i];
        }
        double sqrt_prod = 1;
        for (uint32_t i = 0; i < fanout; ++i) sqrt_prod *= std::sqrt((double)k[i]);
        const double p = std::sqrt((double)m) / (std::pow(2 * M_PI, (fanout - 1.) / 2) * sqrt_prod);
        uint32_t len = (uint32_t)std::ceil(std::log2(-std::log((std::sqrt(5.0) + 1) / 2) / std::log1p(-p)));
        memo[m] = len << 27;
        for (uint32_t i = 0; i < fanout; ++i) len += memo[k[i]] & 0xFFFF;
        memo[m] |= len;
        uint32_t nodes = 1;
        for (uint32_t i = 0; i < fanout; ++i) nodes += (memo[k[i]] >> 16) & 0x7FF;
        memo[m] |= nodes << 16;
    }
}

static inline uint32_t golomb_param(const uint32_t *memo, uint32_t m) { return memo[m] >> 27; }   // :251
static inline uint32_t skip_bits(const uint32_t *memo, uint32_t m) { return memo[m] & 0xFFFF; }    // :252
static inline uint32_t skip_nodes(const uint32_t *memo, uint32_t m) { return (memo[m] >> 16) & 0x7FF; }  // :253

// remix32, AbstractParallelRecSplit.hpp:277-284 (MurmurHash3 32-bit finalizer).
static inline uint32_t remix32(uint32_t z) {
    z ^= z >> 16;
    z *= 0x85ebca6b;
    z ^= z >> 13;
    z *= 0xc2b2ae35;
    z ^= z >> 16;
    return z;
}

// remixAndRemap with USE_64_BIT_REMAP=false, AbstractParallelRecSplit.hpp:327-337
// (identical to the SIMD remap, SIMDRecSplit.hpp:109-122, and GPURecSplit.cuh:82-87).
static inline uint32_t remap16(uint64_t x, uint32_t n) {
    return ((remix32(uint32_t(x >> 32) ^ uint32_t(x)) & 0xFFFFu) * n) >> 16;
}

// remap128, support/common.hpp:273-280.
static inline uint64_t remap128(uint64_t x, uint64_t n) { return (uint64_t)(((__uint128_t)x * (__uint128_t)n) >> 64); }

static inline int lambda64(uint64_t w) { return 63 ^ __builtin_clzll(w); }  // common.hpp:205
static inline int rho64(uint64_t w) { return __builtin_ctzll(w); }          // common.hpp:177
static inline int nu64(uint64_t w) { return __builtin_popcountll(w); }     // common.hpp:378-384
// select64, common.hpp:417-437: position of the k-th (0-based) one bit.
static inline uint64_t select64(uint64_t x, uint64_t k) {
    for (int i = 0; i < 64; ++i)
        if ((x >> i) & 1) {
            if (k == 0) return (uint64_t)i;
            --k;
        }
    return 64;
}

struct Stats {
    uint64_t evals_alg = 0;  // sum over nodes of (trials to the found seed) * node size
};

// ---------------------------------------------------------------------------------------
// Seed searches. Each returns the minimum x >= 0 (x counted from the level's start seed),
// which is what the vectorised loops of SIMDRecSplit.hpp find (lanes are consecutive
// seeds and the first successful lane wins, :268-286, :349-393, :475-509, :520-537).
// Early exits below only prune failing candidates; they never change the minimum.
// ---------------------------------------------------------------------------------------

#ifndef ORC_SIMD
namespace scalar {

// higherLevel, SIMDRecSplit.hpp:250-317: exactly `split` keys must remap below `split`.
static uint64_t search_higher(const uint64_t *keys, uint32_t m, uint32_t split, uint64_t seed) {
    for (uint64_t x = 0;; ++x) {
        const uint64_t sx = seed + x;
        uint32_t c0 = 0, c1 = 0;
        const uint32_t t1 = m - split;
        bool ok = true;
        for (uint32_t i = 0; i < m; ++i) {
            if (remap16(keys[i] + sx, m) < split) {
                if (++c0 > split) { ok = false; break; }
            } else if (++c1 > t1) {
                ok = false;
                break;
            }
        }
        if (ok) return x;
    }
}

// aggrLevel, SIMDRecSplit.hpp:319-423. The reference packs part counts into 8-bit lanes
// (the last part implicit for fanout 5 and 9); since every target is below 255 and a node
// holds at most fanout*SPLIT keys, a carry between lanes would need more keys than the
// node has, so packed equality is equivalent to the exact counts used here.
static uint64_t search_aggr(const uint64_t *keys, uint32_t m, uint32_t split, uint64_t seed) {
    const uint32_t fanout = uint16_t(m + split - 1) / split;
    uint32_t target[kMaxFanout];
    for (uint32_t i = 0; i + 1 < fanout; ++i) target[i] = split;
    target[fanout - 1] = m - (fanout - 1) * split;
    for (uint64_t x = 0;; ++x) {
        const uint64_t sx = seed + x;
        uint32_t count[kMaxFanout] = {0};
        bool ok = true;
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t part = remap16(keys[i] + sx, m) / split;
            if (++count[part] > target[part]) { ok = false; break; }
        }
        if (ok) return x;
    }
}

// leafLevel brute force, SIMDRecSplit.hpp:510-599 (midstop/backlog only prune).
static uint64_t search_leaf_bruteforce(const uint64_t *keys, uint32_t m, uint64_t seed) {
    for (uint64_t x = 0;; ++x) {
        const uint64_t sx = seed + x;
        uint32_t mask = 0;
        bool ok = true;
        for (uint32_t i = 0; i < m; ++i) {
            const uint32_t bit = 1u << remap16(keys[i] + sx, m);
            if (mask & bit) { ok = false; break; }
            mask |= bit;
        }
        if (ok) return x;
    }
}

static inline uint32_t rotl_leaf(uint32_t v, uint32_t r, uint32_t leaf) {
    const uint32_t full = (1u << leaf) - 1;
    return ((v << r) | (v >> (leaf - r))) & full;
}

// leafLevel with rotation fitting, SIMDRecSplit.hpp:452-509. Keys with even `second` form
// the left part, odd ones the right part. For bases x = SEED + leaf*k the encoded seed is
// leaf*k + r with r the smallest rotation for which maskL | rotl(maskR, r) is full (the
// reference rotates right by leaf-r, which is a left rotation by r, :437-439,:500-503).
static uint64_t search_leaf_rotate(const uint64_t *keys, uint32_t leaf, uint64_t seed) {
    uint64_t left[kMaxLeafSize], right[kMaxLeafSize];
    uint32_t nl = 0, nr = 0;
    for (uint32_t i = 0; i < leaf; ++i) {
        if (keys[i] % 2 == 0) left[nl++] = keys[i];
        else right[nr++] = keys[i];
    }
    const uint32_t full = (1u << leaf) - 1;
    for (uint64_t k = 0;; ++k) {
        const uint64_t base = seed + k * leaf;
        uint32_t ml = 0, mr = 0;
        bool ok = true;
        for (uint32_t i = 0; i < nl && ok; ++i) {
            const uint32_t bit = 1u << remap16(left[i] + base, leaf);
            if (ml & bit) ok = false;
            ml |= bit;
        }
        if (!ok) continue;  // a collision inside one part can never be completed by a rotation
        for (uint32_t i = 0; i < nr && ok; ++i) {
            const uint32_t bit = 1u << remap16(right[i] + base, leaf);
            if (mr & bit) ok = false;
            mr |= bit;
        }
        if (!ok) continue;
        for (uint32_t r = 0; r < leaf; ++r)
            if ((ml | rotl_leaf(mr, r, leaf)) == full) return k * leaf + r;
    }
}

}  // namespace scalar
namespace search = scalar;
#else
#include "simd_search.inc"
namespace search = simd;
#endif

// ---------------------------------------------------------------------------------------
// recSplit DFS, SIMDRecSplit.hpp:624-693. Seeds are recorded in DFS pre-order together
// with their node sizes; children are partitioned stably by part as in :288-306, :395-412.
// ---------------------------------------------------------------------------------------
struct BucketOut {
    std::vector<uint64_t> seeds;
    std::vector<uint32_t> sizes;
};

struct Ctx {
    Shape shape;
    bool rotate;
    const uint32_t *memo;
};

static void add_stat(Stats &st, uint64_t trials, uint32_t m) { st.evals_alg += trials * m; }

static void leaf_level(const Ctx &c, uint64_t *keys, uint32_t m, BucketOut &out, Stats &st) {
    const uint64_t seed = kStartSeed[kNumStartSeeds - 1];
    uint64_t x;
    if (c.rotate && m == c.shape.leaf) {
        x = search::search_leaf_rotate(keys, m, seed);
        add_stat(st, x / m + 1, m);
    } else {
        x = search::search_leaf_bruteforce(keys, m, seed);
        add_stat(st, x + 1, m);
    }
    out.seeds.push_back(x);
    out.sizes.push_back(m);
}

static void rec_split(const Ctx &c, uint64_t *keys, uint64_t *tmp, uint32_t m, int level, BucketOut &out, Stats &st) {
    const Shape &s = c.shape;
    if (m <= s.leaf) {
        leaf_level(c, keys, m, out, st);
        return;
    }
    if (m > s.upper) {  // fanout 2, SIMDRecSplit.hpp:631-635
        const uint32_t split = (uint16_t(m / 2 + s.upper - 1) / s.upper) * s.upper;
        const uint64_t seed = kStartSeed[level];
        const uint64_t x = search::search_higher(keys, m, split, seed);
        add_stat(st, x + 1, m);
        out.seeds.push_back(x);
        out.sizes.push_back(m);
        uint32_t c0 = 0, c1 = split;
        for (uint32_t i = 0; i < m; ++i) tmp[remap16(keys[i] + seed + x, m) < split ? c0++ : c1++] = keys[i];
        std::memcpy(keys, tmp, m * sizeof(uint64_t));
        rec_split(c, keys, tmp, split, level + 1, out, st);
        if (m - split > 1) rec_split(c, keys + split, tmp, m - split, level + 1, out, st);
        return;
    }
    const bool upper_level = m > s.lower;  // :640 (second aggregation level) vs :651
    const uint32_t split = upper_level ? s.lower : s.leaf;
    const uint64_t seed = kStartSeed[kNumStartSeeds - (upper_level ? 3 : 2)];
    const uint64_t x = search::search_aggr(keys, m, split, seed);
    add_stat(st, x + 1, m);
    out.seeds.push_back(x);
    out.sizes.push_back(m);
    const uint32_t fanout = uint16_t(m + split - 1) / split;
    uint32_t cur[kMaxFanout];
    for (uint32_t i = 0; i < fanout; ++i) cur[i] = i * split;
    for (uint32_t i = 0; i < m; ++i) tmp[cur[remap16(keys[i] + seed + x, m) / split]++] = keys[i];
    std::memcpy(keys, tmp, m * sizeof(uint64_t));
    uint32_t i;
    for (i = 0; i < m - split; i += split) rec_split(c, keys + i, tmp, split, level + 1, out, st);
    if (m - i > 1) rec_split(c, keys + i, tmp, m - i, level + 1, out, st);
}

// ---------------------------------------------------------------------------------------
// RiceBitVector::Builder, RiceBitVector.hpp:58-134. The word array is resized on every
// append to ((ceil(bits/8)) + 7 + 7) / 8 words, so the final length is set by the sentinel.
// ---------------------------------------------------------------------------------------
struct RiceBuilder {
    std::vector<uint64_t> data = std::vector<uint64_t>(16, 0);
    uint64_t bit_count = 0;

    static size_t words_for(uint64_t bits) { return (((bits + 7) / 8) + 7 + 7) / 8; }
    void resize(size_t words) { data.resize(words, 0); }

    void append_fixed(uint64_t v, int log2golomb) {  // :73-90
        const uint64_t lower = v & ((uint64_t(1) << log2golomb) - 1);
        int used = bit_count & 63;
        resize(words_for(bit_count + log2golomb));
        uint64_t *p = data.data() + bit_count / 64;
        uint64_t cur = *p;
        cur |= lower << used;
        if (used + log2golomb > 64) {
            *(p++) = cur;
            cur = lower >> (64 - used);
        }
        *p = cur;
        bit_count += log2golomb;
    }

    void append_unary_all(const std::vector<uint32_t> &unary) {  // :92-106
        uint64_t inc = 0;
        for (uint32_t u : unary) inc += uint64_t(u) + 1;
        resize(words_for(bit_count + inc));
        for (uint32_t u : unary) {
            bit_count += u;
            data[bit_count / 64] |= uint64_t(1) << (bit_count & 63);
            ++bit_count;
        }
    }
};

// ---------------------------------------------------------------------------------------
// DoubleEF<AT, true> constructor, DoubleEF.hpp:140-365 (scalar loops :173-179, :274-281;
// FAST_CONSTRUCTION jump table :286-320, equivalent to the slow loop :321-349). Entries of
// the jump table that fall outside jump_size_words() (:90-94) are not part of the output.
// ---------------------------------------------------------------------------------------
struct DoubleEF {
    static constexpr uint64_t log2q = 8, q = 1 << log2q, q_mask = q - 1;
    static constexpr uint64_t super_q = 1 << 14, super_q_mask = super_q - 1;
    static constexpr uint64_t q_per_super_q = super_q / q, super_q_size = 1 + q_per_super_q / 4;
    std::vector<uint64_t> lower_bits, upper_bits_position, upper_bits_cum_keys, jump;
    uint64_t lower_bits_mask_cum_keys = 0, lower_bits_mask_position = 0;
    uint64_t num_buckets = 0, u_cum_keys = 0, u_position = 0;
    uint64_t l_position = 0, l_cum_keys = 0;
    int64_t cum_keys_min_delta = 0, min_diff = 0;
    uint64_t bits_per_key_fixed_point = 0;

    size_t lower_bits_size_words() const { return ((num_buckets + 1) * (l_cum_keys + l_position) + 63) / 64 + 1; }
    size_t cum_keys_size_words() const { return (num_buckets + 1 + (u_cum_keys >> l_cum_keys) + 63) / 64; }
    size_t position_size_words() const { return (num_buckets + 1 + (u_position >> l_position) + 63) / 64; }
    size_t jump_size_words() const {
        size_t size = (num_buckets / super_q) * super_q_size * 2;
        if (num_buckets % super_q != 0) size += (1 + ((num_buckets % super_q + q - 1) / q + 3) / 4) * 2;
        return size;
    }

    static void set_bit(std::vector<uint64_t> &bits, uint64_t pos) { bits[pos / 64] |= uint64_t(1) << (pos % 64); }
    // set_bits, DoubleEF.hpp:80-86: an unaligned 8-byte read-modify-write at byte start/8.
    static void set_bits(std::vector<uint64_t> &bits, uint64_t start, int width, uint64_t value) {
        const uint64_t mask = ((uint64_t(1) << width) - 1) << (start % 8);
        uint64_t t;
        uint8_t *base = (uint8_t *)bits.data() + start / 8;
        std::memcpy(&t, base, 8);
        t = (t & ~mask) | value << (start % 8);
        std::memcpy(base, &t, 8);
    }

    void build(const std::vector<uint64_t> &cum_keys, const std::vector<uint64_t> &position) {
        num_buckets = cum_keys.size() - 1;
        // :144 — the one floating-point operation of the path (IEEE double, round to nearest).
        // With no keys this is 0/0; the reference's x86-64 build converts that NaN to 0x8000000000000000.
        bits_per_key_fixed_point = cum_keys[num_buckets] == 0 ? (uint64_t(1) << 63)
            : (uint64_t)((double)(uint64_t(1) << 20) * (position[num_buckets] / (double)cum_keys[num_buckets]));
        min_diff = INT64_MAX / 2;
        cum_keys_min_delta = INT64_MAX / 2;
        int64_t prev_bucket_bits = 0;
        for (uint64_t i = 1; i <= num_buckets; ++i) {
            const int64_t nkeys_delta = cum_keys[i] - cum_keys[i - 1];
            cum_keys_min_delta = std::min(cum_keys_min_delta, nkeys_delta);
            const int64_t bucket_bits = int64_t(position[i]) - int64_t(bits_per_key_fixed_point * cum_keys[i] >> 20);
            min_diff = std::min(min_diff, bucket_bits - prev_bucket_bits);
            prev_bucket_bits = bucket_bits;
        }
        u_position = int64_t(position[num_buckets]) - int64_t(bits_per_key_fixed_point * cum_keys[num_buckets] >> 20) -
                     int64_t(num_buckets * min_diff) + 1;
        l_position = u_position / (num_buckets + 1) == 0 ? 0 : lambda64(u_position / (num_buckets + 1));
        u_cum_keys = cum_keys[num_buckets] - num_buckets * cum_keys_min_delta + 1;
        l_cum_keys = u_cum_keys / (num_buckets + 1) == 0 ? 0 : lambda64(u_cum_keys / (num_buckets + 1));
        lower_bits_mask_cum_keys = (uint64_t(1) << l_cum_keys) - 1;
        lower_bits_mask_position = (uint64_t(1) << l_position) - 1;

        lower_bits.assign(lower_bits_size_words(), 0);
        upper_bits_cum_keys.assign(cum_keys_size_words(), 0);
        upper_bits_position.assign(position_size_words(), 0);

        uint64_t cum_delta = 0, bit_delta = 0;
        for (uint64_t i = 0; i <= num_buckets; i++, cum_delta += cum_keys_min_delta, bit_delta += min_diff) {
            if (l_cum_keys != 0)
                set_bits(lower_bits, i * (l_cum_keys + l_position), (int)l_cum_keys, (cum_keys[i] - cum_delta) & lower_bits_mask_cum_keys);
            set_bit(upper_bits_cum_keys, ((cum_keys[i] - cum_delta) >> l_cum_keys) + i);
            const int64_t pval = int64_t(position[i]) - int64_t(bits_per_key_fixed_point * cum_keys[i] >> 20);
            if (l_position != 0)
                set_bits(lower_bits, i * (l_cum_keys + l_position) + l_cum_keys, (int)l_position, (pval - bit_delta) & lower_bits_mask_position);
            set_bit(upper_bits_position, ((pval - bit_delta) >> l_position) + i);
        }

        jump.assign(jump_size_words(), 0);
        fill_jump(upper_bits_cum_keys, 0);
        fill_jump(upper_bits_position, 1);
    }

    // Jump entries for every q-th one: an absolute position every super_q ones and a 16-bit
    // offset from it every q ones (DoubleEF.hpp:288-320).
    void fill_jump(const std::vector<uint64_t> &bits, int which) {
        uint64_t c = 0, last_super_q = 0;
        for (uint64_t i = 0; i < bits.size(); i++) {
            for (int b = 0; b < 64; b++) {
                if (!(bits[i] >> b & 1)) continue;
                const uint64_t pos = i * 64 + b;
                const uint64_t block = (c / super_q) * (super_q_size * 2);
                if ((c & super_q_mask) == 0) {
                    last_super_q = pos;
                    if (block + which < jump.size()) jump[block + which] = pos;
                }
                if ((c & q_mask) == 0) {
                    const uint64_t slot = 2 * ((c & super_q_mask) / q) + which;  // uint16 index after 2 words
                    const uint64_t word = block + 2 + slot / 4;
                    if (word < jump.size()) {
                        uint16_t *p = (uint16_t *)(jump.data() + block + 2);
                        p[slot] = (uint16_t)(pos - last_super_q);
                    }
                }
                c++;
            }
        }
    }

    // get(i, cum_keys, cum_keys_next, position), DoubleEF.hpp:367-402.
    void get(uint64_t i, uint64_t &cum_keys, uint64_t &cum_keys_next, uint64_t &position) const {
        const uint64_t pos_lower = i * (l_cum_keys + l_position);
        uint64_t lower;
        std::memcpy(&lower, (const uint8_t *)lower_bits.data() + pos_lower / 8, 8);
        lower >>= pos_lower % 8;
        const uint64_t jump_super_q = (i / super_q) * super_q_size * 2;
        const uint64_t jump_inside_super_q = (i % super_q) / q;
        const uint16_t *j16 = (const uint16_t *)(jump.data() + jump_super_q + 2);
        const uint64_t jump_cum_keys = jump[jump_super_q] + j16[2 * jump_inside_super_q];
        const uint64_t jump_position = jump[jump_super_q + 1] + j16[2 * jump_inside_super_q + 1];
        uint64_t curr_word_cum_keys = jump_cum_keys / 64;
        uint64_t curr_word_position = jump_position / 64;
        uint64_t window_cum_keys = upper_bits_cum_keys[curr_word_cum_keys] & UINT64_C(-1) << jump_cum_keys % 64;
        uint64_t window_position = upper_bits_position[curr_word_position] & UINT64_C(-1) << jump_position % 64;
        uint64_t delta_cum_keys = i & q_mask;
        uint64_t delta_position = i & q_mask;
        for (uint64_t bc; (bc = nu64(window_cum_keys)) <= delta_cum_keys; delta_cum_keys -= bc)
            window_cum_keys = upper_bits_cum_keys[++curr_word_cum_keys];
        for (uint64_t bc; (bc = nu64(window_position)) <= delta_position; delta_position -= bc)
            window_position = upper_bits_position[++curr_word_position];
        const uint64_t select_cum_keys = select64(window_cum_keys, delta_cum_keys);
        const int64_t cum_delta = i * cum_keys_min_delta;
        cum_keys = ((curr_word_cum_keys * 64 + select_cum_keys - i) << l_cum_keys | (lower & lower_bits_mask_cum_keys)) + cum_delta;
        lower >>= l_cum_keys;
        const int64_t bit_delta = i * min_diff;
        position = ((curr_word_position * 64 + select64(window_position, delta_position) - i) << l_position |
                    (lower & lower_bits_mask_position)) +
                   bit_delta + int64_t(bits_per_key_fixed_point * cum_keys >> 20);
        window_cum_keys &= (-1ULL << select_cum_keys) << 1;
        while (window_cum_keys == 0) window_cum_keys = upper_bits_cum_keys[++curr_word_cum_keys];
        lower >>= l_position;
        cum_keys_next = ((curr_word_cum_keys * 64 + rho64(window_cum_keys) - i - 1) << l_cum_keys | (lower & lower_bits_mask_cum_keys)) +
                        cum_delta + cum_keys_min_delta;
    }
};

// ---------------------------------------------------------------------------------------
// Byte stream helpers. Serialized layout, AbstractParallelRecSplit.hpp:480-488 and
// DoubleEF.hpp:100-113; a word vector is a uint64 element count followed by the words.
// ---------------------------------------------------------------------------------------
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
struct Reader {
    const uint8_t *p, *end;
    bool ok = true;
    uint64_t get64() {
        if (end - p < 8) { ok = false; return 0; }
        uint64_t v;
        std::memcpy(&v, p, 8);
        p += 8;
        return v;
    }
    std::vector<uint64_t> get_vec() {
        const uint64_t n = get64();
        std::vector<uint64_t> v;
        if (!ok || (uint64_t)(end - p) / 8 < n) { ok = false; return v; }
        v.resize(n);
        std::memcpy(v.data(), p, n * 8);
        p += n * 8;
        return v;
    }
};

struct Mphf {
    uint32_t leaf = 0;
    uint64_t bucket_size = 0, keys_count = 0, nbuckets = 0;
    std::vector<uint64_t> descriptors;
    DoubleEF ef;
    std::vector<uint32_t> memo;
    Shape shape{};
    bool rotate = true;
};

// Builds the MPHF. `keys` is n (first, second) pairs. Buckets are searched by `threads`
// worker threads (contiguous bucket ranges as in compute_thread, SIMDRecSplit.hpp:695-745);
// the per-bucket outputs are then concatenated in bucket order, which is what the ordered
// builder merge of the reference produces.
struct BuildResult {
    std::vector<uint8_t> bytes;
    std::vector<uint64_t> seeds;     // all nodes, bucket order, DFS pre-order inside a bucket
    std::vector<uint32_t> sizes;     // node size for each seed
    std::vector<uint64_t> bucket_size_acc, bucket_pos_acc;
    Stats stats;
    Mphf mphf;
};

static int partition_keys(const uint64_t *keys, uint64_t n, uint64_t nbuckets, std::vector<uint64_t> &sorted,
                          std::vector<uint64_t> &acc) {
    // parallelPartition, AbstractParallelRecSplit.hpp:339-359: bucket = remap128(first, nbuckets),
    // keys grouped by bucket; the order inside a bucket does not affect any seed.
    acc.assign(nbuckets + 1, 0);
    for (uint64_t i = 0; i < n; ++i) acc[remap128(keys[2 * i], nbuckets) + 1]++;
    for (uint64_t b = 0; b < nbuckets; ++b) acc[b + 1] += acc[b];
    std::vector<uint64_t> cur(acc.begin(), acc.end() - 1);
    sorted.assign(n, 0);
    for (uint64_t i = 0; i < n; ++i) sorted[cur[remap128(keys[2 * i], nbuckets)]++] = keys[2 * i + 1];
    return OK;
}

static int check_bucket(uint64_t *b, uint64_t m) {
    if (m >= (uint64_t)kMaxBucketSize) return ERR_BUCKET_TOO_LARGE;
    std::vector<uint64_t> t(b, b + m);
    std::sort(t.begin(), t.end());
    for (uint64_t i = 1; i < m; ++i)
        if (t[i] == t[i - 1]) return ERR_DUPLICATE_KEY;  // would make the reference search forever
    return OK;
}

static int build(const uint64_t *keys, uint64_t n, uint32_t leaf, uint64_t bucket_size, bool rotate, int threads,
                 const uint64_t *bucket_subset, uint64_t subset_n, BuildResult &R) {
    if (leaf < 2 || leaf > (uint32_t)kMaxLeafSize || bucket_size == 0) return ERR_BAD_ARG;
    Mphf &M = R.mphf;
    M.leaf = leaf;
    M.shape = make_shape(leaf);
    M.rotate = rotate;
    M.memo.assign(kMaxBucketSize, 0);
    fill_memo(M.shape, M.memo.data());
    M.bucket_size = bucket_size;
    M.keys_count = n;
    M.nbuckets = std::max<uint64_t>(1, (n + bucket_size - 1) / bucket_size);  // SIMDRecSplit.hpp:774
    std::vector<uint64_t> sorted;
    partition_keys(keys, n, M.nbuckets, sorted, R.bucket_size_acc);
    const uint64_t nb = M.nbuckets;
    for (uint64_t b = 0; b < nb; ++b) {
        int st = check_bucket(sorted.data() + R.bucket_size_acc[b], R.bucket_size_acc[b + 1] - R.bucket_size_acc[b]);
        if (st != OK) return st;
    }
    // Which buckets to search: all, or a subset (sampled parity checks at full size).
    std::vector<uint64_t> todo;
    if (bucket_subset) todo.assign(bucket_subset, bucket_subset + subset_n);
    else {
        todo.resize(nb);
        for (uint64_t b = 0; b < nb; ++b) todo[b] = b;
    }
    std::vector<BucketOut> outs(todo.size());
    std::vector<Stats> stats(std::max(1, threads));
    Ctx ctx{M.shape, rotate, M.memo.data()};
    std::atomic<uint64_t> next{0};
    auto worker = [&](int tid) {
        std::vector<uint64_t> tmp(kMaxBucketSize);
        for (;;) {
            const uint64_t j = next.fetch_add(1);
            if (j >= todo.size()) break;
            const uint64_t b = todo[j];
            const uint64_t m = R.bucket_size_acc[b + 1] - R.bucket_size_acc[b];
            if (m > 1) rec_split(ctx, sorted.data() + R.bucket_size_acc[b], tmp.data(), (uint32_t)m, 0, outs[j], stats[tid]);
        }
    };
    if (threads <= 1) worker(0);
    else {
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; ++t) ts.emplace_back(worker, t);
        for (auto &t : ts) t.join();
    }
    for (auto &s : stats) R.stats.evals_alg += s.evals_alg;
    for (auto &o : outs) {
        R.seeds.insert(R.seeds.end(), o.seeds.begin(), o.seeds.end());
        R.sizes.insert(R.sizes.end(), o.sizes.begin(), o.sizes.end());
    }
    if (bucket_subset) return OK;  // no encoding for a partial build

    // Encoding: per bucket, fixed parts in DFS order then unary parts (SIMDRecSplit.hpp:308-311,
    // :709-714); x >> g is held as uint32 in the reference's unary vector.
    RiceBuilder builder;
    R.bucket_pos_acc.assign(nb + 1, 0);
    std::vector<uint32_t> unary;
    for (uint64_t b = 0; b < nb; ++b) {
        const BucketOut &o = outs[b];
        if (!o.seeds.empty()) {
            unary.clear();
            for (size_t k = 0; k < o.seeds.size(); ++k) {
                const uint32_t g = golomb_param(M.memo.data(), o.sizes[k]);
                builder.append_fixed(o.seeds[k], (int)g);
                unary.push_back((uint32_t)(o.seeds[k] >> g));
            }
            builder.append_unary_all(unary);
        }
        R.bucket_pos_acc[b + 1] = builder.bit_count;
    }
    builder.append_fixed(1, 1);  // sentinel, SIMDRecSplit.hpp:810
    M.descriptors = builder.data;
    M.ef.build(R.bucket_size_acc, R.bucket_pos_acc);

    std::vector<uint8_t> &o = R.bytes;
    put64(o, leaf);
    put64(o, bucket_size);
    put64(o, n);
    put_vec(o, M.descriptors);
    put64(o, M.ef.num_buckets);
    put64(o, M.ef.u_cum_keys);
    put64(o, M.ef.u_position);
    put64(o, (uint64_t)M.ef.cum_keys_min_delta);
    put64(o, (uint64_t)M.ef.min_diff);
    put64(o, M.ef.bits_per_key_fixed_point);
    put_vec(o, M.ef.lower_bits);
    put_vec(o, M.ef.upper_bits_cum_keys);
    put_vec(o, M.ef.upper_bits_position);
    put_vec(o, M.ef.jump);
    return OK;
}

// operator>>, AbstractParallelRecSplit.hpp:490-504 and DoubleEF.hpp:115-135.
static int deserialize(const uint8_t *p, size_t len, bool rotate, Mphf &M) {
    Reader r{p, p + len};
    M.leaf = (uint32_t)r.get64();
    M.bucket_size = r.get64();
    M.keys_count = r.get64();
    if (!r.ok || M.leaf < 2 || M.leaf > (uint32_t)kMaxLeafSize || M.bucket_size == 0) return ERR_FORMAT;
    M.nbuckets = std::max<uint64_t>(1, (M.keys_count + M.bucket_size - 1) / M.bucket_size);
    M.descriptors = r.get_vec();
    DoubleEF &e = M.ef;
    e.num_buckets = r.get64();
    e.u_cum_keys = r.get64();
    e.u_position = r.get64();
    e.cum_keys_min_delta = (int64_t)r.get64();
    e.min_diff = (int64_t)r.get64();
    e.bits_per_key_fixed_point = r.get64();
    e.l_position = e.u_position / (e.num_buckets + 1) == 0 ? 0 : lambda64(e.u_position / (e.num_buckets + 1));
    e.l_cum_keys = e.u_cum_keys / (e.num_buckets + 1) == 0 ? 0 : lambda64(e.u_cum_keys / (e.num_buckets + 1));
    e.lower_bits_mask_cum_keys = (uint64_t(1) << e.l_cum_keys) - 1;
    e.lower_bits_mask_position = (uint64_t(1) << e.l_position) - 1;
    e.lower_bits = r.get_vec();
    e.upper_bits_cum_keys = r.get_vec();
    e.upper_bits_position = r.get_vec();
    e.jump = r.get_vec();
    if (!r.ok) return ERR_FORMAT;
    M.shape = make_shape(M.leaf);
    M.memo.assign(kMaxBucketSize, 0);
    fill_memo(M.shape, M.memo.data());
    M.rotate = rotate;
    return OK;
}

// RiceBitVector::Reader, RiceBitVector.hpp:150-218.
struct RiceReader {
    const std::vector<uint64_t> &data;
    uint64_t curr_fixed_offset = 0, curr_window_unary = 0;
    size_t curr_ptr_unary = 0;
    int valid_lower_bits_unary = 0;
    explicit RiceReader(const std::vector<uint64_t> &d) : data(d) {}
    uint64_t word(size_t i) const { return i < data.size() ? data[i] : 0; }
    uint64_t read_next(int log2golomb) {
        uint64_t result = 0;
        if (curr_window_unary == 0) {
            result += valid_lower_bits_unary;
            curr_window_unary = word(curr_ptr_unary++);
            valid_lower_bits_unary = 64;
            while (curr_window_unary == 0) {
                result += 64;
                curr_window_unary = word(curr_ptr_unary++);
            }
        }
        const int pos = rho64(curr_window_unary);
        curr_window_unary >>= pos;
        curr_window_unary >>= 1;
        valid_lower_bits_unary -= pos + 1;
        result += pos;
        result <<= log2golomb;
        uint64_t fixed = 0;
        const size_t byte = curr_fixed_offset / 8;
        const uint8_t *bytes = (const uint8_t *)data.data();
        const size_t nbytes = data.size() * 8;
        for (int k = 0; k < 8 && byte + k < nbytes; ++k) fixed |= uint64_t(bytes[byte + k]) << (8 * k);
        result |= (fixed >> curr_fixed_offset % 8) & ((uint64_t(1) << log2golomb) - 1);
        curr_fixed_offset += log2golomb;
        return result;
    }
    void skip_subtree(size_t nodes, size_t fixed_len) {
        size_t missing = nodes, cnt;
        while ((cnt = nu64(curr_window_unary)) < missing) {
            curr_window_unary = word(curr_ptr_unary++);
            missing -= cnt;
            valid_lower_bits_unary = 64;
        }
        cnt = select64(curr_window_unary, missing - 1);
        curr_window_unary >>= cnt;
        curr_window_unary >>= 1;
        valid_lower_bits_unary -= (int)cnt + 1;
        curr_fixed_offset += fixed_len;
    }
    void read_reset(size_t bit_pos, size_t unary_offset) {
        curr_fixed_offset = bit_pos;
        const size_t unary_pos = bit_pos + unary_offset;
        curr_ptr_unary = unary_pos / 64;
        curr_window_unary = word(curr_ptr_unary++) >> (unary_pos & 63);
        valid_lower_bits_unary = 64 - (unary_pos & 63);
    }
};

// operator()(hash128_t), AbstractParallelRecSplit.hpp:409-466.
static uint64_t query(const Mphf &M, uint64_t first, uint64_t second) {
    const uint32_t *memo = M.memo.data();
    const Shape &s = M.shape;
    const uint64_t bucket = remap128(first, M.nbuckets);
    uint64_t cum_keys, cum_keys_next, bit_pos;
    M.ef.get(bucket, cum_keys, cum_keys_next, bit_pos);
    uint64_t m = cum_keys_next - cum_keys;
    RiceReader reader(M.descriptors);
    reader.read_reset(bit_pos, skip_bits(memo, (uint32_t)m));
    int level = 0;
    while (m > s.upper) {
        const uint64_t d = reader.read_next((int)golomb_param(memo, (uint32_t)m));
        const uint64_t hmod = remap16(second + d + kStartSeed[level], (uint32_t)m);
        const uint32_t split = ((uint16_t(m / 2 + s.upper - 1) / s.upper)) * s.upper;
        if (hmod < split) {
            m = split;
        } else {
            reader.skip_subtree(skip_nodes(memo, split), skip_bits(memo, split));
            m -= split;
            cum_keys += split;
        }
        level++;
    }
    if (m > s.lower) {
        const uint64_t d = reader.read_next((int)golomb_param(memo, (uint32_t)m));
        const uint64_t hmod = remap16(second + d + kStartSeed[kNumStartSeeds - 3], (uint32_t)m);
        const int part = uint16_t(hmod) / s.lower;
        m = std::min<uint64_t>(s.lower, m - part * s.lower);
        cum_keys += s.lower * part;
        if (part) reader.skip_subtree(skip_nodes(memo, s.lower) * part, skip_bits(memo, s.lower) * part);
    }
    if (m > s.leaf) {
        const uint64_t d = reader.read_next((int)golomb_param(memo, (uint32_t)m));
        const uint64_t hmod = remap16(second + d + kStartSeed[kNumStartSeeds - 2], (uint32_t)m);
        const int part = uint16_t(hmod) / s.leaf;
        m = std::min<uint64_t>(s.leaf, m - part * s.leaf);
        cum_keys += s.leaf * part;
        if (part) reader.skip_subtree(part, skip_bits(memo, s.leaf) * part);
    }
    const uint64_t b = reader.read_next((int)golomb_param(memo, (uint32_t)m));
    const uint64_t x = second + b + kStartSeed[kNumStartSeeds - 1];
    uint64_t leaf_val;
    if (M.rotate && m == s.leaf) {
        const uint64_t rotation = b % s.leaf;
        leaf_val = remap16(x - rotation, s.leaf);
        if (second % 2 != 0) leaf_val = (leaf_val + rotation) % s.leaf;
    } else {
        leaf_val = remap16(x, (uint32_t)m);
    }
    return cum_keys + leaf_val;
}

// ---------------------------------------------------------------------------------------
// Input generators shared by tests and benchmarks (project definitions, not reference code).
// splitmix64 (Steele, Lea, Flood 2014) drives every synthetic input.
// ---------------------------------------------------------------------------------------
static inline uint64_t splitmix64(uint64_t &state) {
    uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
// Project 64->128-bit key mixer: first = MurmurHash3 fmix64(k), second = Stafford variant 13
// (the splitmix64 finalizer) of k + golden ratio. Both halves are bijections of k, so distinct
// 64-bit keys give distinct `second` halves and can never collide inside a bucket.
static inline uint64_t fmix64(uint64_t k) {
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}
static inline uint64_t stafford13(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// SpookyHash V2 128-bit (Bob Jenkins, public domain), restated from the published algorithm.
// The reference hashes string keys with spooky(key, len, 0) and returns {h1, h0}
// (util/Hash128.h:32-36). No golden vectors exist in the reference or this container,
// so agreement with upstream string hashing is unpinned.
namespace spooky {
constexpr uint64_t kConst = 0xdeadbeefdeadbeefULL;
static inline uint64_t rot(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static inline uint64_t load64(const uint8_t *p) { uint64_t v; std::memcpy(&v, p, 8); return v; }
static inline uint32_t load32(const uint8_t *p) { uint32_t v; std::memcpy(&v, p, 4); return v; }

static inline void short_mix(uint64_t &a, uint64_t &b, uint64_t &c, uint64_t &d) {
    static const int r[12] = {50, 52, 30, 41, 54, 48, 38, 37, 62, 34, 5, 36};
    uint64_t *h[4] = {&a, &b, &c, &d};
    for (int i = 0; i < 12; ++i) {
        // step i rotates h[(i+2)%4], adds h[(i+3)%4] to it, and xors the result into h[i%4]
        uint64_t &x = *h[(i + 2) % 4];
        x = rot(x, r[i]);
        x += *h[(i + 3) % 4];
        *h[i % 4] ^= x;
    }
}
static inline void short_end(uint64_t &a, uint64_t &b, uint64_t &c, uint64_t &d) {
    static const int r[11] = {15, 52, 26, 51, 28, 9, 47, 54, 32, 25, 63};
    uint64_t *h[4] = {&a, &b, &c, &d};
    for (int i = 0; i < 11; ++i) {
        // step i: h[(i+3)%4] ^= h[(i+2)%4]; h[(i+2)%4] = rot(h[(i+2)%4], r); h[(i+3)%4] += h[(i+2)%4]
        uint64_t &y = *h[(i + 3) % 4];
        uint64_t &x = *h[(i + 2) % 4];
        y ^= x;
        x = rot(x, r[i]);
        y += x;
    }
}
static void short_hash(const uint8_t *msg, size_t len, uint64_t &h1, uint64_t &h2) {
    uint64_t a = h1, b = h2, c = kConst, d = kConst;
    size_t rem = len % 32;
    const uint8_t *p = msg;
    if (len > 15) {
        const uint8_t *end = msg + (len / 32) * 32;
        for (; p < end; p += 32) {
            c += load64(p);
            d += load64(p + 8);
            short_mix(a, b, c, d);
            a += load64(p + 16);
            b += load64(p + 24);
        }
        if (rem >= 16) {
            c += load64(p);
            d += load64(p + 8);
            short_mix(a, b, c, d);
            p += 16;
            rem -= 16;
        }
    }
    d += uint64_t(len) << 56;
    // tail of 0..15 bytes: bytes 0..7 go to c, bytes 8..14 to d (little endian)
    if (rem == 0) {
        c += kConst;
        d += kConst;
    } else {
        uint64_t lo = 0, hi = 0;
        for (size_t k = 0; k < rem && k < 8; ++k) lo |= uint64_t(p[k]) << (8 * k);
        for (size_t k = 8; k < rem; ++k) hi |= uint64_t(p[k]) << (8 * (k - 8));
        c += lo;
        d += hi;
    }
    short_end(a, b, c, d);
    h1 = a;
    h2 = b;
}
static inline void mix(const uint64_t *data, uint64_t *s) {
    static const int r[12] = {11, 32, 43, 31, 17, 28, 39, 57, 55, 54, 22, 46};
    for (int i = 0; i < 12; ++i) {
        s[i] += data[i];
        s[(i + 2) % 12] ^= s[(i + 10) % 12];
        s[(i + 11) % 12] ^= s[i];
        s[i] = rot(s[i], r[i]);
        s[(i + 11) % 12] += s[(i + 1) % 12];
    }
}
static inline void end_partial(uint64_t *h) {
    static const int r[12] = {44, 15, 34, 21, 38, 33, 10, 13, 38, 53, 42, 54};
    for (int i = 0; i < 12; ++i) {
        h[(i + 11) % 12] += h[(i + 1) % 12];
        h[(i + 2) % 12] ^= h[(i + 11) % 12];
        h[(i + 1) % 12] = rot(h[(i + 1) % 12], r[i]);
    }
}
static void hash128(const uint8_t *msg, size_t len, uint64_t &h1, uint64_t &h2) {
    if (len < 192) {
        short_hash(msg, len, h1, h2);
        return;
    }
    uint64_t h[12];
    for (int i = 0; i < 12; i += 3) {
        h[i] = h1;
        h[i + 1] = h2;
        h[i + 2] = kConst;
    }
    const size_t blocks = len / 96;
    uint64_t buf[12];
    for (size_t k = 0; k < blocks; ++k) {
        std::memcpy(buf, msg + k * 96, 96);
        mix(buf, h);
    }
    const size_t rem = len - blocks * 96;
    uint8_t last[96];
    std::memcpy(last, msg + blocks * 96, rem);
    std::memset(last + rem, 0, 96 - rem);
    last[95] = (uint8_t)rem;
    std::memcpy(buf, last, 96);
    for (int i = 0; i < 12; ++i) h[i] += buf[i];
    end_partial(h);
    end_partial(h);
    end_partial(h);
    h1 = h[0];
    h2 = h[1];
}
}  // namespace spooky

}  // namespace orc

// =========================================================================================
// C interface for ctypes (tests and benchmarks only).
// =========================================================================================
using namespace orc;

struct OrcHandle {
    BuildResult r;
};

extern "C" {

int orc_memo(uint32_t leaf, uint32_t *out /* 3000 */, uint32_t *lower, uint32_t *upper) {
    if (leaf < 2 || leaf > (uint32_t)kMaxLeafSize) return ERR_BAD_ARG;
    Shape s = make_shape(leaf);
    fill_memo(s, out);
    if (lower) *lower = s.lower;
    if (upper) *upper = s.upper;
    return OK;
}

// keys128: n pairs (first, second). Returns a handle (NULL and *status on error).
void *orc_build(const uint64_t *keys128, uint64_t n, uint32_t leaf, uint64_t bucket_size, int rotate, int threads,
                int *status) {
    auto *h = new OrcHandle;
    int st = build(keys128, n, leaf, bucket_size, rotate != 0, threads, nullptr, 0, h->r);
    if (status) *status = st;
    if (st != OK) {
        delete h;
        return nullptr;
    }
    return h;
}

// Seeds of a subset of buckets only (no encoding): for sampled checks of full-size builds.
void *orc_build_buckets(const uint64_t *keys128, uint64_t n, uint32_t leaf, uint64_t bucket_size, int rotate, int threads,
                        const uint64_t *buckets, uint64_t nsel, int *status) {
    auto *h = new OrcHandle;
    int st = build(keys128, n, leaf, bucket_size, rotate != 0, threads, buckets, nsel, h->r);
    if (status) *status = st;
    if (st != OK) {
        delete h;
        return nullptr;
    }
    return h;
}

// which: 0 serialized bytes, 1 seeds (u64), 2 node sizes (u32), 3 bucket_size_acc (u64),
// 4 bucket_pos_acc (u64), 5 algorithmic evaluations (u64 scalar). Returns element count.
uint64_t orc_result_len(void *hp, int which) {
    auto *h = (OrcHandle *)hp;
    switch (which) {
        case 0: return h->r.bytes.size();
        case 1: return h->r.seeds.size();
        case 2: return h->r.sizes.size();
        case 3: return h->r.bucket_size_acc.size();
        case 4: return h->r.bucket_pos_acc.size();
        case 5: return 1;
    }
    return 0;
}
void orc_result_copy(void *hp, int which, void *dst) {
    auto *h = (OrcHandle *)hp;
    switch (which) {
        case 0: std::memcpy(dst, h->r.bytes.data(), h->r.bytes.size()); break;
        case 1: std::memcpy(dst, h->r.seeds.data(), h->r.seeds.size() * 8); break;
        case 2: std::memcpy(dst, h->r.sizes.data(), h->r.sizes.size() * 4); break;
        case 3: std::memcpy(dst, h->r.bucket_size_acc.data(), h->r.bucket_size_acc.size() * 8); break;
        case 4: std::memcpy(dst, h->r.bucket_pos_acc.data(), h->r.bucket_pos_acc.size() * 8); break;
        case 5: std::memcpy(dst, &h->r.stats.evals_alg, 8); break;
    }
}
void orc_free(void *hp) { delete (OrcHandle *)hp; }

// Queries every key against a serialized MPHF. Returns status.
int orc_query(const uint8_t *bytes, uint64_t len, int rotate, const uint64_t *keys128, uint64_t n, uint64_t *out) {
    Mphf M;
    int st = deserialize(bytes, len, rotate != 0, M);
    if (st != OK) return st;
    for (uint64_t i = 0; i < n; ++i) out[i] = query(M, keys128[2 * i], keys128[2 * i + 1]);
    return OK;
}

// Bits of the structure as reported by getBits() (AbstractParallelRecSplit.hpp:476-478,
// DoubleEF.hpp:435-437); `object_bytes` stands for 8*sizeof(*this) of the C++ object.
uint64_t orc_get_bits(const uint8_t *bytes, uint64_t len, uint64_t object_bytes) {
    Mphf M;
    if (deserialize(bytes, len, true, M) != OK) return 0;
    const DoubleEF &e = M.ef;
    const uint64_t jump_half = e.jump_size_words() / 2;
    const uint64_t cum = (e.num_buckets + 1) * e.l_cum_keys + e.num_buckets + 1 + (e.u_cum_keys >> e.l_cum_keys) + jump_half;
    const uint64_t pos = (e.num_buckets + 1) * e.l_position + e.num_buckets + 1 + (e.u_position >> e.l_position) + jump_half;
    return cum + pos + M.descriptors.size() * 64 + 8 * object_bytes;
}

void orc_keygen_hash128(uint64_t seed, uint64_t n, uint64_t *out) {
    uint64_t s = seed;
    for (uint64_t i = 0; i < n; ++i) {
        out[2 * i] = splitmix64(s);
        out[2 * i + 1] = splitmix64(s);
    }
}
void orc_keygen_u64(uint64_t seed, uint64_t n, uint64_t *out) {
    uint64_t s = seed;
    for (uint64_t i = 0; i < n; ++i) out[i] = splitmix64(s);
}
void orc_hash_u64(const uint64_t *keys, uint64_t n, uint64_t *out128) {
    for (uint64_t i = 0; i < n; ++i) {
        out128[2 * i] = fmix64(keys[i]);
        out128[2 * i + 1] = stafford13(keys[i] + 0x9e3779b97f4a7c15ULL);
    }
}
// Random printable strings: length uniform in [min_len, max_len], bytes in 0x21..0x7E.
// With bytes == NULL only offsets (n+1 entries) are produced.
void orc_keygen_strings(uint64_t seed, uint64_t n, uint32_t min_len, uint32_t max_len, uint64_t *offsets, uint8_t *bytes) {
    uint64_t s = seed, off = 0;
    for (uint64_t i = 0; i < n; ++i) {
        offsets[i] = off;
        const uint32_t len = min_len + (uint32_t)(splitmix64(s) % (max_len - min_len + 1));
        for (uint32_t k = 0; k < len; ++k) {
            const uint8_t c = (uint8_t)(0x21 + splitmix64(s) % 94);
            if (bytes) bytes[off + k] = c;
        }
        off += len;
    }
    offsets[n] = off;
}
void orc_hash_strings(const uint8_t *bytes, const uint64_t *offsets, uint64_t n, uint64_t *out128) {
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t h0 = 0, h1 = 0;
        spooky::hash128(bytes + offsets[i], offsets[i + 1] - offsets[i], h0, h1);
        out128[2 * i] = h1;  // first  (util/Hash128.h:35: return {h1, h0})
        out128[2 * i + 1] = h0;
    }
}

uint32_t orc_remap16(uint64_t x, uint32_t n) { return remap16(x, n); }

// One aggregation-level search (the build's search_aggr) on m keys with parts of `split`
// keys from `seed`: lets tests compare the scalar and AVX-512 builds on single nodes.
uint64_t orc_search_aggr(const uint64_t *keys, uint32_t m, uint32_t split, uint64_t seed) {
    return search::search_aggr(keys, m, split, seed);
}

}  // extern "C"
