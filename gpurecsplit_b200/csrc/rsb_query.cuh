// Evaluation of a built function (host and device), operator() of the reference:
//   AbstractParallelRecSplit.hpp:409-466   query walk down the tree
//   RiceBitVector.hpp:150-218              Reader (readNext / skipSubtree / readReset)
//   DoubleEF.hpp:367-402                   get(bucket, cum_keys, cum_keys_next, position)
// Every memory read is bounds-checked (a word outside an array reads as zero), so a
// malformed or foreign structure can return a wrong value but never read out of bounds.
#pragma once

#include "rsb_common.cuh"

namespace rsb {

struct MphfView {
    Shape sh;
    uint64_t nbuckets;
    const uint64_t *desc;
    uint64_t desc_words;
    uint64_t u_cum_keys, u_position, l_cum_keys, l_position;
    int64_t cum_keys_min_delta, min_diff;
    uint64_t bits_per_key_fixed_point;
    const uint64_t *lower, *upper_cum, *upper_pos, *jump;
    uint64_t lower_words, cum_words, pos_words, jump_words;
    const uint32_t *memo;
};

__host__ __device__ __forceinline__ int q_popc(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}
__host__ __device__ __forceinline__ int q_ctz(uint64_t x) {
#ifdef __CUDA_ARCH__
    return __ffsll((long long)x) - 1;
#else
    return __builtin_ctzll(x);
#endif
}
// Position of the k-th (0-based) one of x; x must have more than k ones.
__host__ __device__ __forceinline__ uint64_t q_select(uint64_t x, uint64_t k) {
    uint64_t pos = 0;
    for (int w = 32; w >= 1; w >>= 1) {
        const uint64_t low = x & ((1ull << w) - 1);
        const uint64_t c = (uint64_t)q_popc(low);
        if (k >= c) {
            k -= c;
            x >>= w;
            pos += w;
        }
    }
    return pos;
}
__host__ __device__ __forceinline__ uint64_t q_word(const uint64_t *a, uint64_t n, uint64_t i) { return i < n ? a[i] : 0; }
// 64 bits starting at bit `bit` (little endian), the unaligned 8-byte read of the reference.
__host__ __device__ __forceinline__ uint64_t q_bits64(const uint64_t *a, uint64_t n, uint64_t bit) {
    const uint64_t w = bit / 64, sh = bit % 64;
    const uint64_t lo = q_word(a, n, w) >> sh;
    return sh ? lo | (q_word(a, n, w + 1) << (64 - sh)) : lo;
}

struct RiceReader {
    const uint64_t *data;
    uint64_t words;
    uint64_t fixed_off, window, ptr;
    int valid;

    __host__ __device__ void reset(uint64_t bit_pos, uint64_t unary_offset) {
        fixed_off = bit_pos;
        const uint64_t up = bit_pos + unary_offset;
        ptr = up / 64;
        window = q_word(data, words, ptr++) >> (up & 63);
        valid = 64 - (int)(up & 63);
    }
    __host__ __device__ uint64_t next(int log2golomb) {
        uint64_t result = 0;
        if (window == 0) {
            result += valid;
            window = q_word(data, words, ptr++);
            valid = 64;
            while (window == 0) {
                if (ptr > words + 1) return 0;  // ran off the stream: malformed input
                result += 64;
                window = q_word(data, words, ptr++);
            }
        }
        const int pos = q_ctz(window);
        window >>= pos;
        window >>= 1;
        valid -= pos + 1;
        result += pos;
        result <<= log2golomb;
        // fixed part: 8 bytes at fixed_off / 8, shifted by fixed_off % 8
        const uint64_t byte = fixed_off / 8;
        const uint64_t fixed = q_bits64(data, words, byte * 8);
        result |= (fixed >> (fixed_off % 8)) & ((1ull << log2golomb) - 1);
        fixed_off += log2golomb;
        return result;
    }
    __host__ __device__ void skip_subtree(uint64_t nodes, uint64_t fixed_len) {
        uint64_t missing = nodes, cnt;
        while ((cnt = (uint64_t)q_popc(window)) < missing) {
            if (ptr > words + 1) return;
            window = q_word(data, words, ptr++);
            missing -= cnt;
            valid = 64;
        }
        cnt = q_select(window, missing - 1);
        window >>= cnt;
        window >>= 1;
        valid -= (int)cnt + 1;
        fixed_off += fixed_len;
    }
};

__host__ __device__ inline void ef_get(const MphfView &f, uint64_t i, uint64_t &cum_keys, uint64_t &cum_keys_next,
                                       uint64_t &position) {
    constexpr uint64_t q = 256, q_mask = q - 1, super_q = 1 << 14, super_q_size = 1 + (super_q / q) / 4;
    const uint64_t lc = f.l_cum_keys, lp = f.l_position;
    const uint64_t pos_lower = i * (lc + lp);
    uint64_t lower = q_bits64(f.lower, f.lower_words, (pos_lower / 8) * 8) >> (pos_lower % 8);
    const uint64_t jsq = (i / super_q) * super_q_size * 2;
    const uint64_t jin = (i % super_q) / q;
    const uint64_t w16 = jsq + 2 + (2 * jin) / 4;
    const uint64_t jw = q_word(f.jump, f.jump_words, w16);
    const uint64_t j_cum = q_word(f.jump, f.jump_words, jsq) + ((jw >> (16 * ((2 * jin) % 4))) & 0xFFFF);
    const uint64_t j_pos = q_word(f.jump, f.jump_words, jsq + 1) + ((jw >> (16 * ((2 * jin + 1) % 4))) & 0xFFFF);
    uint64_t cw = j_cum / 64, pw = j_pos / 64;
    uint64_t win_c = q_word(f.upper_cum, f.cum_words, cw) & (~0ull << (j_cum % 64));
    uint64_t win_p = q_word(f.upper_pos, f.pos_words, pw) & (~0ull << (j_pos % 64));
    uint64_t dc = i & q_mask, dp = i & q_mask;
    for (uint64_t bc; (bc = (uint64_t)q_popc(win_c)) <= dc; dc -= bc) {
        if (cw + 1 >= f.cum_words) break;  // malformed structure
        win_c = q_word(f.upper_cum, f.cum_words, ++cw);
    }
    for (uint64_t bc; (bc = (uint64_t)q_popc(win_p)) <= dp; dp -= bc) {
        if (pw + 1 >= f.pos_words) break;  // malformed structure
        win_p = q_word(f.upper_pos, f.pos_words, ++pw);
    }
    const uint64_t sel_c = q_select(win_c, dc);
    const uint64_t cum_delta = i * (uint64_t)f.cum_keys_min_delta;
    cum_keys = ((cw * 64 + sel_c - i) << lc | (lower & ((1ull << lc) - 1))) + cum_delta;
    lower >>= lc;
    const uint64_t bit_delta = i * (uint64_t)f.min_diff;
    position = ((pw * 64 + q_select(win_p, dp) - i) << lp | (lower & ((1ull << lp) - 1))) + bit_delta +
               (uint64_t)(int64_t)(f.bits_per_key_fixed_point * cum_keys >> 20);
    win_c &= (~0ull << sel_c) << 1;
    while (win_c == 0) {
        if (cw + 1 >= f.cum_words) break;
        win_c = q_word(f.upper_cum, f.cum_words, ++cw);
    }
    lower >>= lp;
    cum_keys_next = ((cw * 64 + (uint64_t)q_ctz(win_c | (win_c == 0 ? (1ull << 63) : 0)) - i - 1) << lc |
                     (lower & ((1ull << lc) - 1))) +
                    cum_delta + (uint64_t)f.cum_keys_min_delta;
}

__host__ __device__ inline uint64_t mphf_query(const MphfView &f, uint64_t first, uint64_t second) {
    const uint32_t *memo = f.memo;
    const Shape &s = f.sh;
    const uint64_t bucket = remap128(first, f.nbuckets);
    uint64_t cum_keys, cum_keys_next, bit_pos;
    ef_get(f, bucket, cum_keys, cum_keys_next, bit_pos);
    uint64_t m = cum_keys_next - cum_keys;
    if (m >= (uint64_t)kMaxBucketSize) return cum_keys;  // not a key of this function
    RiceReader r{f.desc, f.desc_words, 0, 0, 0, 0};
    r.reset(bit_pos, memo[m] & 0xFFFF);
    int level = 0;
    while (m > s.upper) {
        const uint64_t d = r.next((int)(memo[m] >> 27));
        const uint64_t hmod = remap16(second + d + start_seed(level), (uint32_t)m);
        const uint32_t split = (uint16_t(m / 2 + s.upper - 1) / s.upper) * s.upper;
        if (hmod < split) {
            m = split;
        } else {
            r.skip_subtree((memo[split] >> 16) & 0x7FF, memo[split] & 0xFFFF);
            m -= split;
            cum_keys += split;
        }
        level++;
        if (level >= kMaxHigherDepth) break;
    }
    if (m > s.lower) {
        const uint64_t d = r.next((int)(memo[m] >> 27));
        const uint64_t hmod = remap16(second + d + start_seed(kNumStartSeeds - 3), (uint32_t)m);
        const uint32_t part = uint16_t(hmod) / s.lower;
        m = m - part * s.lower < s.lower ? m - part * s.lower : s.lower;
        cum_keys += (uint64_t)s.lower * part;
        if (part) r.skip_subtree(((memo[s.lower] >> 16) & 0x7FF) * part, (memo[s.lower] & 0xFFFF) * part);
    }
    if (m > s.leaf) {
        const uint64_t d = r.next((int)(memo[m] >> 27));
        const uint64_t hmod = remap16(second + d + start_seed(kNumStartSeeds - 2), (uint32_t)m);
        const uint32_t part = uint16_t(hmod) / s.leaf;
        m = m - part * s.leaf < s.leaf ? m - part * s.leaf : s.leaf;
        cum_keys += (uint64_t)s.leaf * part;
        if (part) r.skip_subtree(part, (memo[s.leaf] & 0xFFFF) * part);
    }
    const uint64_t b = r.next((int)(memo[m] >> 27));
    const uint64_t x = second + b + start_seed(kNumStartSeeds - 1);
    uint64_t leaf_val;
    if (s.rotate && m == s.leaf) {
        const uint64_t rotation = b % s.leaf;
        leaf_val = remap16(x - rotation, s.leaf);
        if (second % 2 != 0) leaf_val = (leaf_val + rotation) % s.leaf;
    } else {
        leaf_val = remap16(x, (uint32_t)(m ? m : 1));
    }
    return cum_keys + leaf_val;
}

}  // namespace rsb
