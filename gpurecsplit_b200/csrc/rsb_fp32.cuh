// The fp32 forms of the seed-search filters (device functions shared by the search kernels
// in rsb_search.cu and the exhaustive device check tests/cpp/fp32_device_check.cu).
//
// Both filters turn a 16-bit remap into an exact small integer with one fp32 fused
// multiply-add rounded toward minus infinity, so that the work runs on the FP32 pipes beside
// the integer hash. Their exactness for every 16-bit hash, fanout and leaf size is checked on
// the host (tests/cpp/fp32_filters.c) and on the device (tests/cpp/fp32_device_check.cu).
#pragma once

#include <cstdint>

namespace rsb {

// remix32 without its final xor-shift: hash16 = (z ^ z >> 16) & 0xFFFF = lo16(z) ^ hi16(z).
__device__ __forceinline__ uint32_t remix32_core(uint32_t z) {
    z ^= z >> 16;
    z *= 0x85ebca6bu;
    z ^= z >> 13;
    return z * 0xc2b2ae35u;
}

// Starting value of a full node's part-index accumulator: the bits of the fp32 2^23.
constexpr uint32_t kAccF0 = 0x4B000000u;

// Adds the part index of one candidate, given z = remix32_core of its key + seed, to acc.
// Full node (m = fan * SPLIT): the part index ((hash16 * m) >> 16) / SPLIT is
// p = floor(hash16 * fan / 2^16). The bits kAccF0 | hash16 are the fp32 F = 2^23 + hash16, and
// F * (fan / 2^16) = 128 fan + hash16 * fan / 2^16, so with acc an integer-valued fp32 in
// [2^23, 2^24), where the spacing of fp32 values is 1, one fused multiply-add rounded toward
// minus infinity gives exactly acc + 128 fan + p: acc counts 2^23 + 128 fan m + sum p after m
// keys, which stays below 2^24 for every node (128 fan m < 2^23). The add runs on the FP32
// pipes, beside the integer hash. Other nodes: with b = hash16 << 16, p = umulhi(b, mult) >> 28
// for mult = ceil(m * 2^28 / SPLIT) (< 2^32 as m < 16 * SPLIT; exact for every 16-bit hash,
// leaf size and node size, checked exhaustively).
template <bool FULL>
__device__ __forceinline__ void add_part(uint32_t z, uint32_t mult, float cf, uint32_t &acc) {
    if (FULL) {
        const uint32_t f = (z & 0xFFFFu) ^ __funnelshift_r(z, kAccF0 >> 16, 16);
        acc = __float_as_uint(__fmaf_rd(__uint_as_float(f), cf, __uint_as_float(acc)));
    } else {
        acc += __umulhi((z << 16) ^ (z & 0xFFFF0000u), mult) >> 28;
    }
}

// Adds the bit of one key, given z = remix32_core of key + seed, to a left-mask sum. The
// bit index p = remap16 = floor(hash16 * LEAF / 2^16) comes from one fp32 fused multiply-add
// rounded toward minus infinity, as in add_part: F = 2^23 + hash16 (bits kAccF0 | hash16)
// times LEAF / 2^16 plus 2^23 - 128 LEAF is exactly 2^23 + hash16 * LEAF / 2^16, which rounds
// down to the integer-valued fp32 2^23 + p, whose bits are kAccF0 + p. Times 2^23 plus
// 127 << 23 (mod 2^32) these bits become (127 + p) << 23, the fp32 2^p, which is added to the
// fp32 sum acc. Only the final integer add runs on the ALU pipe beside the hash.
template <int LEAF>
__device__ __forceinline__ void add_bit(uint32_t z, uint32_t &acc) {
    constexpr float kScale = (float)LEAF * 0x1p-16f, kBias = 0x1p23f - 128.0f * LEAF;
    const uint32_t f = (z & 0xFFFFu) ^ __funnelshift_r(z, kAccF0 >> 16, 16);
    const uint32_t t = __float_as_uint(__fmaf_rd(__uint_as_float(f), kScale, kBias));
    acc = __float_as_uint(__fadd_rn(__uint_as_float(acc), __uint_as_float(t * (1u << 23) + (127u << 23))));
}

// The left mask of a sum formed by add_bit over nl keys, or ~0u when two keys share a bit.
// Without a shared bit the terms are distinct powers of two below 2^LEAF <= 2^24, every
// partial sum is an integer below 2^24 and exact in fp32, and the sum is the mask with nl
// bits set. With one, either every partial sum stays below 2^24 (exact), and the carry leaves
// fewer than nl bits set, or the sum reaches 2^24 or more, out of the mask's range.
template <int LEAF>
__device__ __forceinline__ uint32_t left_mask_of(uint32_t acc, uint32_t nl) {
    static_assert(LEAF <= 24, "left-mask sums are exact below 2^24 only");
    const uint32_t mk = __float2uint_rz(__uint_as_float(acc));
    return (mk >> LEAF) == 0 && __popc(mk) == (int)nl ? mk : ~0u;
}

}  // namespace rsb
