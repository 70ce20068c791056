// SpookyHash V2 128-bit (Bob Jenkins, public domain), host and device.
//
// The reference hashes string keys with spooky(key, len, 0) and keeps {first = h1, second = h0}
// (util/Hash128.h:32-36); SpookyV2 itself lives in the reference's sux submodule, which is
// not available here, so this is a restatement of the published algorithm.
#pragma once

#include <cstdint>

namespace rsb {

// Short path below 192 bytes (4-word state), block path otherwise (12-word state).
constexpr uint64_t kSpookyConst = 0xdeadbeefdeadbeefULL;
__host__ __device__ __forceinline__ uint64_t rotl64(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

__host__ __device__ __forceinline__ uint64_t load_le(const uint8_t *p, int nbytes) {
    uint64_t v = 0;
    for (int k = 0; k < nbytes; ++k) v |= uint64_t(p[k]) << (8 * k);
    return v;
}

// The same bytes from the aligned 32-bit words that hold them (one to three words, each
// holding at least one of the bytes), for keys staged in shared memory, where byte loads of
// a warp's keys at scattered offsets cost a shared-memory wavefront each.
__host__ __device__ __forceinline__ uint64_t load_le_words(const uint8_t *p, int nbytes) {
    if (nbytes <= 0) return 0;
    const uintptr_t a = (uintptr_t)p;
    const uint32_t *w = (const uint32_t *)(a & ~(uintptr_t)3);
    const uint32_t sh = (uint32_t)(a & 3) * 8;
    const int nw = (int)(((a & 3) + (uint32_t)nbytes + 3) >> 2);
    const uint32_t w0 = w[0], w1 = nw > 1 ? w[1] : 0u, w2 = nw > 2 ? w[2] : 0u;
#ifdef __CUDA_ARCH__
    const uint32_t lo = __funnelshift_r(w0, w1, sh), hi = __funnelshift_r(w1, w2, sh);
#else
    const uint32_t lo = (uint32_t)((((uint64_t)w1 << 32) | w0) >> sh);
    const uint32_t hi = (uint32_t)((((uint64_t)w2 << 32) | w1) >> sh);
#endif
    const uint64_t v = ((uint64_t)hi << 32) | lo;
    return nbytes >= 8 ? v : v & ((1ull << (8 * nbytes)) - 1);
}

// Loads through word reads (WORDS, for 4-byte-aligned buffers whose words around the key
// may be read) or byte reads.
template <bool WORDS>
__host__ __device__ __forceinline__ uint64_t sp_load(const uint8_t *p, int nbytes) {
    return WORDS ? load_le_words(p, nbytes) : load_le(p, nbytes);
}

__host__ __device__ __forceinline__ void sp_short_mix(uint64_t &h0, uint64_t &h1, uint64_t &h2, uint64_t &h3) {
    h2 = rotl64(h2, 50); h2 += h3; h0 ^= h2;
    h3 = rotl64(h3, 52); h3 += h0; h1 ^= h3;
    h0 = rotl64(h0, 30); h0 += h1; h2 ^= h0;
    h1 = rotl64(h1, 41); h1 += h2; h3 ^= h1;
    h2 = rotl64(h2, 54); h2 += h3; h0 ^= h2;
    h3 = rotl64(h3, 48); h3 += h0; h1 ^= h3;
    h0 = rotl64(h0, 38); h0 += h1; h2 ^= h0;
    h1 = rotl64(h1, 37); h1 += h2; h3 ^= h1;
    h2 = rotl64(h2, 62); h2 += h3; h0 ^= h2;
    h3 = rotl64(h3, 34); h3 += h0; h1 ^= h3;
    h0 = rotl64(h0, 5);  h0 += h1; h2 ^= h0;
    h1 = rotl64(h1, 36); h1 += h2; h3 ^= h1;
}
__host__ __device__ __forceinline__ void sp_short_end(uint64_t &h0, uint64_t &h1, uint64_t &h2, uint64_t &h3) {
    h3 ^= h2; h2 = rotl64(h2, 15); h3 += h2;
    h0 ^= h3; h3 = rotl64(h3, 52); h0 += h3;
    h1 ^= h0; h0 = rotl64(h0, 26); h1 += h0;
    h2 ^= h1; h1 = rotl64(h1, 51); h2 += h1;
    h3 ^= h2; h2 = rotl64(h2, 28); h3 += h2;
    h0 ^= h3; h3 = rotl64(h3, 9);  h0 += h3;
    h1 ^= h0; h0 = rotl64(h0, 47); h1 += h0;
    h2 ^= h1; h1 = rotl64(h1, 54); h2 += h1;
    h3 ^= h2; h2 = rotl64(h2, 32); h3 += h2;
    h0 ^= h3; h3 = rotl64(h3, 25); h0 += h3;
    h1 ^= h0; h0 = rotl64(h0, 63); h1 += h0;
}

template <bool WORDS = false>
__host__ __device__ inline void spooky_short(const uint8_t *p, uint64_t len, uint64_t &o1, uint64_t &o2) {
    uint64_t a = o1, b = o2, c = kSpookyConst, d = kSpookyConst;
    uint64_t rem = len % 32;
    if (len > 15) {
        const uint8_t *end = p + (len / 32) * 32;
        for (; p < end; p += 32) {
            c += sp_load<WORDS>(p, 8);
            d += sp_load<WORDS>(p + 8, 8);
            sp_short_mix(a, b, c, d);
            a += sp_load<WORDS>(p + 16, 8);
            b += sp_load<WORDS>(p + 24, 8);
        }
        if (rem >= 16) {
            c += sp_load<WORDS>(p, 8);
            d += sp_load<WORDS>(p + 8, 8);
            sp_short_mix(a, b, c, d);
            p += 16;
            rem -= 16;
        }
    }
    d += len << 56;
    if (rem == 0) {
        c += kSpookyConst;
        d += kSpookyConst;
    } else if (rem >= 8) {
        c += sp_load<WORDS>(p, 8);
        d += sp_load<WORDS>(p + 8, (int)rem - 8);
    } else {
        c += sp_load<WORDS>(p, (int)rem);
    }
    sp_short_end(a, b, c, d);
    o1 = a;
    o2 = b;
}

__host__ __device__ inline void sp_mix(const uint64_t *data, uint64_t *s) {
    const int r[12] = {11, 32, 43, 31, 17, 28, 39, 57, 55, 54, 22, 46};
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        s[i] += data[i];
        s[(i + 2) % 12] ^= s[(i + 10) % 12];
        s[(i + 11) % 12] ^= s[i];
        s[i] = rotl64(s[i], r[i]);
        s[(i + 11) % 12] += s[(i + 1) % 12];
    }
}
__host__ __device__ inline void sp_end_partial(uint64_t *h) {
    const int r[12] = {44, 15, 34, 21, 38, 33, 10, 13, 38, 53, 42, 54};
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        h[(i + 11) % 12] += h[(i + 1) % 12];
        h[(i + 2) % 12] ^= h[(i + 11) % 12];
        h[(i + 1) % 12] = rotl64(h[(i + 1) % 12], r[i]);
    }
}

template <bool WORDS = false>
__host__ __device__ inline void spooky128(const uint8_t *msg, uint64_t len, uint64_t &o1, uint64_t &o2) {
    if (len < 192) {
        spooky_short<WORDS>(msg, len, o1, o2);
        return;
    }
    uint64_t h[12], buf[12];
#pragma unroll
    for (int i = 0; i < 12; i += 3) {
        h[i] = o1;
        h[i + 1] = o2;
        h[i + 2] = kSpookyConst;
    }
    const uint64_t blocks = len / 96;
    for (uint64_t k = 0; k < blocks; ++k) {
#pragma unroll
        for (int i = 0; i < 12; ++i) buf[i] = sp_load<WORDS>(msg + k * 96 + 8 * i, 8);
        sp_mix(buf, h);
    }
    const uint64_t rem = len - blocks * 96;
    const uint8_t *tail = msg + blocks * 96;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const int64_t avail = (int64_t)rem - 8 * i;
        buf[i] = avail <= 0 ? 0 : sp_load<WORDS>(tail + 8 * i, avail >= 8 ? 8 : (int)avail);
    }
    buf[11] = (buf[11] & ~(0xFFull << 56)) | (rem << 56);
#pragma unroll
    for (int i = 0; i < 12; ++i) h[i] += buf[i];
    sp_end_partial(h);
    sp_end_partial(h);
    sp_end_partial(h);
    o1 = h[0];
    o2 = h[1];
}

}  // namespace rsb
