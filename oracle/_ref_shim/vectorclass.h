/*
 * TEST INFRASTRUCTURE ONLY — used to compile the reference's own SIMDRecSplit sources into
 * oracle/_ref/ (the checker and the timed CPU reference arm), never by the product.
 *
 * Stand-in for the subset of Agner Fog's "vectorclass" library (VCL 2, Apache-2.0) that
 * GpuRecSplit's include/function/SIMDRecSplit.hpp and include/function/DoubleEF.hpp use.
 * The vectorclass submodule (extlib/vectorclass) is empty in this checkout, so this header
 * implements the documented semantics of those classes and functions for the AVX-512
 * instruction set (VCL's INSTRSET 10), written for this project:
 *
 *   Vec16ui  16 x uint32 lanes      Vec8uq  8 x uint64 lanes     Vec8q  8 x int64 lanes
 *   Vec64c   64 x int8 lanes        Vec16ib 16 boolean lanes (an AVX-512 mask register)
 *
 *   arithmetic and bit operators lane by lane with the scalar broadcast to every lane;
 *   >> is logical for unsigned element types and arithmetic for Vec8q;
 *   comparisons give Vec16ib; load/store are unaligned; operator[] reads one lane;
 *   blend16<i0..i15>(a, b) lane j = (i_j < 16 ? a[i_j] : b[i_j - 16]);
 *   lookup<n>(index, table) lane j = table[index[j]] (n <= 16: index taken mod 16 as VCL's
 *     in-register permute does; larger n: index limited to n - 1 and gathered);
 *   if_add(f, a, b) = a + (f ? b : 0); select(s, a, b) = s ? a : b;
 *   x / const_uint(d) lane-wise unsigned division by a compile-time constant;
 *   horizontal_or / horizontal_and / horizontal_find_first / to_bits on Vec16ib;
 *   horizontal_min and min on Vec8q (signed); shift_bytes_up/down<b> on Vec64c (zero fill).
 *
 * Only what those two reference headers call is provided. Lane arithmetic uses GCC vector
 * extensions (C semantics per lane, so wrap-around and division are exact by construction)
 * and AVX-512 intrinsics for masks and permutes.
 */
#pragma once

#include <immintrin.h>
#include <cstdint>
#include <cstring>

#if defined(__AVX512F__) && defined(__AVX512BW__) && defined(__AVX512DQ__) && defined(__AVX512VL__)
#define INSTRSET 10
#else
#error "this vectorclass stand-in implements the AVX-512 (F/BW/DQ/VL) subset only"
#endif

namespace vcl_shim {
typedef uint32_t u32x16 __attribute__((vector_size(64)));
typedef uint64_t u64x8 __attribute__((vector_size(64)));
typedef int64_t i64x8 __attribute__((vector_size(64)));
}  // namespace vcl_shim

// ----------------------------------------------------------------------------------------
// Vec16ib: 16 boolean lanes
// ----------------------------------------------------------------------------------------
class Vec16ib {
  public:
    __mmask16 m;
    Vec16ib() = default;
    Vec16ib(__mmask16 x) : m(x) {}
    operator __mmask16() const { return m; }
};
static inline Vec16ib operator&(Vec16ib a, Vec16ib b) { return Vec16ib(__mmask16(a.m & b.m)); }
static inline Vec16ib operator|(Vec16ib a, Vec16ib b) { return Vec16ib(__mmask16(a.m | b.m)); }
static inline Vec16ib operator^(Vec16ib a, Vec16ib b) { return Vec16ib(__mmask16(a.m ^ b.m)); }
static inline Vec16ib operator!(Vec16ib a) { return Vec16ib(__mmask16(~a.m)); }
static inline bool horizontal_or(Vec16ib a) { return a.m != 0; }
static inline bool horizontal_and(Vec16ib a) { return a.m == 0xFFFF; }
static inline int horizontal_find_first(Vec16ib a) { return a.m == 0 ? -1 : __builtin_ctz(a.m); }
static inline uint16_t to_bits(Vec16ib a) { return a.m; }

// ----------------------------------------------------------------------------------------
// Vec16ui: 16 x uint32
// ----------------------------------------------------------------------------------------
class Vec16ui {
  public:
    __m512i v;
    Vec16ui() = default;
    Vec16ui(uint32_t x) : v(_mm512_set1_epi32((int)x)) {}
    Vec16ui(__m512i x) : v(x) {}
    operator __m512i() const { return v; }
    vcl_shim::u32x16 lanes() const { return (vcl_shim::u32x16)v; }
    static Vec16ui of(vcl_shim::u32x16 x) { return Vec16ui((__m512i)x); }
    Vec16ui &load(const void *p) { v = _mm512_loadu_si512(p); return *this; }
    void store(void *p) const { _mm512_storeu_si512(p, v); }
    uint32_t operator[](int i) const {
        uint32_t t[16];
        store(t);
        return t[i & 15];
    }
};
static inline Vec16ui operator+(Vec16ui a, Vec16ui b) { return Vec16ui::of(a.lanes() + b.lanes()); }
static inline Vec16ui operator-(Vec16ui a, Vec16ui b) { return Vec16ui::of(a.lanes() - b.lanes()); }
static inline Vec16ui operator*(Vec16ui a, Vec16ui b) { return Vec16ui::of(a.lanes() * b.lanes()); }
static inline Vec16ui operator&(Vec16ui a, Vec16ui b) { return Vec16ui::of(a.lanes() & b.lanes()); }
static inline Vec16ui operator|(Vec16ui a, Vec16ui b) { return Vec16ui::of(a.lanes() | b.lanes()); }
static inline Vec16ui operator^(Vec16ui a, Vec16ui b) { return Vec16ui::of(a.lanes() ^ b.lanes()); }
static inline Vec16ui operator>>(Vec16ui a, uint32_t s) { return Vec16ui(_mm512_srl_epi32(a.v, _mm_cvtsi32_si128((int)s))); }
static inline Vec16ui operator<<(Vec16ui a, uint32_t s) { return Vec16ui(_mm512_sll_epi32(a.v, _mm_cvtsi32_si128((int)s))); }
static inline Vec16ui &operator+=(Vec16ui &a, Vec16ui b) { return a = a + b; }
static inline Vec16ui &operator*=(Vec16ui &a, Vec16ui b) { return a = a * b; }
static inline Vec16ui &operator&=(Vec16ui &a, Vec16ui b) { return a = a & b; }
static inline Vec16ui &operator|=(Vec16ui &a, Vec16ui b) { return a = a | b; }
static inline Vec16ui &operator^=(Vec16ui &a, Vec16ui b) { return a = a ^ b; }
static inline Vec16ib operator==(Vec16ui a, Vec16ui b) { return Vec16ib(_mm512_cmpeq_epu32_mask(a.v, b.v)); }
static inline Vec16ib operator!=(Vec16ui a, Vec16ui b) { return Vec16ib(_mm512_cmpneq_epu32_mask(a.v, b.v)); }
static inline Vec16ib operator<(Vec16ui a, Vec16ui b) { return Vec16ib(_mm512_cmplt_epu32_mask(a.v, b.v)); }
static inline Vec16ib operator<=(Vec16ui a, Vec16ui b) { return Vec16ib(_mm512_cmple_epu32_mask(a.v, b.v)); }
static inline Vec16ib operator>(Vec16ui a, Vec16ui b) { return Vec16ib(_mm512_cmpgt_epu32_mask(a.v, b.v)); }
static inline Vec16ib operator>=(Vec16ui a, Vec16ui b) { return Vec16ib(_mm512_cmpge_epu32_mask(a.v, b.v)); }

// a + (f ? b : 0), lane by lane
static inline Vec16ui if_add(Vec16ib f, Vec16ui a, Vec16ui b) { return Vec16ui(_mm512_mask_add_epi32(a.v, f.m, a.v, b.v)); }
// s ? a : b, lane by lane
static inline Vec16ui select(Vec16ib s, Vec16ui a, Vec16ui b) { return Vec16ui(_mm512_mask_mov_epi32(b.v, s.m, a.v)); }

template <int i0, int i1, int i2, int i3, int i4, int i5, int i6, int i7, int i8, int i9, int i10, int i11, int i12,
          int i13, int i14, int i15>
static inline Vec16ui blend16(Vec16ui a, Vec16ui b) {
    static_assert(i0 >= 0 && i1 >= 0 && i2 >= 0 && i3 >= 0 && i4 >= 0 && i5 >= 0 && i6 >= 0 && i7 >= 0 && i8 >= 0 &&
                      i9 >= 0 && i10 >= 0 && i11 >= 0 && i12 >= 0 && i13 >= 0 && i14 >= 0 && i15 >= 0,
                  "only lane indices 0..31 are provided");
    const __m512i idx = _mm512_setr_epi32(i0, i1, i2, i3, i4, i5, i6, i7, i8, i9, i10, i11, i12, i13, i14, i15);
    return Vec16ui(_mm512_permutex2var_epi32(a.v, idx, b.v));
}

template <int n>
static inline Vec16ui lookup(Vec16ui index, const void *table) {
    static_assert(n > 0, "table size must be positive");
    if constexpr (n <= 16) {
        return Vec16ui(_mm512_permutexvar_epi32(index.v, _mm512_loadu_si512(table)));
    } else {
        __m512i idx;
        if constexpr ((n & (n - 1)) == 0)
            idx = _mm512_and_si512(index.v, _mm512_set1_epi32(n - 1));
        else
            idx = _mm512_min_epu32(index.v, _mm512_set1_epi32(n - 1));
        return Vec16ui(_mm512_i32gather_epi32(idx, table, 4));
    }
}

// Division by a compile-time constant: x / const_uint(d)
template <uint32_t d> struct Const_uint_t {};
#define const_uint(x) Const_uint_t<(x)>()
template <uint32_t d>
static inline Vec16ui operator/(Vec16ui a, Const_uint_t<d>) {
    static_assert(d != 0, "division by zero");
    return Vec16ui::of(a.lanes() / d);
}

// ----------------------------------------------------------------------------------------
// Vec8uq: 8 x uint64 ; Vec8q: 8 x int64 ; Vec64c: 64 x int8
// ----------------------------------------------------------------------------------------
class Vec8uq {
  public:
    __m512i v;
    Vec8uq() = default;
    Vec8uq(uint64_t x) : v(_mm512_set1_epi64((long long)x)) {}
    Vec8uq(uint64_t a0, uint64_t a1, uint64_t a2, uint64_t a3, uint64_t a4, uint64_t a5, uint64_t a6, uint64_t a7)
        : v(_mm512_setr_epi64((long long)a0, (long long)a1, (long long)a2, (long long)a3, (long long)a4,
                              (long long)a5, (long long)a6, (long long)a7)) {}
    Vec8uq(__m512i x) : v(x) {}
    Vec8uq &operator=(__m512i x) { v = x; return *this; }
    operator __m512i() const { return v; }
    vcl_shim::u64x8 lanes() const { return (vcl_shim::u64x8)v; }
    static Vec8uq of(vcl_shim::u64x8 x) { return Vec8uq((__m512i)x); }
    Vec8uq &load(const void *p) { v = _mm512_loadu_si512(p); return *this; }
    void store(void *p) const { _mm512_storeu_si512(p, v); }
    uint64_t operator[](int i) const {
        uint64_t t[8];
        store(t);
        return t[i & 7];
    }
};
static inline Vec8uq operator+(Vec8uq a, Vec8uq b) { return Vec8uq::of(a.lanes() + b.lanes()); }
static inline Vec8uq operator-(Vec8uq a, Vec8uq b) { return Vec8uq::of(a.lanes() - b.lanes()); }
static inline Vec8uq operator*(Vec8uq a, Vec8uq b) { return Vec8uq::of(a.lanes() * b.lanes()); }
static inline Vec8uq operator&(Vec8uq a, Vec8uq b) { return Vec8uq::of(a.lanes() & b.lanes()); }
static inline Vec8uq operator|(Vec8uq a, Vec8uq b) { return Vec8uq::of(a.lanes() | b.lanes()); }
static inline Vec8uq operator^(Vec8uq a, Vec8uq b) { return Vec8uq::of(a.lanes() ^ b.lanes()); }
static inline Vec8uq operator>>(Vec8uq a, uint32_t s) { return Vec8uq(_mm512_srl_epi64(a.v, _mm_cvtsi32_si128((int)s))); }
static inline Vec8uq operator<<(Vec8uq a, uint32_t s) { return Vec8uq(_mm512_sll_epi64(a.v, _mm_cvtsi32_si128((int)s))); }
static inline Vec8uq &operator+=(Vec8uq &a, Vec8uq b) { return a = a + b; }
static inline Vec8uq &operator-=(Vec8uq &a, Vec8uq b) { return a = a - b; }
static inline Vec8uq &operator|=(Vec8uq &a, Vec8uq b) { return a = a | b; }
static inline Vec8uq &operator&=(Vec8uq &a, Vec8uq b) { return a = a & b; }

class Vec8q {
  public:
    __m512i v;
    Vec8q() = default;
    Vec8q(int64_t x) : v(_mm512_set1_epi64((long long)x)) {}
    Vec8q(__m512i x) : v(x) {}
    Vec8q &operator=(__m512i x) { v = x; return *this; }
    operator __m512i() const { return v; }
    vcl_shim::i64x8 lanes() const { return (vcl_shim::i64x8)v; }
    static Vec8q of(vcl_shim::i64x8 x) { return Vec8q((__m512i)x); }
    Vec8q &load(const void *p) { v = _mm512_loadu_si512(p); return *this; }
    void store(void *p) const { _mm512_storeu_si512(p, v); }
    int64_t operator[](int i) const {
        int64_t t[8];
        store(t);
        return t[i & 7];
    }
};
// Signed lanes: + - * wrap like the unsigned ones (computed unsigned), >> is arithmetic.
static inline Vec8q operator+(Vec8q a, Vec8q b) { return Vec8q((__m512i)((vcl_shim::u64x8)a.v + (vcl_shim::u64x8)b.v)); }
static inline Vec8q operator-(Vec8q a, Vec8q b) { return Vec8q((__m512i)((vcl_shim::u64x8)a.v - (vcl_shim::u64x8)b.v)); }
static inline Vec8q operator*(Vec8q a, Vec8q b) { return Vec8q((__m512i)((vcl_shim::u64x8)a.v * (vcl_shim::u64x8)b.v)); }
static inline Vec8q operator&(Vec8q a, Vec8q b) { return Vec8q(_mm512_and_si512(a.v, b.v)); }
static inline Vec8q operator|(Vec8q a, Vec8q b) { return Vec8q(_mm512_or_si512(a.v, b.v)); }
static inline Vec8q operator>>(Vec8q a, uint32_t s) { return Vec8q(_mm512_sra_epi64(a.v, _mm_cvtsi32_si128((int)s))); }
static inline Vec8q operator<<(Vec8q a, uint32_t s) { return Vec8q(_mm512_sll_epi64(a.v, _mm_cvtsi32_si128((int)s))); }
static inline Vec8q &operator+=(Vec8q &a, Vec8q b) { return a = a + b; }
static inline Vec8q &operator-=(Vec8q &a, Vec8q b) { return a = a - b; }
static inline Vec8q &operator|=(Vec8q &a, Vec8q b) { return a = a | b; }
static inline Vec8q min(Vec8q a, Vec8q b) { return Vec8q(_mm512_min_epi64(a.v, b.v)); }
static inline int64_t horizontal_min(Vec8q a) {
    int64_t t[8];
    a.store(t);
    int64_t r = t[0];
    for (int i = 1; i < 8; i++) r = t[i] < r ? t[i] : r;
    return r;
}

class Vec64c {
  public:
    __m512i v;
    Vec64c() = default;
    Vec64c(__m512i x) : v(x) {}
    operator __m512i() const { return v; }
};
static inline Vec8q &operator|=(Vec8q &a, Vec64c b) { return a = a | Vec8q(b.v); }

// Bytes move toward higher positions by b; the b lowest bytes become zero.
template <unsigned b>
static inline Vec64c shift_bytes_up(Vec64c a) {
    static_assert(b <= 64, "shift count");
    unsigned char in[64], out[64] = {0};
    std::memcpy(in, &a.v, 64);
    for (unsigned i = b; i < 64; i++) out[i] = in[i - b];
    __m512i r;
    std::memcpy(&r, out, 64);
    return Vec64c(r);
}

// Bytes move toward lower positions by b; the b highest bytes become zero.
template <unsigned b>
static inline Vec64c shift_bytes_down(Vec64c a) {
    static_assert(b <= 64, "shift count");
    unsigned char in[64], out[64] = {0};
    std::memcpy(in, &a.v, 64);
    for (unsigned i = 0; i + b < 64; i++) out[i] = in[i + b];
    __m512i r;
    std::memcpy(&r, out, 64);
    return Vec64c(r);
}

// AVX2-width names that the reference's headers mention only in their non-AVX-512 branches.
class Vec8ui;
class Vec4uq;
class Vec8ib;
class Vec4q;
class Vec32c;
