/* Host check of the fp32 arithmetic the seed-search filters run on the device (IEEE-754
 * binary32 on both sides): the part index of a full aggregation node added by one fused
 * multiply-add rounded toward minus infinity, the rotation-leaf bit index taken the same way
 * and turned into the fp32 2^p by an integer multiply-add, and the collision test of a
 * left-mask sum of powers of two. Exhaustive over every 16-bit hash; prints "fp32 ok" and
 * exits 0 when every case holds. */
#include <fenv.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

static float as_float(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static uint32_t as_bits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static int popc(uint32_t v) { int c = 0; while (v) { v &= v - 1; ++c; } return c; }

static long bad = 0;
static void fail(const char *what, unsigned a, unsigned b, unsigned c) {
    if (bad++ < 10) printf("FAIL %s %u %u %u\n", what, a, b, c);
}

int main(void) {
    const uint32_t k_acc0 = 0x4B000000u;  /* fp32 2^23 */
    /* 1: full-node part index, acc + 128 fan + floor(h * fan / 2^16), accumulators across the
     * whole range a node can reach (a fanout-9 node of 1296 keys stays below 2^23 + 1.5e6). */
    fesetround(FE_DOWNWARD);
    for (uint32_t fan = 2; fan <= 16; ++fan) {
        volatile float cf = (float)fan * 0x1p-16f;
        const uint32_t accs[] = {0, 1, 12345, 777777, 3000000, 0x7FFFFF - 20000};
        for (int a = 0; a < 6; ++a)
            for (uint32_t h = 0; h < 65536; ++h) {
                const uint32_t acc = k_acc0 + accs[a];
                const uint32_t r = as_bits(fmaf(as_float(k_acc0 | h), cf, as_float(acc)));
                if (r != acc + 128u * fan + ((h * fan) >> 16)) fail("part", fan, accs[a], h);
            }
    }
    /* 2: leaf bit index p = floor(h * LEAF / 2^16) and the fp32 2^p */
    for (uint32_t leaf = 2; leaf <= 24; ++leaf) {
        volatile float scale = (float)leaf * 0x1p-16f, bias = 0x1p23f - 128.0f * leaf;
        for (uint32_t h = 0; h < 65536; ++h) {
            const uint32_t p = (h * leaf) >> 16;
            const uint32_t t = as_bits(fmaf(as_float(k_acc0 | h), scale, bias));
            if (t != k_acc0 + p) fail("bit", leaf, h, t);
            const float pw = as_float(t * (1u << 23) + (127u << 23));
            if (pw != ldexpf(1.0f, (int)p)) fail("pow", leaf, h, p);
        }
    }
    /* 3: a sum (round to nearest) of nl powers 2^p, p < LEAF, read back by truncation, has nl
     * bits set and no bit at or above LEAF exactly when the p are distinct */
    fesetround(FE_TONEAREST);
    uint64_t s = 0x9E3779B97F4A7C15ull;
    for (uint32_t leaf = 2; leaf <= 24; ++leaf)
        for (uint32_t nl = 0; nl <= leaf; ++nl)
            for (int rep = 0; rep < 4000; ++rep) {
                volatile float acc = 0.0f;
                uint32_t seen = 0;
                int distinct = 1;
                for (uint32_t i = 0; i < nl; ++i) {
                    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
                    /* mostly small index ranges so that collisions and carries are frequent */
                    const uint32_t p = (uint32_t)(s >> 40) % (rep & 1 ? leaf : (leaf < 4 ? leaf : 4 + (leaf - 4) * (rep & 2) / 2));
                    if (seen >> p & 1) distinct = 0;
                    seen |= 1u << p;
                    acc = acc + ldexpf(1.0f, (int)p);
                }
                const uint32_t mk = (uint32_t)acc;
                const int pass = (mk >> leaf) == 0 && popc(mk) == (int)nl;
                if (pass != distinct || (pass && mk != seen)) fail("mask", leaf, nl, mk);
            }
    /* a worst case of carries: every key of a 24-key leaf on bit 23 */
    {
        volatile float acc = 0.0f;
        for (int i = 0; i < 24; ++i) acc = acc + 0x1p23f;
        const uint32_t mk = (uint32_t)acc;
        if ((mk >> 24) == 0 && popc(mk) == 24) fail("carry", 24, 24, mk);
    }
    if (bad) {
        printf("%ld failures\n", bad);
        return 1;
    }
    printf("fp32 ok\n");
    return 0;
}
