// Device check of the fp32 seed-search filters (gpurecsplit_b200/csrc/rsb_fp32.cuh), run on
// the GPU with the same device functions the search kernels use, exhaustively:
//   1. add_part<true>: for every fanout 2..9 and 16-bit hash h, one rounded-down fused
//      multiply-add adds exactly 128 * fan + floor(h * fan / 2^16) to an integer-valued fp32
//      accumulator, for accumulators across [2^23, 2^24) up to the largest a node reaches;
//   2. add_part<false>: for every leaf size 2..24, both aggregation levels, every node size
//      that is not a multiple of the part size, and every h, the integer multiply-high gives
//      the reference's part index ((h * m) >> 16) / SPLIT (AbstractParallelRecSplit.hpp:334-336,
//      SIMDRecSplit.hpp:355,379);
//   3. add_bit<LEAF>: for every leaf size 2..24 and h, the term added is the fp32 2^p with
//      p = (h * LEAF) >> 16, and summing distinct powers of two gives the mask itself.
// Prints "fp32 device ok" and exits 0 when every case holds.
//   nvcc -gencode arch=compute_100a,code=sm_100a -I gpurecsplit_b200/csrc fp32_device_check.cu
#include <cstdio>

#include "rsb_fp32.cuh"

using namespace rsb;

__device__ unsigned long long g_bad[3];

// (lower_aggr, upper_aggr) per leaf size, AbstractParallelRecSplit.hpp:133,135
__constant__ unsigned c_lower[25] = {0, 0, 4, 6, 8, 15, 18, 21, 32, 36, 40, 55, 60, 78, 84, 90, 112, 119, 126, 152, 160, 168, 198, 207, 216};
__constant__ unsigned c_upper[25] = {0, 0, 8, 12, 16, 30, 36, 63, 96, 108, 120, 220, 240, 312, 336, 450, 560, 595, 630, 760, 960, 1008, 1188, 1242, 1296};

__global__ void k_full(void) {
    const unsigned h = blockIdx.x * blockDim.x + threadIdx.x;  // 0 .. 65535
    if (h >= 65536u) return;
    for (unsigned fan = 2; fan <= 9; ++fan) {
        const float cf = (float)fan * 0x1p-16f;
        const unsigned p = (h * fan) >> 16;
        const unsigned accs[6] = {0u, 1u, 12345u, 777777u, 3000000u, 0x7FFFFFu - 20000u};
        for (int a = 0; a < 6; ++a) {
            unsigned acc = kAccF0 + accs[a];
            add_part<true>(h, fan, cf, acc);  // z = h: hash16 = lo16 ^ hi16 = h
            if (acc != kAccF0 + accs[a] + 128u * fan + p) atomicAdd(&g_bad[0], 1ull);
        }
    }
}

__global__ void k_nonfull(void) {
    const unsigned h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 65536u) return;
    for (int leaf = 2; leaf <= 24; ++leaf) {
        for (int stage = 0; stage < 2; ++stage) {
            const unsigned split = stage ? c_lower[leaf] : (unsigned)leaf;
            const unsigned maxm = stage ? c_upper[leaf] : c_lower[leaf];
            for (unsigned m = split + 1; m <= maxm; ++m) {
                if (m % split == 0) continue;
                const unsigned mult = (unsigned)((((unsigned long long)m << 28) + split - 1) / split);
                unsigned acc = 0;
                add_part<false>(h, mult, 0.0f, acc);
                if (acc != ((h * m) >> 16) / split) atomicAdd(&g_bad[1], 1ull);
            }
        }
    }
}

template <int LEAF>
__device__ void check_bits(unsigned h) {
    const unsigned p = (h * LEAF) >> 16;
    unsigned acc = 0;
    add_bit<LEAF>(h, acc);
    if (acc != __float_as_uint((float)(1u << p))) atomicAdd(&g_bad[2], 1ull);
    // a sum of distinct powers of two is the mask; the last bit at p
    unsigned sum = __float_as_uint((float)((1u << LEAF) - 1 - (1u << p)));
    add_bit<LEAF>(h, sum);
    if (left_mask_of<LEAF>(sum, LEAF) != (1u << LEAF) - 1) atomicAdd(&g_bad[2], 1ull);
    // a collision: two keys on bit p sum to 2^(p+1), one bit for two keys
    unsigned dup = __float_as_uint((float)(1u << p));
    add_bit<LEAF>(h, dup);
    if (left_mask_of<LEAF>(dup, 2) != ~0u) atomicAdd(&g_bad[2], 1ull);
}

template <int LEAF>
__device__ void check_bits_upto(unsigned h) {
    check_bits<LEAF>(h);
    if constexpr (LEAF < 24) check_bits_upto<LEAF + 1>(h);
}

__global__ void k_bits(void) {
    const unsigned h = blockIdx.x * blockDim.x + threadIdx.x;
    if (h >= 65536u) return;
    check_bits_upto<2>(h);
}

int main() {
    unsigned long long zero[3] = {0, 0, 0}, bad[3];
    if (cudaMemcpyToSymbol(g_bad, zero, sizeof(zero)) != cudaSuccess) {
        std::printf("no device\n");
        return 2;
    }
    k_full<<<256, 256>>>();
    k_nonfull<<<256, 256>>>();
    k_bits<<<256, 256>>>();
    if (cudaDeviceSynchronize() != cudaSuccess || cudaMemcpyFromSymbol(bad, g_bad, sizeof(bad)) != cudaSuccess) {
        std::printf("cuda error\n");
        return 2;
    }
    std::printf("mismatches: full %llu, non-full %llu, bits %llu\n", bad[0], bad[1], bad[2]);
    if (bad[0] || bad[1] || bad[2]) return 1;
    std::printf("fp32 device ok\n");
    return 0;
}
