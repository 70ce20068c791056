// Shared definitions of the B200 RecSplit construction engine (device and host).
//
// The construction follows ByteHamster/GpuRecSplit's SIMDRecSplit semantics:
//   remixAndRemap (16-bit remap), AbstractParallelRecSplit.hpp:277-284,327-337
//   start seeds, AbstractParallelRecSplit.hpp:95-98
//   tree shape (SplittingStrategy), AbstractParallelRecSplit.hpp:121-184
// All device arithmetic is exact 32/64-bit integer work.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "rsb.h"  // include/ is on the include path of every build

namespace rsb {

constexpr int kMaxBucketSize = 3000;  // AbstractParallelRecSplit.hpp:60
constexpr int kMaxLeafSize = 24;      // AbstractParallelRecSplit.hpp:62
constexpr int kMaxFanout = 9;         // AbstractParallelRecSplit.hpp:63
constexpr int kNumStartSeeds = 20;

// Search stages. Fanout-2 nodes at depth d use stage d (start_seed[d]); the two aggregation
// levels and the leaves use start_seed[17], [18] and [19] whatever their depth.
constexpr int kStageUpper = 17;
constexpr int kStageLower = 18;
constexpr int kStageLeafRot = 19;
constexpr int kStageLeafBF = 20;
constexpr int kNumStages = 21;
constexpr int kMaxHigherDepth = 17;

constexpr uint64_t kSeedNotFound = ~0ull;      // search still running
constexpr uint64_t kSeedFailed = ~0ull - 1;    // search abandoned (budget / duplicate)

// AbstractParallelRecSplit.hpp:95-97
__host__ __device__ constexpr uint64_t start_seed(int i) {
    constexpr uint64_t s[20] = {
        0x106393c187cae21a, 0x6453cec3f7376937, 0x643e521ddbd2be98, 0x3740c6412f6572cb, 0x717d47562f1ce470,
        0x4cd6eb4c63befb7c, 0x9bfd8c5e18c8da73, 0x082f20e10092a9a3, 0x2ada2ce68d21defc, 0xe33cb4f3e7c6466b,
        0x3980be458c509c59, 0xc466fd9584828e8c, 0x45f0aabe1a61ede6, 0xf6e7b8b33ad9b98d, 0x4ef95e25f4b4983d,
        0x81175195173b92d3, 0x4e50927d8dd15978, 0x1ea2099d1fafae7f, 0x425c8a06fbaaa815, 0xcd4216006c74052a};
    return s[i];
}

// remix32 (MurmurHash3 32-bit finalizer), AbstractParallelRecSplit.hpp:277-284.
__host__ __device__ __forceinline__ uint32_t remix32(uint32_t z) {
    z ^= z >> 16;
    z *= 0x85ebca6bu;
    z ^= z >> 13;
    z *= 0xc2b2ae35u;
    z ^= z >> 16;
    return z;
}

// remixAndRemap<false>: ((remix32(hi ^ lo) & 0xFFFF) * n) >> 16, AbstractParallelRecSplit.hpp:327-337.
__host__ __device__ __forceinline__ uint32_t remap16(uint64_t x, uint32_t n) {
    return ((remix32(uint32_t(x >> 32) ^ uint32_t(x)) & 0xFFFFu) * n) >> 16;
}

// remap128: (x * n) >> 64, support/common.hpp:273-280.
__host__ __device__ __forceinline__ uint64_t remap128(uint64_t x, uint64_t n) {
#ifdef __CUDA_ARCH__
    return __umul64hi(x, n);
#else
    return (uint64_t)(((unsigned __int128)x * n) >> 64);
#endif
}

// Per-leaf-size constants (SplittingStrategy::lower_aggr/upper_aggr and the Golomb-Rice table).
struct Shape {
    uint32_t leaf, lower, upper;
    uint32_t rotate;
};

// Device-resident description of one build ("set"). The batched form concatenates many.
struct NodeArrays {
    uint32_t *start;     // first key of the node (index into the key array)
    uint16_t *size;      // number of keys
    uint8_t *stage;      // search stage
    uint64_t *seed;      // encoded seed x (DFS order), kSeedNotFound while searching
    uint32_t *next_win;  // next seed window to hand out (search scheduler)
};

// Status word written by kernels (first error wins).
struct DevStatus {
    int code;
    int pad;
    uint64_t detail;
};

#ifdef __CUDACC__
__device__ __forceinline__ void set_error(DevStatus *st, int code, uint64_t detail) {
    if (atomicCAS(&st->code, 0, code) == 0) st->detail = detail;
}
#endif

}  // namespace rsb
