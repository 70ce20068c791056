// Host-side per-leaf-size tables of the construction engine.
#pragma once

#include <array>
#include <cstdint>
#include <vector>

#include "rsb_common.cuh"

namespace rsb {

struct LeafTables {
    Shape shape;
    std::vector<uint32_t> memo;       // Golomb-Rice table (kMaxBucketSize entries)
    std::vector<uint32_t> nodes;      // number of seeds of a bucket of size m
    uint32_t max_higher_depth = 0;    // fanout-2 depths that occur for m < kMaxBucketSize
};

Shape make_shape(uint32_t leaf, bool rotate);
// fill_golomb_rice, AbstractParallelRecSplit.hpp:191-227.
void fill_memo(const Shape &s, uint32_t *memo);
// Children of a split node of size m (fanout and unit), AbstractParallelRecSplit.hpp:137-148.
void split_params(const Shape &s, uint32_t m, uint32_t &fanout, uint32_t &unit);
const LeafTables &leaf_tables(uint32_t leaf, bool rotate);

inline uint32_t golomb_param(const uint32_t *memo, uint32_t m) { return memo[m] >> 27; }
inline uint32_t skip_bits(const uint32_t *memo, uint32_t m) { return memo[m] & 0xFFFF; }
inline uint32_t skip_nodes(const uint32_t *memo, uint32_t m) { return (memo[m] >> 16) & 0x7FF; }

}  // namespace rsb
