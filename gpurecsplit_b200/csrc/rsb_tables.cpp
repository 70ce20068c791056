// Per-leaf-size constants: tree shape, Golomb-Rice parameters and node counts.
#include "rsb_tables.h"

#include <atomic>
#include <cmath>
#include <map>
#include <mutex>

#include "rsb_kernels.cuh"

namespace rsb {

static std::atomic<uint64_t> g_launches{0};
void count_launches(uint64_t k) { g_launches.fetch_add(k, std::memory_order_relaxed); }
uint64_t launches_so_far() { return g_launches.load(std::memory_order_relaxed); }

// AbstractParallelRecSplit.hpp:106 — Rice parameters of bijection leaves.
static const uint8_t kBijMemo[25] = {0, 0, 0, 1, 3, 4, 5, 7, 8, 10, 11, 12, 14, 15, 16, 18, 19, 21, 22, 23, 25, 26, 28, 29, 30};

// lower_aggr = leaf * max(2, ceil(0.35 leaf + 1/2)); upper_aggr = lower_aggr * (leaf < 7 ? 2 :
// ceil(0.21 leaf + 9/10)), AbstractParallelRecSplit.hpp:133,135 (the second factor is a double).
Shape make_shape(uint32_t leaf, bool rotate) {
    Shape s{};
    s.leaf = leaf;
    const double a = std::ceil(0.35 * leaf + 1. / 2);
    s.lower = leaf * (uint32_t)(a > 2 ? a : 2);
    const double b = leaf < 7 ? 2.0 : std::ceil(0.21 * leaf + 9. / 10);
    s.upper = (uint32_t)((double)s.lower * b);
    s.rotate = rotate ? 1 : 0;
    return s;
}

void split_params(const Shape &s, uint32_t m, uint32_t &fanout, uint32_t &unit) {
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

// Bits 27-31: Rice parameter of the node; 16-26: nodes in its subtree; 0-15: fixed bits in
// its subtree. The subtree fields are or-ed in without masking, exactly as the reference
// does, so that large leaf-2 entries carry the same (overflowing) values.
void fill_memo(const Shape &s, uint32_t *memo) {
    uint32_t m = 0;
    for (; m <= s.leaf; ++m) memo[m] = uint32_t(kBijMemo[m]) << 27 | uint32_t(m > 1) << 16 | kBijMemo[m];
    for (; m < (uint32_t)kMaxBucketSize; ++m) {
        uint32_t fanout, unit;
        split_params(s, m, fanout, unit);
        int part[kMaxFanout] = {0};
        part[fanout - 1] = (int)m;
        for (uint32_t i = 0; i + 1 < fanout; ++i) {
            part[i] = (int)unit;
            part[fanout - 1] -= (int)unit;
        }
        // Probability that a random seed splits m keys into the parts (Stirling), and the
        // Rice parameter ceil(log2(log(phi) / -log1p(-p))) of the resulting geometric law.
        double prod = 1;
        for (uint32_t i = 0; i < fanout; ++i) prod *= std::sqrt((double)part[i]);
        const double p = std::sqrt((double)m) / (std::pow(2 * M_PI, (fanout - 1.) / 2) * prod);
        uint32_t bits = (uint32_t)std::ceil(std::log2(-std::log((std::sqrt(5.0) + 1) / 2) / std::log1p(-p)));
        memo[m] = bits << 27;
        for (uint32_t i = 0; i < fanout; ++i) bits += memo[part[i]] & 0xFFFF;
        memo[m] |= bits;
        uint32_t nodes = 1;
        for (uint32_t i = 0; i < fanout; ++i) nodes += (memo[part[i]] >> 16) & 0x7FF;
        memo[m] |= nodes << 16;
    }
}

// Exact seed counts per bucket size (the memo's 11-bit node field saturates for leaf 2).
static void fill_nodes(const Shape &s, std::vector<uint32_t> &nodes, uint32_t &max_depth) {
    nodes.assign(kMaxBucketSize, 0);
    std::vector<uint32_t> depth(kMaxBucketSize, 0);  // fanout-2 levels below a node of size m
    for (uint32_t m = 2; m < (uint32_t)kMaxBucketSize; ++m) {
        if (m <= s.leaf) {
            nodes[m] = 1;
            continue;
        }
        uint32_t fanout, unit;
        split_params(s, m, fanout, unit);
        uint32_t c = 1;
        for (uint32_t i = 0; i + 1 < fanout; ++i) c += nodes[unit];
        c += nodes[m - (fanout - 1) * unit];
        nodes[m] = c;
        if (m > s.upper) depth[m] = 1 + std::max(depth[unit], depth[m - unit]);
    }
    max_depth = 0;
    for (uint32_t m = 0; m < (uint32_t)kMaxBucketSize; ++m) max_depth = std::max(max_depth, depth[m]);
}

const LeafTables &leaf_tables(uint32_t leaf, bool rotate) {
    static std::mutex mu;
    static std::map<uint32_t, LeafTables> cache;
    std::lock_guard<std::mutex> lock(mu);
    const uint32_t key = leaf * 2 + (rotate ? 1 : 0);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
    LeafTables t;
    t.shape = make_shape(leaf, rotate);
    t.memo.assign(kMaxBucketSize, 0);
    fill_memo(t.shape, t.memo.data());
    fill_nodes(t.shape, t.nodes, t.max_higher_depth);
    return cache.emplace(key, std::move(t)).first->second;
}

}  // namespace rsb
