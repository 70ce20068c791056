// C++ drop-in check: code written against the reference's class API compiles unchanged
// against include/function/*.{cuh,hpp} and builds a bijection on the GPU.
//   usage: dropin_test <serialized-output-path>
#include <function/GPURecSplit.cuh>
#include <function/SIMDRecSplit.hpp>

#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

using bez::function::hash128_t;

static uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

template <class RS, class K>
static bool bijective(RS &rs, const std::vector<K> &keys) {
    std::vector<bool> seen(keys.size(), false);
    for (const auto &k : keys) {
        const size_t v = rs(k);
        if (v >= keys.size() || seen[v]) return false;
        seen[v] = true;
    }
    return true;
}

int main(int argc, char **argv) {
    if (argc < 2) return 2;
    uint64_t s = 0x5603141978c51071ULL;  // the reference tests' key seed (test/correctness.hpp:40)
    std::vector<hash128_t> keys;
    for (int i = 0; i < 100000; ++i) {
        const uint64_t a = splitmix64(s), b = splitmix64(s);
        keys.push_back(hash128_t(a, b));
    }
    const std::vector<hash128_t> copy = keys;
    bez::function::GPURecSplit<8> rs(keys, 100, 4);
    if (!bijective(rs, keys)) { std::puts("hash128 build is not a bijection"); return 1; }
    for (size_t i = 0; i < keys.size(); ++i)
        if (keys[i].first != copy[i].first || keys[i].second != copy[i].second) { std::puts("keys modified"); return 1; }
    {
        std::ofstream out(argv[1], std::ios::binary);
        out << rs;
    }
    bez::function::GPURecSplit<8> back;
    {
        std::ifstream in(argv[1], std::ios::binary);
        in >> back;
    }
    for (const auto &k : keys)
        if (back(k) != rs(k)) { std::puts("round trip differs"); return 1; }
    std::printf("bits/key %.4f\n", (double)rs.getBits() / keys.size());
    std::printf("getBits %zu\n", rs.getBits());

    std::vector<std::string> words;
    for (int i = 0; i < 5000; ++i) words.push_back("key-" + std::to_string(i * 7919));
    bez::function::SIMDRecSplit<5, sux::util::AllocType::MALLOC, true> sr(words, 10, 8);
    if (!bijective(sr, words)) { std::puts("string build is not a bijection"); return 1; }

    std::stringstream lines;
    for (auto &w : words) lines << w << "\n";
    {
        std::ofstream f(std::string(argv[1]) + ".keys");
        f << lines.str();
    }
    std::ifstream kin(std::string(argv[1]) + ".keys");
    bez::function::GPURecSplit<12, sux::util::AllocType::MALLOC, false> fr(kin, 100, 2);
    if (!bijective(fr, words)) { std::puts("stream build is not a bijection"); return 1; }

    bool threw = false;
    try {
        std::vector<hash128_t> dup = {hash128_t(1, 2), hash128_t(1, 2), hash128_t(3, 4)};
        bez::function::GPURecSplit<8> bad(dup, 100, 1);
    } catch (const std::runtime_error &) {
        threw = true;
    }
    if (!threw) { std::puts("duplicate keys were accepted"); return 1; }
    std::puts("dropin ok");
    return 0;
}
