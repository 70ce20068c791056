"""CPU checks of the oracle (no GPU): pins against the reference's own fixtures.

The reference ships no golden outputs (its tests check bijectivity and GPU/SIMD
equivalence); the pins available for the oracle are its Golomb-Rice table
(include/function/golombRiceMemo.hpp), the bijection property over the correctness grid
(test/correctness.hpp:24-27, test/recsplitCorrectness.hpp:10-35) and the published
bits/object values (README.md:16-23).
"""
import hashlib
import json
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
SEED = 0x5603141978c51071  # seed of the reference's test key generator, test/correctness.hpp:40


def memo_digests():
    with open(os.path.join(GOLDEN, "memo_digests.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("leaf", range(2, 25))
def test_oracle_memo_matches_reference_table(oracle_mod, leaf):
    d = memo_digests()["leaf"][str(leaf)]
    memo, _, _ = oracle_mod.memo(leaf)
    assert hashlib.sha256(memo.astype("<u4").tobytes()).hexdigest() == d["sha256"]
    for m, v in d["spot"].items():
        assert int(memo[int(m)]) == v


def test_oracle_aggregation_bounds(oracle_mod):
    # lower_aggr / upper_aggr, AbstractParallelRecSplit.hpp:133,135
    expect = {8: (32, 96), 12: (60, 240), 16: (112, 560), 24: (216, 1296), 2: (4, 8), 7: (21, 63)}
    for leaf, (lo, up) in expect.items():
        _, l, u = oracle_mod.memo(leaf)
        assert (l, u) == (lo, up)


def _grid():
    # The reference correctness grid (test/correctness.hpp:24-38) restricted to sizes a
    # scalar oracle finishes in seconds: full leaf range, small buckets for large leaves.
    out = []
    for leaf in range(2, 25):
        for b in (2, 3, 5, 10, 25, 100, 231):
            if leaf >= 13 and b > 25:
                continue
            if leaf >= 19 and b > 10:
                continue
            for n in (1, 10, 100, 123, 1000):
                out.append((leaf, b, n))
    return out


@pytest.mark.parametrize("leaf,b,n", _grid())
def test_oracle_bijection_grid(oracle_mod, leaf, b, n):
    keys = oracle_mod.keygen_hash128(SEED, n)
    res = oracle_mod.build_mphf(keys, leaf, b, True)
    q = oracle_mod.query(res.bytes, keys)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


@pytest.mark.parametrize("leaf,b,n", [(8, 100, 20000), (5, 7, 5000), (12, 231, 5000)])
def test_oracle_bijection_bruteforce_leaves(oracle_mod, leaf, b, n):
    keys = oracle_mod.keygen_hash128(SEED, n)
    res = oracle_mod.build_mphf(keys, leaf, b, False)
    q = oracle_mod.query(res.bytes, keys, rotate=False)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


def test_oracle_bits_per_key_l16_b2000(oracle_mod):
    # README.md:16-18: 1.560 bits/object at l=16, b=2000 (n=5M). A 20-bucket sample of the
    # same shape lands within sampling noise of it.
    n = 40000
    keys = oracle_mod.keygen_hash128(SEED, n)
    res = oracle_mod.build_mphf(keys, 16, 2000, True)
    bpk = oracle_mod.get_bits(res.bytes) / n
    assert 1.50 < bpk < 1.64, bpk


def test_oracle_bits_per_key_l8_b100(oracle_mod):
    n = 200000
    keys = oracle_mod.keygen_hash128(SEED, n)
    res = oracle_mod.build_mphf(keys, 8, 100, True)
    bpk = oracle_mod.get_bits(res.bytes) / n
    assert 1.7 < bpk < 1.9, bpk


def test_oracle_duplicate_key_is_an_error(oracle_mod):
    keys = oracle_mod.keygen_hash128(SEED, 100)
    keys[7] = keys[3]
    with pytest.raises(oracle_mod.OracleError) as e:
        oracle_mod.build_mphf(keys, 8, 100)
    assert e.value.status == 2


def test_oracle_seed_order_independent(oracle_mod):
    # F5: the seed of a node depends only on the set of its keys.
    keys = oracle_mod.keygen_hash128(SEED, 3000)
    a = oracle_mod.build_mphf(keys, 8, 100)
    perm = np.random.default_rng(1).permutation(3000)
    b = oracle_mod.build_mphf(keys[perm], 8, 100)
    assert a.bytes.tobytes() == b.bytes.tobytes()


def test_oracle_u64_mixer_distinct_seconds(oracle_mod):
    k = oracle_mod.keygen_u64(42, 100000)
    h = oracle_mod.hash_u64(k)
    assert np.unique(h[:, 1]).size == k.size


_SIMD_GRID = [(leaf, b, n, rot) for leaf in (2, 3, 5, 8, 11, 12, 16, 20, 24) for (b, n) in ((7, 500), (100, 3000), (2000, 2500))
              for rot in (True, False) if not (leaf >= 20 and n > 600) and not (not rot and leaf >= 16 and n > 600)]


@pytest.mark.parametrize("leaf,b,n,rot", _SIMD_GRID)
def test_simd_oracle_equals_scalar(oracle_mod, leaf, b, n, rot):
    """The AVX-512 search loops (the timed CPU baseline) give the scalar oracle's bytes."""
    if not oracle_mod.simd_supported():
        pytest.skip("CPU lacks AVX-512 F/DQ/BW/VL/VPOPCNTDQ")
    keys = oracle_mod.keygen_hash128(leaf * 1000 + b + n, n)
    a = oracle_mod.build_mphf(keys, leaf, b, rot, threads=4)
    s = oracle_mod.build_mphf(keys, leaf, b, rot, threads=4, simd=True)
    assert a.bytes.tobytes() == s.bytes.tobytes()
    assert np.array_equal(a.seeds, s.seeds)


# Minimum seed of each node from `seed` below, found once by the scalar search (minutes).
_FANOUT9_SEEDS = {(22, 190): 111351572, (23, 200): 33009561, (24, 200): 176426661}


@pytest.mark.parametrize("leaf,m", sorted(_FANOUT9_SEEDS))
def test_simd_oracle_fanout9_remainder(oracle_mod, leaf, m):
    """A lower-aggregation node of fanout 9 whose last part is short: the ninth part is
    implied by the packed counts of the other eight. Both searches start 40 candidates before
    the node's minimum seed, so both must return exactly 40."""
    if not oracle_mod.simd_supported():
        pytest.skip("CPU lacks AVX-512 F/DQ/BW/VL/VPOPCNTDQ")
    seconds = oracle_mod.keygen_hash128(leaf * 7 + m, m)[:, 1]
    seed = (0x9E3779B97F4A7C15 * (leaf + 1) + _FANOUT9_SEEDS[(leaf, m)] - 40) & (2**64 - 1)
    assert oracle_mod.search_aggr(seconds, leaf, seed) == 40
    assert oracle_mod.search_aggr(seconds, leaf, seed, simd=True) == 40
