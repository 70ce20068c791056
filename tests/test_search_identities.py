"""Integer identities the seed-search kernels rely on, checked on the host with numpy:

* the part index of a non-full aggregation node, ((hash16 * m) >> 16) / SPLIT, equals
  umulhi(hash16 << 16, ceil(m * 2^28 / SPLIT)) >> 28 for every 16-bit hash, every node size of
  both aggregation stages and every leaf size (add_part in rsb_search.cu);
* the per-key term of remix32's first round: when the low 16 bits L of key + window base cannot
  overflow inside the window, (hi ^ lo) ^ (hi ^ lo) >> 16 of the candidate key + base + j is
  (L + j) ^ K' with K' = hi ^ hi >> 16 ^ lo >> 16 ^ (lo & 0xFFFF0000) (moment_sums and
  left_masks), for aggregation windows (offsets 0..32*S-1) and rotation-leaf windows
  (offsets (lane + 32 s) * LEAF).

Aggregation sizes follow AbstractParallelRecSplit.hpp:133,135 (lower_aggr, upper_aggr)."""
import math

import numpy as np
import pytest

M32 = np.uint64(0xFFFFFFFF)


def lower_aggr(leaf: int) -> int:
    return leaf * max(2, math.ceil(0.35 * leaf + 1.0 / 2))


def upper_aggr(leaf: int) -> int:
    return lower_aggr(leaf) * (2 if leaf < 7 else math.ceil(0.21 * leaf + 9.0 / 10))


def test_aggregation_sizes_match_known_values():
    assert (lower_aggr(8), upper_aggr(8)) == (32, 96)
    assert (lower_aggr(12), upper_aggr(12)) == (60, 240)
    assert (lower_aggr(16), upper_aggr(16)) == (112, 560)
    assert (lower_aggr(24), upper_aggr(24)) == (216, 1296)


@pytest.mark.parametrize("leaf", range(2, 25))
def test_nonfull_part_index_multiplier(leaf):
    h = np.arange(1 << 16, dtype=np.uint64)
    b = h << np.uint64(16)
    for split, maxm in ((leaf, lower_aggr(leaf)), (lower_aggr(leaf), upper_aggr(leaf))):
        assert maxm < 16 * split  # mult stays below 2^32
        for m in range(1, maxm + 1):
            mult = ((m << 28) + split - 1) // split
            assert mult < (1 << 32)
            got = ((b * np.uint64(mult)) >> np.uint64(32)) >> np.uint64(28)
            want = ((h * np.uint64(m)) >> np.uint64(16)) // np.uint64(split)
            assert np.array_equal(got, want), (leaf, split, m)


def _first_round(v: np.ndarray) -> np.ndarray:
    x = (v >> np.uint64(32)) ^ (v & M32)
    return x ^ (x >> np.uint64(16))


def _check_window(tu: np.ndarray, offsets: np.ndarray, span: int):
    lo = tu & M32
    hi = tu >> np.uint64(32)
    fast = (lo & np.uint64(0xFFFF)) <= np.uint64(0x10000 - span)
    tu, lo, hi = tu[fast], lo[fast], hi[fast]
    kp = hi ^ (hi >> np.uint64(16)) ^ (lo >> np.uint64(16)) ^ (lo & np.uint64(0xFFFF0000))
    L = lo & np.uint64(0xFFFF)
    for j in offsets:
        j = np.uint64(j)
        got = (L + j) ^ kp
        want = _first_round(tu + j)  # 64-bit wrap of key + base + j
        assert np.array_equal(got, want)
    return int(fast.sum())


def _keys(n: int, seed: int, span: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    tu = rng.integers(0, 1 << 63, size=n, dtype=np.uint64) * np.uint64(2) + rng.integers(0, 2, size=n, dtype=np.uint64)
    # boundary cases: the last fast low half, the first slow one, and a carry into the high word
    edge = np.array([0x10000 - span, 0x10000 - span + 1, 0xFFFF, 0, 0xFFFFFFFF, 0xFFFFFFFFFFFF0000 | (0x10000 - span)],
                    dtype=np.uint64)
    hi_rand = rng.integers(0, 1 << 63, size=len(edge), dtype=np.uint64) << np.uint64(1)
    edge = np.where(edge > M32, edge, (hi_rand & ~np.uint64(0xFFFF)) | edge)
    return np.concatenate([tu, edge])


@pytest.mark.parametrize("seeds_per_lane", [8, 12])
def test_aggregation_window_key_terms(seeds_per_lane):
    span = 32 * seeds_per_lane
    tu = _keys(4000, 7 + seeds_per_lane, span)
    assert _check_window(tu, np.arange(span), span) > 3500


@pytest.mark.parametrize("leaf", [2, 5, 8, 12, 16, 20, 24])
def test_leaf_window_key_terms(leaf):
    s = 8
    span = 32 * s * leaf
    offsets = np.array([(lane + 32 * k) * leaf for lane in range(32) for k in range(s)])
    tu = _keys(1500, 100 + leaf, span)
    assert _check_window(tu, offsets, span) > 1000
