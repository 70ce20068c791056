"""rsb_hash_strings_static: string hashing for callers that cannot allocate device memory.

Such callers (a plugin whose host process owns all device memory, or a serving thread that
must not call cudaMalloc) use this entry point, which stages its data in a fixed device
array inside the library instead of allocating. Its hashes must equal those of the
allocating entry point rsb_hash_strings, bit for bit, on consecutive calls that reuse the
same array. This file is collected last so a failure here cannot hide other results.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _keys(seed: int, n: int, lo: int, hi: int):
    rng = np.random.default_rng(seed)
    lens = rng.integers(lo, hi + 1, n)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    data = rng.integers(0, 256, int(offsets[-1]), dtype=np.uint8)
    return data, offsets


def test_static_hash_matches_allocating_entry_point_on_consecutive_calls():
    import gpurecsplit_b200 as rsb
    import torch

    torch.cuda.set_device(0)
    engine = rsb.Engine(0)
    try:
        # first call: keys up to 300 bytes (SpookyHash's block path from 192), about 600 KiB;
        # second call: more but shorter keys, so stale bytes of the first call lie beyond its data
        first = _keys(1, 4000, 0, 300)
        assert int(first[1][-1]) < (1 << 20)
        second = _keys(2, 20000, 10, 50)
        for keys in (first, second):
            got = rsb.hash_strings_static(keys)
            want = rsb.hash_strings(keys, engine)
            assert got.shape == want.shape
            assert np.array_equal(got, want)
    finally:
        engine.close()


def test_static_hash_rejects_oversized_input():
    import gpurecsplit_b200 as rsb

    data, offsets = _keys(3, 40000, 1, 4)  # more keys than the static array holds
    with pytest.raises(rsb.RSBError) as e:
        rsb.hash_strings_static((data, offsets))
    assert e.value.name == "BAD_ARG"
    big = (np.zeros(2 << 20, dtype=np.uint8), np.array([0, 2 << 20], dtype=np.uint64))  # 2 MiB key
    with pytest.raises(rsb.RSBError):
        rsb.hash_strings_static(big)
