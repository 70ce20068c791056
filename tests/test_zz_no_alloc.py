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


def test_static_hash_of_a_slice_deep_inside_a_larger_buffer():
    """offsets[0] > 0: only bytes[offsets[0] .. offsets[n]) is read and counted against the
    1 MiB limit, as in rsb_hash_strings, so a window past the first MiB of a buffer works."""
    import gpurecsplit_b200 as rsb
    import torch

    torch.cuda.set_device(0)
    engine = rsb.Engine(0)
    try:
        data, offsets = _keys(4, 60000, 10, 50)  # about 1.8 MiB of key bytes in all
        lo, hi = 40000, 45000
        window = offsets[lo:hi + 1]
        assert int(window[0]) > (1 << 20) and int(window[-1] - window[0]) < (1 << 20)
        for _ in range(2):
            got = rsb.hash_strings_static((data, window))
            want = rsb.hash_strings((data, window), engine)
            assert np.array_equal(got, want)
    finally:
        engine.close()


def test_static_hash_refuses_a_capturing_stream():
    """The call copies through pageable memory and waits for its stream, so while that
    stream is being captured it returns BAD_ARG before doing any work."""
    import gpurecsplit_b200 as rsb
    import torch

    torch.cuda.set_device(0)
    keys = _keys(5, 100, 10, 20)
    rsb.hash_strings_static(keys)  # first call on the device: resolves the array before capture
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    x = torch.zeros(16, device="cuda")
    refused = None
    with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
        x.add_(1)  # the captured work of the graph; the hashing call adds none
        try:
            rsb.hash_strings_static(keys, stream=s.cuda_stream)
        except rsb.RSBError as e:
            refused = e.name
    assert refused == "BAD_ARG"
    g.replay()
    torch.cuda.synchronize()
    assert float(x.sum()) == 16.0
    del g
    torch.cuda.synchronize()
    assert np.array_equal(rsb.hash_strings_static(keys), rsb.hash_strings(keys))


def test_static_hash_rejects_oversized_input():
    import gpurecsplit_b200 as rsb

    data, offsets = _keys(3, 40000, 1, 4)  # more keys than the static array holds
    with pytest.raises(rsb.RSBError) as e:
        rsb.hash_strings_static((data, offsets))
    assert e.value.name == "BAD_ARG"
    big = (np.zeros(2 << 20, dtype=np.uint8), np.array([0, 2 << 20], dtype=np.uint64))  # 2 MiB key
    with pytest.raises(rsb.RSBError):
        rsb.hash_strings_static(big)
