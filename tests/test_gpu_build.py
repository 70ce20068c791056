"""GPU parity tests: every device build must be bit-identical to the oracle.

Mirrors the reference's GPU/SIMD equivalence grid (test/GPUandSIMDequivalence.cu:8-11) and
correctness grid (test/correctness.hpp:24-27) at sizes the scalar oracle finishes quickly,
compares full-size builds with committed oracle digests (tests/golden/golden_builds.json),
and covers the edge cases: empty and single-key sets, buckets of size 0/1, brute-force
leaves, duplicates, oversized buckets and exhausted search budgets. All calls go through
the C ABI (librsb.so via ctypes).
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SEED = 0x5603141978c51071
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_builds.json")


def _grid():
    out = []
    for leaf in range(2, 25):
        for b in (2, 5, 10, 25, 100, 483, 2000):
            if leaf >= 13 and b > 25:
                continue
            if leaf >= 19 and b > 10:
                continue
            for n in (1, 10, 100, 123, 2000):
                out.append((leaf, b, n))
    return out


def _build_both(rsb, oracle_mod, engine, keys, leaf, b, rot=True):
    ref = oracle_mod.build_mphf(keys, leaf, b, rot)
    f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, rotate=rot, engine=engine, keep_seeds=True)
    return ref, f


@pytest.mark.parametrize("leaf,b,n", _grid())
def test_equivalence_grid(rsb, oracle_mod, engine, leaf, b, n):
    keys = oracle_mod.keygen_hash128(SEED, n)
    ref, f = _build_both(rsb, oracle_mod, engine, keys, leaf, b)
    seeds, sizes = f.seeds()
    assert np.array_equal(sizes, ref.sizes)
    assert np.array_equal(seeds, ref.seeds)
    assert f.serialize() == ref.bytes.tobytes()
    q = f.query(keys)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


def _grid_other_buckets():
    """The remaining bucket sizes of the reference's correctness grid (test/correctness.hpp:25),
    with the same leaf-size limits as _grid."""
    out = []
    for leaf in range(2, 25):
        for b in (3, 4, 6, 7, 8, 9, 75, 231, 1009, 1300):
            if leaf >= 13 and b > 25:
                continue
            if leaf >= 19 and b > 10:
                continue
            for n in (100, 2000):
                out.append((leaf, b, n))
    return out


@pytest.mark.parametrize("leaf,b,n", _grid_other_buckets())
def test_equivalence_grid_other_buckets(rsb, oracle_mod, engine, leaf, b, n):
    keys = oracle_mod.keygen_hash128(SEED ^ b, n)
    ref, f = _build_both(rsb, oracle_mod, engine, keys, leaf, b)
    seeds, sizes = f.seeds()
    assert np.array_equal(sizes, ref.sizes)
    assert np.array_equal(seeds, ref.seeds)
    assert f.serialize() == ref.bytes.tobytes()


@pytest.mark.parametrize("leaf,b,n", [(8, 100, 100000), (12, 1000, 30000), (16, 2000, 12000), (10, 483, 20000),
                                      (6, 25, 50000), (14, 75, 20000), (4, 1009, 20000), (20, 10, 5000)])
def test_equivalence_larger(rsb, oracle_mod, engine, leaf, b, n):
    keys = oracle_mod.keygen_hash128(SEED + leaf, n)
    ref, f = _build_both(rsb, oracle_mod, engine, keys, leaf, b)
    seeds, _ = f.seeds()
    assert np.array_equal(seeds, ref.seeds)
    assert f.serialize() == ref.bytes.tobytes()


@pytest.mark.parametrize("leaf,b,n", [(8, 100, 20000), (5, 7, 5000), (12, 231, 5000), (16, 2000, 4000), (3, 2, 3000)])
def test_equivalence_bruteforce_leaves(rsb, oracle_mod, engine, leaf, b, n):
    keys = oracle_mod.keygen_hash128(SEED ^ leaf, n)
    ref, f = _build_both(rsb, oracle_mod, engine, keys, leaf, b, rot=False)
    assert f.serialize() == ref.bytes.tobytes()
    q = f.query(keys)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))


def test_empty_and_tiny_sets(rsb, oracle_mod, engine):
    for n in (0, 1, 2, 3):
        keys = oracle_mod.keygen_hash128(SEED, n)
        ref, f = _build_both(rsb, oracle_mod, engine, keys, 8, 100)
        assert f.serialize() == ref.bytes.tobytes()


def test_u64_keys_hash_like_oracle(rsb, oracle_mod, engine):
    k = oracle_mod.keygen_u64(42, 200000)
    assert np.array_equal(rsb.hash_u64(k, engine), oracle_mod.hash_u64(k))
    f = rsb.GPURecSplit(k, bucket_size=2000, leaf_size=16, key_type="u64", engine=engine)
    ref = oracle_mod.build_mphf(oracle_mod.hash_u64(k[:20000]), 16, 2000)
    g = rsb.GPURecSplit(k[:20000], bucket_size=2000, leaf_size=16, key_type="u64", engine=engine)
    assert g.serialize() == ref.bytes.tobytes()
    q = f.query(oracle_mod.hash_u64(k))
    assert np.array_equal(np.sort(q), np.arange(k.size, dtype=np.uint64))


def test_string_keys_hash_like_oracle(rsb, oracle_mod, engine):
    # lengths 0..400 cover SpookyHash's short (<192 bytes) and block paths
    rng = np.random.default_rng(5)
    lens = np.concatenate([np.arange(0, 401), rng.integers(10, 51, 3000)])
    offsets = np.zeros(lens.size + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    data = rng.integers(0, 256, int(offsets[-1]), dtype=np.uint8)
    assert np.array_equal(rsb.hash_strings((data, offsets), engine), oracle_mod.hash_strings(data, offsets))


@pytest.mark.parametrize("shift", [0, 1, 7, 15, 16, 33])
def test_string_hash_staging_paths(rsb, oracle_mod, engine, shift):
    """Warps of 32 keys whose bytes fit the per-warp staging buffer hash from shared memory,
    wider ones from global memory; both, at every start alignment (keys sliced `shift`
    bytes into a larger buffer), give the oracle's hashes."""
    rng = np.random.default_rng(100 + shift)
    lens = np.concatenate([rng.integers(0, 64, 3000),           # staged warps
                           rng.integers(60, 300, 200),          # warps wider than the buffer
                           np.zeros(40, dtype=np.int64),        # empty keys
                           rng.integers(0, 16, 1000)])          # short keys, one 16-byte block
    offsets = np.zeros(lens.size + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    body = rng.integers(0, 256, int(offsets[-1]), dtype=np.uint8)
    data = np.concatenate([rng.integers(0, 256, shift, dtype=np.uint8), body,
                           rng.integers(0, 256, 19, dtype=np.uint8)])
    want = oracle_mod.hash_strings(body, offsets)
    assert np.array_equal(rsb.hash_strings((data, offsets + np.uint64(shift)), engine), want)


def test_evaluation_statistic_matches_seeds(rsb, oracle_mod, engine):
    """The build's algorithmic evaluation count (used for the measured evaluation rates) is
    the sum over nodes of (candidates up to the seed) x (node size), candidates being
    rotation bases for full leaves."""
    for leaf, b, n in ((8, 100, 50_000), (12, 1000, 30_000), (16, 2000, 10_000)):
        keys = oracle_mod.keygen_hash128(SEED + 3 * leaf, n)
        f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=engine, keep_seeds=True)
        seeds, sizes = f.seeds()
        s = seeds.astype(object)
        m = sizes.astype(object)
        trials = [x // leaf + 1 if k == leaf else x + 1 for x, k in zip(s, m)]
        want = sum(t * k for t, k in zip(trials, m))
        st = f.stats()
        assert st["evals_alg"] == want
        assert sum(st["evals_stage"]) == want
        f.close()


def test_string_build_and_query(rsb, oracle_mod, engine):
    data, offsets = oracle_mod.keygen_strings(42, 50000)
    ref = oracle_mod.build_mphf(oracle_mod.hash_strings(data, offsets), 8, 100)
    f = rsb.GPURecSplit((data, offsets), bucket_size=100, leaf_size=8, key_type="strings", engine=engine)
    assert f.serialize() == ref.bytes.tobytes()
    q = f.query_strings((data, offsets))
    assert np.array_equal(np.sort(q), np.arange(50000, dtype=np.uint64))
    words = ["alpha", "beta", "gamma", "delta", "epsilon"]
    g = rsb.GPURecSplit(words, bucket_size=100, leaf_size=8, engine=engine)
    assert sorted(g(w) for w in words) == list(range(5))


def test_device_query_matches_host(rsb, oracle_mod, engine):
    import torch
    keys = oracle_mod.keygen_hash128(11, 300000)
    f = rsb.GPURecSplit(keys, bucket_size=1000, leaf_size=12, engine=engine)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    out = torch.empty(keys.shape[0], dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    f.query_device(dk.data_ptr(), keys.shape[0], out.data_ptr(), engine)
    dev = out.cpu().numpy().view(np.uint64)
    assert np.array_equal(dev, f.query(keys))
    assert np.array_equal(np.sort(dev), np.arange(keys.shape[0], dtype=np.uint64))


def test_device_resident_build_matches_host_input(rsb, oracle_mod, engine):
    import torch
    keys = oracle_mod.keygen_hash128(12, 100000)
    a = rsb.GPURecSplit(keys, bucket_size=100, leaf_size=8, engine=engine)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    torch.cuda.synchronize()
    b = rsb.GPURecSplit.from_device(dk.data_ptr(), keys.shape[0], 100, 8, engine=engine)
    assert a.serialize() == b.serialize()


def test_engine_reuse_across_shapes(rsb, oracle_mod, engine):
    cases = [(20000, 8, 100), (3000, 16, 2000), (500, 3, 5), (20000, 8, 100), (100, 24, 5)]
    for n, leaf, b in cases:
        keys = oracle_mod.keygen_hash128(n + leaf, n)
        ref = oracle_mod.build_mphf(keys, leaf, b)
        f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=engine)
        assert f.serialize() == ref.bytes.tobytes()


def test_roundtrip_serialization(rsb, oracle_mod, engine):
    keys = oracle_mod.keygen_hash128(13, 50000)
    f = rsb.GPURecSplit(keys, bucket_size=2000, leaf_size=12, engine=engine)
    blob = f.serialize()
    g = rsb.GPURecSplit.deserialize(blob, 12)
    assert np.array_equal(f.query(keys), g.query(keys))
    assert g.serialize() == blob


# ---- failure detection (made on the host: no GPU fault, trap or hang) -----------------

def test_duplicate_keys_rejected(rsb, oracle_mod, engine):
    keys = oracle_mod.keygen_hash128(SEED, 5000)
    keys[4000] = keys[17]
    with pytest.raises(rsb.RSBError) as e:
        rsb.GPURecSplit(keys, bucket_size=100, leaf_size=8, engine=engine)
    assert e.value.name == "DUPLICATE_KEY"
    # the engine stays usable
    f = rsb.GPURecSplit(keys[:3000], bucket_size=100, leaf_size=8, engine=engine)
    assert f.get_bits() > 0


@pytest.mark.parametrize("b", [100, 1000, 2000])
def test_duplicates_in_small_and_large_buckets(rsb, oracle_mod, engine, b):
    """Buckets of at most 256 keys are checked by one warp each, larger ones by a CTA; both
    find a repeated key, a repeated empty-slot marker (second half all ones) and nothing in
    keys that only share a table slot."""
    keys = oracle_mod.keygen_hash128(SEED + b, 20_000)
    same_slot = keys.copy()
    same_slot[5, 0] = same_slot[9, 0]                    # same bucket, second halves that
    same_slot[5, 1] = same_slot[9, 1] ^ (1 << 40)        # differ only above the slot bits
    f = rsb.GPURecSplit(same_slot, bucket_size=b, leaf_size=8, engine=engine)
    assert f.serialize() == oracle_mod.build_mphf(same_slot, 8, b).bytes.tobytes()
    one_marker = keys.copy()
    one_marker[7, 1] = np.uint64(0xFFFFFFFFFFFFFFFF)
    f = rsb.GPURecSplit(one_marker, bucket_size=b, leaf_size=8, engine=engine)
    assert f.serialize() == oracle_mod.build_mphf(one_marker, 8, b).bytes.tobytes()
    two_markers = one_marker.copy()
    two_markers[11] = two_markers[7]
    repeated = keys.copy()
    repeated[19_000] = repeated[3]
    for bad in (two_markers, repeated):
        with pytest.raises(rsb.RSBError) as e:
            rsb.GPURecSplit(bad, bucket_size=b, leaf_size=8, engine=engine)
        assert e.value.name == "DUPLICATE_KEY"


def test_oversized_bucket_rejected(rsb, oracle_mod, engine):
    keys = oracle_mod.keygen_hash128(SEED, 7000)
    with pytest.raises(rsb.RSBError) as e:
        rsb.GPURecSplit(keys, bucket_size=3500, leaf_size=8, engine=engine)
    assert e.value.name == "BUCKET_TOO_LARGE"


def test_search_budget_exhaustion_is_reported(rsb, oracle_mod):
    e = rsb.Engine(0)
    try:
        e.set_budget(0, 4)  # at most max(2^g, 4) candidates per node: most searches fail
        keys = oracle_mod.keygen_hash128(SEED, 20000)
        with pytest.raises(rsb.RSBError) as err:
            rsb.GPURecSplit(keys, bucket_size=2000, leaf_size=16, engine=e)
        assert err.value.name == "SEARCH_BUDGET"
        e.set_budget(10, 1 << 16)
        keys = oracle_mod.keygen_hash128(SEED, 3000)
        ref = oracle_mod.build_mphf(keys, 8, 100)
        assert rsb.GPURecSplit(keys, bucket_size=100, leaf_size=8, engine=e).serialize() == ref.bytes.tobytes()
    finally:
        e.close()


@pytest.mark.parametrize("pipeline", [False, True], ids=["stages", "pipeline"])
def test_failed_builds_with_small_nodes_write_nothing(rsb, oracle_mod, pipeline):
    """A build that fails once its searches are under way (here a duplicate key) leaves seeds
    unfound. At l=2 every node has Golomb-Rice parameter 0, and the unary code of an unfound
    seed would start one bit before its bucket's stream (bit -1 for bucket 0): the encoder
    must write nothing, the build must report the failure, plain and batched, and the engine
    must stay usable."""
    e = rsb.Engine(0)
    try:
        e.set_pipeline(pipeline)
        e.set_watchdog(20)
        keys = oracle_mod.keygen_hash128(SEED + 2, 5000)
        dup = keys.copy()
        dup[4000] = dup[1017]  # both in the third set of the batch below
        with pytest.raises(rsb.RSBError) as err:
            rsb.GPURecSplit(dup, bucket_size=2, leaf_size=2, engine=e)
        assert err.value.name == "DUPLICATE_KEY"
        offsets = np.array([0, 1000, 1000, 5000], dtype=np.uint64)
        with pytest.raises(rsb.RSBError) as err:
            rsb.build_batch(dup, offsets, 2, 2, engine=e)
        assert err.value.name == "DUPLICATE_KEY"
        assert rsb.GPURecSplit(keys, bucket_size=2, leaf_size=2, engine=e).serialize() == \
            oracle_mod.build_mphf(keys, 2, 2).bytes.tobytes()
    finally:
        e.close()


def test_bad_arguments(rsb, engine):
    keys = np.zeros((10, 2), dtype=np.uint64)
    for leaf, b in ((1, 100), (25, 100), (8, 0)):
        with pytest.raises(rsb.RSBError) as e:
            rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=engine)
        assert e.value.name == "BAD_ARG"


# ---- full-size workloads against committed oracle digests ----------------------------

def _golden():
    return json.load(open(GOLDEN)) if os.path.exists(GOLDEN) else {}


def _keys(oracle_mod, kind, seed, n):
    if kind == "hash128":
        return ("hash128", oracle_mod.keygen_hash128(seed, n))
    if kind == "u64":
        return ("u64", oracle_mod.keygen_u64(seed, n))
    return ("strings", oracle_mod.keygen_strings(seed, n))


GOLDEN_NAMES = ["hash128_n100k_l12_b1000", "hash128_n50k_l8_b2000_bf", "u64_n100k_l16_b2000", "hash128_n1M_l8_b100",
                "strings_n1M_l8_b100", "u64_n5M_l16_b2000", "u64_n200k_l24_b2000", "u64_n5M_l18_b50",
                "hash128_n1M_l8_b2", "hash128_n1M_l8_b5", "hash128_n1M_l5_b10", "hash128_n12345678_l8_b100",
                "hash128_n10M_l4_b25", "hash128_n10M_l2_b2"]


@pytest.mark.parametrize("name", GOLDEN_NAMES)
def test_golden_digest(rsb, oracle_mod, engine, name):
    """Full-size device builds against digests of the reference's own SIMDRecSplit builds;
    the reference's operator>> and operator() (oracle/_ref) then read the device's function
    as a bijection onto [0, n), key by key equal to this library's query."""
    g = _golden().get(name)
    if g is None:
        pytest.skip(f"no committed digest for {name}")
    kind, keys = _keys(oracle_mod, g["kind"], g["seed"], g["n"])
    f = rsb.GPURecSplit(keys, bucket_size=g["bucket"], leaf_size=g["leaf"], rotate=g["rotate"], key_type=kind,
                        engine=engine)
    blob = f.serialize()
    assert len(blob) == g["bytes"]
    assert hashlib.sha256(blob).hexdigest() == g["sha256"]
    assert hashlib.sha256(blob).hexdigest() == g.get("ref_sha256", g["sha256"])
    assert f.get_bits(object_bytes=224 if "ref_sha256" in g else 0) == g["bits"]  # getBits() of the reference, object size included
    if oracle_mod.ref_available():
        k128 = keys if kind == "hash128" else (oracle_mod.hash_u64(keys) if kind == "u64"
                                              else oracle_mod.hash_strings(*keys))
        ref_vals = oracle_mod.ref_query(np.frombuffer(blob, dtype=np.uint8), g["leaf"], k128, g["rotate"])
        assert np.array_equal(np.sort(ref_vals), np.arange(g["n"], dtype=np.uint64))
        assert np.array_equal(ref_vals, f.query(k128))


def test_string_keys_as_slice_of_larger_buffer(rsb, oracle_mod, engine):
    """offsets[0] > 0: only bytes [offsets[0], offsets[n]) belong to the keys."""
    data, offsets = oracle_mod.keygen_strings(77, 30_000)
    lo, hi = 10_000, 25_000
    sl = offsets[lo:hi + 1]
    rebased = (data[int(sl[0]):int(sl[-1])].copy(), sl - sl[0])
    a = rsb.GPURecSplit((data, sl), bucket_size=100, leaf_size=8, key_type="strings", engine=engine)
    b = rsb.GPURecSplit(rebased, bucket_size=100, leaf_size=8, key_type="strings", engine=engine)
    assert a.serialize() == b.serialize()
    assert np.array_equal(rsb.hash_strings((data, sl), engine=engine), oracle_mod.hash_strings(*rebased))
    funcs, _ = rsb.build_batch((data, sl), np.array([0, 5000, hi - lo], dtype=np.uint64), 100, 8,
                               key_type="strings", engine=engine)
    first = (rebased[0], rebased[1][:5001])
    assert funcs[0].serialize() == rsb.GPURecSplit(first, bucket_size=100, leaf_size=8, key_type="strings",
                                                   engine=engine).serialize()


@pytest.mark.parametrize("pct", [25, 75])
def test_reduced_occupancy_same_function(rsb, oracle_mod, pct):
    """Persistent kernels with fewer resident CTAs find the same minimum seeds."""
    eng = rsb.Engine(0)
    eng.set_occupancy(pct)
    keys = oracle_mod.keygen_hash128(pct, 60_000)
    f = rsb.GPURecSplit(keys, bucket_size=2000, leaf_size=16, engine=eng)
    assert f.serialize() == oracle_mod.build_mphf(keys, 16, 2000).bytes.tobytes()
    eng.close()


@pytest.mark.parametrize("leaf,b,n,kind", [(8, 100, 200_000, "hash128"), (16, 2000, 40_000, "u64"),
                                           (12, 7, 30_000, "hash128"), (24, 2000, 500, "hash128"),
                                           (5, 100, 0, "hash128"), (8, 100, 1, "hash128"), (10, 50, 20_000, "strings")])
def test_verified_builds(rsb, oracle_mod, engine, leaf, b, n, kind):
    """RSB_VERIFY: the device decodes every bucket's Elias-Fano entry and checks the bijection
    of all keys before returning; the function is the same as without verification."""
    if kind == "hash128":
        keys = oracle_mod.keygen_hash128(n + leaf, n)
    elif kind == "u64":
        keys = oracle_mod.keygen_u64(n + leaf, n)
    else:
        keys = oracle_mod.keygen_strings(n + leaf, n)
    f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, key_type=kind, engine=engine, verify=True)
    g = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, key_type=kind, engine=engine)
    assert f.serialize() == g.serialize()
