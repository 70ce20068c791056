"""Device builds against the reference's own SIMDRecSplit (oracle/_ref), through the C ABI.

oracle/_ref/libref_simdrs.so is GpuRecSplit's SIMDRecSplit compiled from its unmodified
sources; here it runs on the GPU box's host cores. Every device build must equal the
reference's build byte for byte over the equivalence grid (test/GPUandSIMDequivalence.cu:8-11,
sizes capped by leaf size), the reference's encoders (RiceBitVector::Builder, DoubleEF) must
turn the device's DFS seeds into the device's bytes, and the reference's operator>> and
operator() must read device-built functions - plain and batched - as bijections onto [0, n)
equal key by key to this library's query.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
SEED = 0x5603141978c51071


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if not oracle_mod.ref_available():
        pytest.skip("oracle/_ref was not built or this CPU lacks AVX-512")
    return oracle_mod


def _sizes(leaf):
    if leaf > 20:
        return (1, 10, 123)
    if leaf > 14:
        return (1, 10, 100, 123)
    return (1, 10, 100, 123, 2000)


@pytest.mark.parametrize("leaf", range(2, 25))
def test_device_equals_reference(rsb, ref, engine, leaf):
    for b in (2, 5, 10, 25, 100, 483, 2000):
        for n in _sizes(leaf):
            keys = ref.keygen_hash128(SEED + 77 * leaf + n, n)
            f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=engine, keep_seeds=True)
            blob = np.frombuffer(f.serialize(), dtype=np.uint8)
            if n == 0:
                continue
            assert np.array_equal(blob, ref.ref_build(keys, leaf, b)), (leaf, b, n)
            seeds, sizes = f.seeds()
            bucket_keys = np.bincount(_bucket_of(keys, b), minlength=max(1, -(-n // b)))
            assert np.array_equal(ref.ref_encode(bucket_keys, b, leaf, seeds, sizes), blob), (leaf, b, n)


def _bucket_of(keys, b):
    """remap128(first, nbuckets) of every key (support/common.hpp:273-280)."""
    n = keys.shape[0]
    nb = max(1, -(-n // b))
    return np.array([(int(k) * nb) >> 64 for k in keys[:, 0]], dtype=np.int64)


@pytest.mark.parametrize("leaf,b,n,rot", [(8, 100, 200_000, True), (12, 1000, 100_000, True), (16, 2000, 30_000, True),
                                          (10, 7, 50_000, False), (24, 2000, 300, True)])
def test_reference_reads_device_functions(rsb, ref, engine, leaf, b, n, rot):
    keys = ref.keygen_hash128(SEED ^ (leaf * n), n)
    f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, rotate=rot, engine=engine, keep_seeds=True)
    blob = np.frombuffer(f.serialize(), dtype=np.uint8)
    vals = ref.ref_query(blob, leaf, keys, rot)
    assert np.array_equal(np.sort(vals), np.arange(n, dtype=np.uint64))
    assert np.array_equal(vals, f.query(keys))
    seeds, sizes = f.seeds()
    bucket_keys = np.bincount(_bucket_of(keys, b), minlength=max(1, -(-n // b)))
    assert np.array_equal(ref.ref_encode(bucket_keys, b, leaf, seeds, sizes, rot), blob)


def test_reference_reads_batched_functions(rsb, ref, engine):
    rng = np.random.default_rng(3)
    sizes = np.rint(np.exp(rng.uniform(np.log(1), np.log(40_000), 60))).astype(np.int64)
    sizes[:3] = (0, 1, 2)
    offsets = np.zeros(sizes.size + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(sizes)
    keys = ref.keygen_hash128(99, int(offsets[-1]))
    funcs, _ = rsb.build_batch(keys, offsets, 1000, 12, engine=engine)
    for s, f in enumerate(funcs):
        lo, hi = int(offsets[s]), int(offsets[s + 1])
        blob = np.frombuffer(f.serialize(), dtype=np.uint8)
        if hi - lo >= 1:
            vals = ref.ref_query(blob, 12, keys[lo:hi])
            assert np.array_equal(np.sort(vals), np.arange(hi - lo, dtype=np.uint64)), s
        if hi - lo >= 1 and s % 6 == 0:
            assert np.array_equal(blob, ref.ref_build(keys[lo:hi], 12, 1000)), s
