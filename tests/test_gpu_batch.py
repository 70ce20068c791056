"""Batched construction: every set of one batched pipeline must equal its plain build.

Uneven set sizes (empty, single-key, tiny, large), both key types, rotation on and off,
and the failure path (a duplicate key in one set fails the batch cleanly)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sets(rng, sizes):
    offsets = np.zeros(len(sizes) + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(sizes)
    return offsets


@pytest.mark.parametrize("leaf,b,rot", [(8, 100, True), (12, 1000, True), (5, 7, False), (16, 2000, True), (2, 2, True)])
def test_batch_equals_plain_builds(rsb, oracle_mod, engine, leaf, b, rot):
    rng = np.random.default_rng(leaf * 131 + b)
    sizes = [0, 1, 2, 3, 17, 100, 999, 1000, 1001] + list(
        np.exp(rng.uniform(np.log(10), np.log(20000), 40)).astype(int))
    if leaf >= 16:
        sizes = [s for s in sizes if s <= 6000]
    offsets = _sets(rng, sizes)
    keys = oracle_mod.keygen_hash128(leaf + b, int(offsets[-1]))
    funcs, stats = rsb.build_batch(keys, offsets, b, leaf, rotate=rot, engine=engine)
    assert len(funcs) == len(sizes)
    assert stats["keys"] == offsets[-1]
    for s, f in enumerate(funcs):
        part = keys[offsets[s]:offsets[s + 1]]
        plain = rsb.GPURecSplit(part, bucket_size=b, leaf_size=leaf, rotate=rot, engine=engine)
        assert f.serialize() == plain.serialize(), f"set {s} (n={len(part)}) differs"
        if len(part):
            q = f.query(part)
            assert np.array_equal(np.sort(q), np.arange(len(part), dtype=np.uint64))


def test_batch_matches_oracle(rsb, oracle_mod, engine):
    sizes = [5000, 1, 0, 12345, 777]
    offsets = _sets(None, sizes)
    keys = oracle_mod.keygen_hash128(99, int(offsets[-1]))
    funcs, _ = rsb.build_batch(keys, offsets, 1000, 12, engine=engine)
    for s, f in enumerate(funcs):
        ref = oracle_mod.build_mphf(keys[offsets[s]:offsets[s + 1]], 12, 1000)
        assert f.serialize() == ref.bytes.tobytes()


def test_batch_u64_keys(rsb, oracle_mod, engine):
    rng = np.random.default_rng(3)
    sizes = list(np.exp(rng.uniform(np.log(1000), np.log(100000), 30)).astype(int))
    offsets = _sets(rng, sizes)
    keys = oracle_mod.keygen_u64(1234, int(offsets[-1]))
    funcs, stats = rsb.build_batch(keys, offsets, 1000, 12, key_type="u64", engine=engine)
    assert stats["kernel_launches"] > 0
    for s in (0, 7, 29):
        part = keys[offsets[s]:offsets[s + 1]]
        plain = rsb.GPURecSplit(part, bucket_size=1000, leaf_size=12, key_type="u64", engine=engine)
        assert funcs[s].serialize() == plain.serialize()


def test_batch_duplicate_fails_cleanly(rsb, oracle_mod, engine):
    offsets = _sets(None, [1000, 2000, 500])
    keys = oracle_mod.keygen_hash128(5, 3500)
    keys[2500] = keys[1500]  # inside the second set
    with pytest.raises(rsb.RSBError) as e:
        rsb.build_batch(keys, offsets, 100, 8, engine=engine)
    assert e.value.name == "DUPLICATE_KEY"
    funcs, _ = rsb.build_batch(keys[:1000], offsets[:2], 100, 8, engine=engine)
    assert len(funcs) == 1


def test_batch_rejects_bad_offsets(rsb, engine):
    keys = np.zeros((10, 2), dtype=np.uint64)
    for bad in ([1, 10], [0, 6, 4, 10]):
        with pytest.raises(rsb.RSBError) as e:
            rsb.build_batch(keys, np.array(bad, dtype=np.uint64), 100, 8, engine=engine)
        assert e.value.name == "BAD_ARG"
