"""Pipeline mode (rsb_engine_set_pipeline): the aggregation and leaf searches of a build in
one persistent launch with device work queues, each node searched as soon as its parent is
partitioned. It must build exactly the functions the stage-by-stage kernels build: the
equivalence grid against the oracle, larger builds, both leaf methods, batched sets, and
full-size digests of the reference's builds."""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
SEED = 0x5603141978c51071
GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "golden_builds.json")


@pytest.fixture(scope="module")
def pipe(rsb):
    e = rsb.Engine(0)
    e.set_pipeline(True)
    e.set_watchdog(120)  # a build of these tests takes well under a second
    yield e
    e.close()


@pytest.mark.parametrize("leaf", range(2, 25))
def test_pipeline_grid(rsb, oracle_mod, pipe, leaf):
    sizes = (1, 10, 100, 123, 2000) if leaf <= 16 else (1, 10, 123)
    for b in (2, 5, 10, 100, 2000):
        for n in sizes:
            keys = oracle_mod.keygen_hash128(SEED + 3 * leaf + n, n)
            f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=pipe)
            assert f.serialize() == oracle_mod.build_mphf(keys, leaf, b).bytes.tobytes(), (leaf, b, n)


@pytest.mark.parametrize("leaf,b,n,rot", [(8, 100, 200_000, True), (12, 1000, 150_000, True), (16, 2000, 40_000, True),
                                          (10, 300, 50_000, False), (5, 7, 30_000, True), (20, 2000, 2_000, True)])
def test_pipeline_larger(rsb, oracle_mod, engine, pipe, leaf, b, n, rot):
    keys = oracle_mod.keygen_hash128(SEED ^ (n + leaf), n)
    f = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, rotate=rot, engine=pipe, verify=True)
    g = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, rotate=rot, engine=engine)
    assert f.serialize() == g.serialize()


def test_pipeline_batched(rsb, oracle_mod, engine, pipe):
    rng = np.random.default_rng(21)
    sizes = np.rint(np.exp(rng.uniform(np.log(1), np.log(60_000), 120))).astype(np.int64)
    sizes[:3] = (0, 1, 2)
    offsets = np.zeros(sizes.size + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(sizes)
    keys = oracle_mod.keygen_hash128(77, int(offsets[-1]))
    a, _ = rsb.build_batch(keys, offsets, 1000, 12, engine=pipe)
    b, _ = rsb.build_batch(keys, offsets, 1000, 12, engine=engine)
    assert all(x.serialize() == y.serialize() for x, y in zip(a, b))


@pytest.mark.parametrize("name", ["hash128_n1M_l8_b100", "u64_n100k_l16_b2000", "hash128_n100k_l12_b1000",
                                  "u64_n5M_l16_b2000"])
def test_pipeline_golden(rsb, oracle_mod, pipe, name):
    g = json.load(open(GOLDEN))[name]
    if g["kind"] == "hash128":
        keys, kind = oracle_mod.keygen_hash128(g["seed"], g["n"]), "hash128"
    else:
        keys, kind = oracle_mod.keygen_u64(g["seed"], g["n"]), "u64"
    f = rsb.GPURecSplit(keys, bucket_size=g["bucket"], leaf_size=g["leaf"], rotate=g["rotate"], key_type=kind,
                        engine=pipe)
    assert hashlib.sha256(f.serialize()).hexdigest() == g["sha256"]


def test_pipeline_watchdog_runs_out(rsb, oracle_mod):
    """A launch that outlives the engine's watchdog stops with RSB_ERR_TIMEOUT (every warp
    leaves at its next step; no fault, no hang) and the engine builds correctly afterwards."""
    e = rsb.Engine(0)
    try:
        e.set_pipeline(True)
        keys = oracle_mod.keygen_hash128(SEED + 99, 200_000)
        e.set_watchdog(1e-6)  # 1 us: far shorter than any launch of 200k keys
        with pytest.raises(rsb.RSBError) as err:
            rsb.GPURecSplit(keys, bucket_size=2000, leaf_size=16, engine=e)
        assert err.value.name == "TIMEOUT"
        e.set_watchdog(0)
        small = keys[:20_000]
        assert rsb.GPURecSplit(small, bucket_size=100, leaf_size=8, engine=e).serialize() == \
            oracle_mod.build_mphf(small, 8, 100).bytes.tobytes()
    finally:
        e.close()
