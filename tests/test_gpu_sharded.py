"""Bucket-range sharding on the GPU: parts built over contiguous bucket ranges
(rsb_build_part_hash128), exported (rsb_part_export) and merged (rsb_merge_parts) equal the
plain build of all keys byte for byte, for any number of parts; malformed or non-tiling
parts are rejected; and the torch.distributed flow (gpurecsplit_b200/sharded.py) with two
gloo ranks, each building its part on cuda:0 (independent builds, no rank waits on a device
for another), returns the plain function on the root."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from gpurecsplit_b200 import sharded

pytestmark = pytest.mark.gpu


def _remap128(first: np.ndarray, nb: int) -> np.ndarray:
    hi = first >> np.uint64(32)
    lo = first & np.uint64(0xFFFFFFFF)
    nbu = np.uint64(nb)
    return ((hi * nbu + ((lo * nbu) >> np.uint64(32))) >> np.uint64(32)).astype(np.int64)


def _parts(rsb, keys, b, leaf, nparts, rotate=True, engine=None, shuffle_seed=0):
    nb = sharded.num_buckets(keys.shape[0], b)
    ids = _remap128(keys[:, 0], nb)
    rng = np.random.default_rng(shuffle_seed)
    out = []
    for lo, hi in sharded.bucket_ranges(nb, nparts):
        if hi == lo:
            continue
        mine = keys[(ids >= lo) & (ids < hi)]
        mine = mine[rng.permutation(mine.shape[0])]  # any key order within a part
        out.append(rsb.build_part(mine, nb, lo, hi, b, leaf, rotate, engine))
    return out


@pytest.mark.parametrize("leaf,b,n,nparts", [(8, 100, 100_000, 1), (8, 100, 100_000, 4), (16, 2000, 60_000, 3),
                                             (12, 1000, 77_777, 8), (5, 2, 20_000, 5), (24, 2000, 300, 2),
                                             (8, 100, 150, 7), (3, 10, 1, 2), (8, 100, 0, 2)])
def test_parts_merge_into_the_plain_function(rsb, oracle_mod, engine, leaf, b, n, nparts):
    keys = oracle_mod.keygen_hash128(31 * n + nparts, n)
    plain = rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, engine=engine).serialize()
    merged = rsb.merge_parts(_parts(rsb, keys, b, leaf, nparts, engine=engine), leaf, engine=engine)
    assert merged.serialize() == plain
    q = merged.query(keys)
    assert np.array_equal(np.sort(q), np.arange(n, dtype=np.uint64))
    if oracle_mod.ref_available() and n > 0:  # n = 0: the reference's one undefined field differs
        assert plain == oracle_mod.ref_build(keys, leaf, b).tobytes()


def test_parts_without_rotation(rsb, oracle_mod, engine):
    keys = oracle_mod.keygen_hash128(5, 30_000)
    plain = rsb.GPURecSplit(keys, bucket_size=500, leaf_size=10, rotate=False, engine=engine).serialize()
    merged = rsb.merge_parts(_parts(rsb, keys, 500, 10, 3, rotate=False, engine=engine), 10, rotate=False,
                             engine=engine)
    assert merged.serialize() == plain


def test_part_rejects_keys_outside_its_range(rsb, oracle_mod, engine):
    keys = oracle_mod.keygen_hash128(6, 10_000)
    nb = sharded.num_buckets(10_000, 100)
    with pytest.raises(rsb.RSBError) as e:
        rsb.build_part(keys, nb, 0, nb // 2, 100, 8, engine=engine)  # holds keys of the upper half too
    assert e.value.name == "BAD_ARG"


def test_merge_rejects_gaps_overlaps_and_corruption(rsb, oracle_mod, engine):
    keys = oracle_mod.keygen_hash128(7, 20_000)
    parts = _parts(rsb, keys, 100, 8, 3, engine=engine)
    for bad in ([parts[0], parts[2]], [parts[0], parts[0], parts[1], parts[2]], [parts[1], parts[0], parts[2]]):
        with pytest.raises(rsb.RSBError) as e:
            rsb.merge_parts(bad, 8, engine=engine)
        assert e.value.name == "BAD_ARG"
    broken = bytearray(parts[1])
    broken[0] ^= 1  # magic
    with pytest.raises(rsb.RSBError) as e:
        rsb.merge_parts([parts[0], bytes(broken), parts[2]], 8, engine=engine)
    assert e.value.name == "FORMAT"
    with pytest.raises(rsb.RSBError) as e:
        rsb.merge_parts([parts[0], parts[1][:-8], parts[2]], 8, engine=engine)
    assert e.value.name == "FORMAT"
    with pytest.raises(rsb.RSBError) as e:
        rsb.merge_parts(parts, 12, engine=engine)  # the parts have leaf size 8
    assert e.value.name == "BAD_ARG"
    assert rsb.merge_parts(parts, 8, engine=engine).serialize() == \
        rsb.GPURecSplit(keys, bucket_size=100, leaf_size=8, engine=engine).serialize()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out, n_per_rank):
    import datetime

    import torch
    import torch.distributed as dist

    import gpurecsplit_b200 as rsb
    import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        torch.cuda.set_device(0)
        local = oracle.keygen_hash128(1000 + rank, n_per_rank[rank])
        f = sharded.build_sharded(torch.from_numpy(local.view(np.int64)), 2000, 16)
        out.put((rank, None if f is None else f.serialize()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_build_sharded_two_ranks(rsb, oracle_mod, engine):
    world, n_per_rank = 2, (40_000, 25_000)
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out, n_per_rank)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=600) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert results[1] is None
    keys = np.concatenate([oracle_mod.keygen_hash128(1000 + r, n_per_rank[r]) for r in range(world)])
    assert results[0] == rsb.GPURecSplit(keys, bucket_size=2000, leaf_size=16, engine=engine).serialize()
