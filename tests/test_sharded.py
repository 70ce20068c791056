"""Bucket-range sharding over several ranks (gpurecsplit_b200/sharded.py), host logic on the
CPU: bucket ids equal remap128 (support/common.hpp:273-280), the ranges tile the buckets, and
with gloo ranks the all-to-all hands every rank exactly the keys of its bucket range and the
root receives every rank's part. Part builds and the merge themselves run on the GPU
(tests/test_gpu_sharded.py); here a stand-in builder reports what each rank received."""
import os
import pickle
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from gpurecsplit_b200 import sharded


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _keys(seed: int, n: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.integers(0, 2**64, (n, 2), dtype=np.uint64, endpoint=False)


def _remap128(first: np.ndarray, nb: int) -> np.ndarray:
    return np.array([(int(f) * nb) >> 64 for f in first], dtype=np.int64)


def test_bucket_ids_equal_remap128():
    k = _keys(1, 5000)
    k[:4, 0] = [0, 2**64 - 1, 2**63, 2**63 - 1]
    for nb in (1, 2, 7, 2500, 12345, (1 << 30) - 1):
        got = sharded.bucket_ids(torch.from_numpy(k.view(np.int64)), nb).numpy()
        assert np.array_equal(got, _remap128(k[:, 0], nb)), nb


def test_ranges_tile_the_buckets():
    for nb in (1, 3, 10, 2500):
        for world in (1, 2, 3, 8):
            r = sharded.bucket_ranges(nb, world)
            assert r[0][0] == 0 and r[-1][1] == nb
            assert all(r[i][1] == r[i + 1][0] for i in range(world - 1))
            ids = torch.arange(nb)
            own = sharded.owners(ids, nb, world).numpy()
            for rank, (lo, hi) in enumerate(r):
                assert np.all(own[lo:hi] == rank)


def _rank_main(rank, world, port, out, n_per_rank, bucket_size):
    import datetime

    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local = torch.from_numpy(_keys(100 + rank, n_per_rank[rank]).view(np.int64))

        def builder(keys, nb, lo, hi):
            return pickle.dumps((rank, nb, lo, hi, keys.numpy().tobytes()))

        res = sharded.build_sharded(local, bucket_size, 8, builder=builder, merger=lambda parts: parts)
        out.put((rank, res))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,n_per_rank,bucket_size", [(2, (3000, 1700), 100), (3, (500, 0, 900), 2000),
                                                          (2, (0, 0), 100)])
def test_exchange_hands_each_rank_its_bucket_range(world, n_per_rank, bucket_size):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out, n_per_rank, bucket_size))
             for r in range(world)]
    for p in procs:
        p.start()
    results = dict(out.get(timeout=180) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(results[r] is None for r in range(1, world))
    parts = [pickle.loads(p) for p in results[0]]
    all_keys = np.concatenate([_keys(100 + r, n_per_rank[r]) for r in range(world)])
    nb = sharded.num_buckets(all_keys.shape[0], bucket_size)
    ids = _remap128(all_keys[:, 0], nb)
    ranges = sharded.bucket_ranges(nb, world)
    expect_ranks = [r for r, (lo, hi) in enumerate(ranges) if hi > lo]
    assert [p[0] for p in parts] == expect_ranks
    for rank, pnb, lo, hi, blob in parts:
        assert pnb == nb and (lo, hi) == ranges[rank]
        got = np.frombuffer(blob, dtype=np.uint64).reshape(-1, 2)
        want = all_keys[(ids >= lo) & (ids < hi)]
        assert sorted(map(tuple, got.tolist())) == sorted(map(tuple, want.tolist()))
