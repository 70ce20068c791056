"""Replicas on several GPUs (bench.py --gpus N under torchrun): each rank builds its own key
set with no data-path collective, and the step time is the maximum over ranks. The host
logic of that path runs here as two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        local_ms = 100.0 + 25.0 * rank  # rank 1 is the slow one
        total = bench.max_over_ranks(local_ms, dist, "cpu")
        keys = bench.rank_keys(rank, 1000)
        out.put((rank, total, bench.ns_per_key(total, 4, 1000, world), keys.tobytes()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_take_the_slowest_rank():
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    results = [out.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = {r: (t, v, k) for r, t, v, k in results}
    for r in range(world):
        total, value, _ = by_rank[r]
        assert total == 125.0                      # every rank sees the maximum
        assert value == pytest.approx(125.0 / 4 * 1e6 / (1000 * world))
    k0 = np.frombuffer(by_rank[0][2], dtype=np.uint64)
    k1 = np.frombuffer(by_rank[1][2], dtype=np.uint64)
    assert np.intersect1d(k0, k1).size == 0         # independent key sets per replica


def test_single_process_needs_no_group():
    import bench
    assert bench.max_over_ranks(3.5) == 3.5
    assert bench.ns_per_key(2000.0, 2, 5_000_000, 1) == pytest.approx(200.0)
