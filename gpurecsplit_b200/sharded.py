"""One function over keys spread across several GPUs: bucket-range sharding.

Every rank holds some of the keys (as 128-bit hashes). The function's buckets
(remap128(first, nbuckets), support/common.hpp:273-280) are split into contiguous ranges,
rank r owning buckets [nb*r/G, nb*(r+1)/G), as the reference's threads split them
(SIMDRecSplit.hpp:695-745). One all-to-all moves every key to the rank that owns its bucket;
each rank builds its range on its own GPU (rsb_build_part_hash128); the exported parts are
gathered and the root merges them (rsb_merge_parts) into the function a single GPU builds
from all keys, byte for byte.

The data path uses torch.distributed: NCCL with CUDA tensors (over NVLink / NVSwitch) or
gloo with CPU tensors. The part builder and merger can be replaced (``builder``, ``merger``)
so that the exchange logic can run where no GPU is present.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np

_MASK32 = 0xFFFFFFFF


def num_buckets(n_total: int, bucket_size: int) -> int:
    """nbuckets = max(1, ceil(n / b)) (AbstractParallelRecSplit.hpp:322, SIMDRecSplit.hpp:774)."""
    return max(1, -(-n_total // bucket_size))


def bucket_ranges(nb: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous bucket range of every rank: [nb*r/G, nb*(r+1)/G)."""
    return [(nb * r // world, nb * (r + 1) // world) for r in range(world)]


def bucket_ids(keys128, nb: int):
    """remap128(first, nb) = (first * nb) >> 64 for a (n, 2) int64 torch tensor of hash128
    keys (first in column 0, as the bits of a uint64), on the tensor's device."""
    import torch
    if not 1 <= nb < (1 << 30):
        raise ValueError("bucket count out of range")
    first = keys128[:, 0]
    hi = (first >> 32) & _MASK32          # arithmetic shift, then the low 32 bits: the high word
    lo = first & _MASK32
    nbt = torch.tensor(nb, dtype=torch.int64, device=keys128.device)
    # (hi * 2^32 + lo) * nb >> 64 = (hi * nb + (lo * nb >> 32)) >> 32, every term below 2^63
    return (hi * nbt + ((lo * nbt) >> 32)) >> 32


def owners(ids, nb: int, world: int):
    """The rank that owns each bucket id."""
    import torch
    starts = torch.tensor([lo for lo, _ in bucket_ranges(nb, world)], dtype=torch.int64, device=ids.device)
    return torch.searchsorted(starts, ids, right=True) - 1


def exchange(keys128, nb: int, group=None):
    """Moves every key to the rank that owns its bucket (one all-to-all). Returns the keys of
    this rank's bucket range, (m, 2) int64 on the same device."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    dest = owners(bucket_ids(keys128, nb), nb, world)
    order = torch.argsort(dest, stable=True)
    send = keys128[order].contiguous()
    send_counts = torch.bincount(dest, minlength=world).to(torch.int64)
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts, group=group)
    sc, rc = send_counts.tolist(), recv_counts.tolist()
    recv = torch.empty((sum(rc), 2), dtype=torch.int64, device=keys128.device)
    dist.all_to_all_single(recv.view(-1), send.view(-1), [2 * c for c in rc], [2 * c for c in sc], group=group)
    return recv


def _gather_bytes(blob: bytes, device, group=None) -> List[bytes]:
    """Every rank's byte string, on every rank (all_gather of padded uint8 tensors)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    n = torch.tensor([len(blob)], dtype=torch.int64, device=device)
    sizes = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(sizes, n, group=group)
    sizes = [int(s.item()) for s in sizes]
    cap = max(sizes)
    mine = torch.zeros(cap, dtype=torch.uint8, device=device)
    if blob:
        mine[:len(blob)] = torch.frombuffer(bytearray(blob), dtype=torch.uint8).to(device)
    bufs = [torch.empty(cap, dtype=torch.uint8, device=device) for _ in range(world)]
    dist.all_gather(bufs, mine, group=group)
    return [b[:s].cpu().numpy().tobytes() for b, s in zip(bufs, sizes)]


def build_sharded(keys128, bucket_size: int, leaf_size: int, rotate: bool = True, group=None, root: int = 0,
                  engine=None, builder: Optional[Callable] = None, merger: Optional[Callable] = None):
    """Builds one function from the keys of all ranks (collective: every rank calls it).

    ``keys128``: this rank's keys as a (n, 2) int64 torch tensor (hash128 bits; CUDA tensors
    with NCCL, CPU tensors with gloo). Returns the merged function on ``root`` and None on the
    other ranks. ``builder(keys, nb, lo, hi) -> bytes`` and ``merger(parts) -> function``
    default to rsb_build_part_hash128 / rsb_part_export and rsb_merge_parts.
    """
    import torch
    import torch.distributed as dist
    if builder is None or merger is None:
        import gpurecsplit_b200 as rsb
    if builder is None:
        def builder(keys, nb, lo, hi):
            if keys.is_cuda:
                return rsb.build_part(keys.data_ptr(), nb, lo, hi, bucket_size, leaf_size, rotate, engine,
                                      n=keys.shape[0])
            return rsb.build_part(keys.numpy().view(np.uint64), nb, lo, hi, bucket_size, leaf_size, rotate, engine)
    if merger is None:
        def merger(parts):
            return rsb.merge_parts(parts, leaf_size, rotate, engine)
    world, rank = dist.get_world_size(group), dist.get_rank(group)
    n = torch.tensor([keys128.shape[0]], dtype=torch.int64, device=keys128.device)
    dist.all_reduce(n, group=group)
    nb = num_buckets(int(n.item()), bucket_size)
    mine = exchange(keys128, nb, group)
    lo, hi = bucket_ranges(nb, world)[rank]
    if keys128.is_cuda:
        torch.cuda.current_stream().synchronize()  # the exchanged keys are complete before the part build reads them
    part = builder(mine, nb, lo, hi) if hi > lo else b""
    parts = _gather_bytes(part, keys128.device, group)
    if rank != root:
        return None
    return merger([p for p in parts if p])
