#!/usr/bin/env python
"""Benchmark of RecSplit construction on B200: build ns/key at l=16, b=2000, n=5M.

One step = one complete construction (hash to 128 bits, bucket partition, every seed
search, Golomb-Rice + double Elias-Fano encoding) of n=5,000,000 uniform random 64-bit
keys (splitmix64, seed 42 + rank) with leaf size 16, bucket size 2000 and rotation fitting.

  value   device time of a build from keys resident in HBM (CUDA events on the engine
          stream, L2 flushed by a 256 MiB write before every timed step), ns per key
  e2e     the same build through the public API from pinned host keys: host->device copy
          of the keys, construction, device->host copy of the built function and its
          serialization, all inside the timed region
  roofline  the dominant search kernel's algorithmic evaluation rate (sum over its nodes
          of candidates x node size / its device time) against the device's measured
          remixAndRemap32 evaluation ceiling (rsb_probe_eval_rate)
  cpu_baseline  the reference's own SIMDRecSplit (compiled from its sources into
          oracle/_ref) on all host cores, on one contiguous fifth of the workload's buckets
  c1, c3, c4_batch, c5_serve  the other configurations (1M string keys l=8 b=100; 200k keys
          l=24 b=2000; 1000 batched sets l=12 b=1000; the serving loop), each with its own
          clock record, timing and parity check (single GPU only)

`--impl reference` times only the CPU build (the reference's SIMDRecSplit from oracle/_ref;
without it, this project's AVX-512 restatement): step i builds the i-th of `steps`
contiguous bucket ranges, so the timed steps together build the whole workload once.

Other modes (one JSON line each): `--mode batch` (many key sets in one pipeline vs
back-to-back plain builds), `--mode serve` (continuous batching of string requests),
`--mode c1`, `--mode c3`, `--mode pipeline` (stage kernels against pipeline mode) and
`--mode build` (plain builds of a chosen size, for profiling).

Multi-GPU (torchrun): every rank builds its own 5M-key set (weak scaling, no data-path
collective); the step time is the max over ranks.
"""
from __future__ import annotations

import argparse
import csv
import datetime
import hashlib
import io
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "build ns/key (l=16,b=2000,n=5M)"
UNIT = "ns/key"
N_KEYS = 5_000_000
LEAF = 16
BUCKET = 2000
SEED = 42
PUBLISHED_NS_PER_KEY = 1000.0  # GpuRecSplit, l=16 b=2000 n=5M: 1.0 us/object (README.md:18)
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_builds.json")
PROFILE_TRAFFIC = os.path.join(ROOT, "profiles", "traffic_k_search_aggr_u64_n5M_l16_b2000.json")


def splitmix64_keys(seed: int, n: int) -> np.ndarray:
    """n outputs of splitmix64 (Steele, Lea, Flood 2014) started at `seed`."""
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def rank_keys(rank: int, n: int) -> np.ndarray:
    """The keys rank `rank` builds: replicas get independent sets (splitmix64 seed 42 + rank)."""
    return splitmix64_keys(SEED + rank, n)


def max_over_ranks(x: float, dist=None, device: str = "cpu") -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def ns_per_key(total_ms: float, steps: int, n: int, world: int) -> float:
    """Whole-job ns/key: the slowest rank's time per step over the keys of all ranks."""
    return total_ms / steps * 1e6 / (n * world)


def workload_config(n: int, world: int) -> dict:
    return {
        "workload": f"u64 keys n={n} (splitmix64 seed 42+rank) hashed to 128 bits (fmix64 / stafford13), "
                    f"RecSplit l={LEAF} b={BUCKET} with rotation fitting",
        "n": n, "leaf": LEAF, "bucket": BUCKET, "nbuckets": (n + BUCKET - 1) // BUCKET,
        "l2": "flushed before every timed step (256 MiB device write)",
        "parallelism": f"replicas x{world} (independent key sets per GPU)" if world > 1 else "single GPU",
    }


# ---------------------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=10)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self) -> dict:
        rows = [r for r in csv.reader(io.StringIO(getattr(self, "out", ""))) if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].strip().lower() == "active":
                    reasons.add(name)
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


# ---------------------------------------------------------------------------------------
# CPU side — the reference's own SIMDRecSplit (oracle/_ref) on bucket ranges of the workload
# ---------------------------------------------------------------------------------------
class CpuWorkload:
    """The bench workload (n keys, l=16, b=2000) hashed to 128 bits and grouped by bucket,
    for timing CPU builds on contiguous bucket ranges.

    A range [lo, hi) of the workload's buckets is built as its own function: the keys keep
    their second halves (which alone decide every seed) and their bucket sizes, and their first
    halves are replaced by the smallest value that remap128 (support/common.hpp:273-280) maps
    to the same bucket of an (hi - lo)-bucket function, whose bucket size is chosen so that it
    has exactly hi - lo buckets. So a range build runs the reference's complete construction
    (sort, partition, every seed search, Rice and Elias-Fano encoding) over exactly the seed
    searches of those buckets in the full build, and ranges that cover the workload cover its
    search work once.
    """

    def __init__(self, n: int = N_KEYS, seed: int = SEED):
        import oracle
        keys = oracle.hash_u64(splitmix64_keys(seed, n))
        self.n = n
        self.nb = (n + BUCKET - 1) // BUCKET
        first = keys[:, 0]
        nb = np.uint64(self.nb)
        hi = first >> np.uint64(32)
        lo = first & np.uint64(0xFFFFFFFF)
        bucket = (hi * nb + ((lo * nb) >> np.uint64(32))) >> np.uint64(32)  # (first * nb) >> 64
        order = np.argsort(bucket, kind="stable")
        self.second = np.ascontiguousarray(keys[order, 1])
        self.start = np.searchsorted(bucket[order], np.arange(self.nb + 1, dtype=np.uint64)).astype(np.int64)

    def range_keys(self, lo: int, hi: int):
        """(keys128, bucket size) of the function over buckets [lo, hi)."""
        nb = hi - lo
        a, z = int(self.start[lo]), int(self.start[hi])
        n = z - a
        b = max(1, -(-n // nb))
        while -(-n // b) > nb:
            b += 1
        while b > 1 and -(-n // (b - 1)) == nb:
            b -= 1
        if max(1, -(-n // b)) != nb:
            raise RuntimeError(f"no bucket size gives {nb} buckets for {n} keys")
        out = np.empty((n, 2), dtype=np.uint64)
        out[:, 1] = self.second[a:z]
        sizes = np.diff(self.start[lo:hi + 1])
        firsts = np.array([-(-(j << 64) // nb) for j in range(nb)], dtype=np.uint64)
        out[:, 0] = np.repeat(firsts, sizes)
        return out, b

    def ranges(self, parts: int):
        """`parts` contiguous bucket ranges covering every bucket once."""
        return [(self.nb * i // parts, self.nb * (i + 1) // parts) for i in range(parts)]


def cpu_impl():
    """(build function, kind, description) of the CPU build that is timed."""
    import oracle
    oracle.build()
    if oracle.ref_available():
        return (lambda k, b, t: oracle.ref_build(k, LEAF, b, True, threads=t), "reference",
                "the reference's own SIMDRecSplit (include/function/SIMDRecSplit.hpp) compiled from its sources "
                "with AVX-512 (oracle/_ref)")
    if oracle.simd_supported():
        return (lambda k, b, t: oracle.build_mphf(k, LEAF, b, True, threads=t, simd=True).bytes, "port",
                "SIMDRecSplit restated with AVX-512 search loops (oracle/_build/libsimdrs.so)")
    return (lambda k, b, t: oracle.build_mphf(k, LEAF, b, True, threads=t).bytes, "port", "scalar oracle")


def time_cpu_ranges(work: CpuWorkload, ranges, threads: int, build):
    """Seconds and keys of one CPU build per bucket range."""
    out = []
    for lo, hi in ranges:
        keys, b = work.range_keys(lo, hi)
        t0 = time.perf_counter()
        blob = build(keys, b, threads)
        dt = time.perf_counter() - t0
        assert blob.size > 0
        out.append((dt, keys.shape[0]))
    return out


def cpu_baseline(args) -> dict:
    """The CPU build timed on a bounded sample: one contiguous fifth of the workload's buckets
    (about 1M keys, 10-30 s on the box's host cores), on all host cores."""
    import oracle
    build, kind, what = cpu_impl()
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    work = CpuWorkload(args.n)
    parts = max(1, args.cpu_fraction)
    lo, hi = work.ranges(parts)[parts // 2]
    (secs, keys), = time_cpu_ranges(work, [(lo, hi)], threads, build)
    return {"value": secs * 1e9 / keys, "unit": UNIT, "cores": threads, "kind": kind,
            "sample": f"buckets [{lo}, {hi}) of the {work.nb}-bucket workload ({keys} keys, built as one function "
                      f"with the same buckets and seed searches); {what}, {threads} threads on {oracle.cpu_model()}",
            "seconds": secs}


def run_reference(args, rank: int, world: int) -> None:
    """The reference arm: the reference's own SIMDRecSplit on all host cores. Step i builds
    buckets [i*nb/steps, (i+1)*nb/steps) of the workload, so the timed steps together build
    the whole n=5M workload exactly once; warm-up steps build a 4-bucket range each."""
    if rank != 0:
        return
    import oracle
    build, kind, what = cpu_impl()
    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    work = CpuWorkload(args.n)
    for w in range(args.warmup):
        lo = (w * 37) % (work.nb - 4)
        time_cpu_ranges(work, [(lo, lo + 4)], threads, build)
    res = time_cpu_ranges(work, work.ranges(args.steps), threads, build)
    secs = sum(r[0] for r in res)
    keys = sum(r[1] for r in res)
    v = secs * 1e9 / keys
    sample = (f"{args.steps} steps of {work.nb // args.steps}-{-(-work.nb // args.steps)} contiguous buckets each, "
              f"together all {work.nb} buckets ({keys} keys) of the workload once; {what}, {threads} threads on "
              f"{oracle.cpu_model()}")
    line = {
        "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": secs / args.steps * 1e3, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": v / PUBLISHED_NS_PER_KEY, "dtype": "u64", "data": "synthetic",
        "impl": "reference",
        "config": workload_config(args.n, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "CPU build on the host cores; the per-range bucket size keeps every range's buckets, and so its "
                "seed searches, those of the full build (the first key halves are re-mapped to the range)",
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------------------
def run_gpu(args, rank: int, world: int, local_rank: int) -> None:
    import torch
    import gpurecsplit_b200 as rsb

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))
    stream = torch.cuda.current_stream()
    engine = rsb.Engine(local_rank, stream.cuda_stream)
    n = args.n
    keys_host = rank_keys(rank, n)
    pinned = torch.from_numpy(keys_host.view(np.int64)).pin_memory()
    keys_dev = pinned.to(f"cuda:{local_rank}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local_rank}")
    torch.cuda.synchronize()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def device_build():
        return rsb.GPURecSplit.from_device(keys_dev.data_ptr(), n, BUCKET, LEAF, key_type="u64", engine=engine,
                                           device_only=True)

    # warm-up (also loads the kernels and sizes the engine's scratch)
    for _ in range(args.warmup):
        flush.zero_()
        device_build().close()
    torch.cuda.synchronize()

    # ---- timed: device-resident builds ----
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    stats = []
    last = None
    with ClockSampler(local_rank) as clocks:
        barrier()
        for i in range(args.steps):
            flush.zero_()
            starts[i].record(stream)
            f = device_build()
            ends[i].record(stream)
            stats.append(f.stats())
            if last is not None:
                last.close()
            last = f
        barrier()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    total_ms = max_over_ranks(sum(step_ms), dist, f"cuda:{local_rank}")
    ms_per_step = total_ms / args.steps
    value = ns_per_key(total_ms, args.steps, n, world)

    # parity of the last timed build with the committed oracle digest
    parity = None
    if rank == 0 and os.path.exists(GOLDEN) and n == N_KEYS:
        g = json.load(open(GOLDEN)).get("u64_n5M_l16_b2000")
        if g is not None:
            blob = last.serialize()
            parity = {"sha256_equals_reference": hashlib.sha256(blob).hexdigest() == g["ref_sha256"],
                      "golden": "u64_n5M_l16_b2000 (the reference's SIMDRecSplit build of the same keys)",
                      "bits_per_key": last.get_bits() / n}
    bits_per_key = last.get_bits() / n
    last.close()

    # ---- timed: end to end through the public API from pinned host keys ----
    e2e_steps = max(1, min(args.steps, 3))
    e2e_ms = []
    d2h_bytes = 0
    host_keys = pinned.numpy().view(np.uint64)
    for i in range(e2e_steps + 1):
        flush.zero_()
        barrier()
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record(stream)
        f = rsb.GPURecSplit(host_keys, bucket_size=BUCKET, leaf_size=LEAF, key_type="u64", engine=engine)
        blob = f.serialize()
        e.record(stream)
        e.synchronize()
        if i > 0:  # the first one is a warm-up of the host paths
            e2e_ms.append(s.elapsed_time(e))
        # structure words copied back (the 14 serialization header words are not copied) plus
        # the status word, encoder parameters and stage counts read at the end of the build
        d2h_bytes = len(blob) - 8 * 14 + 16 + 8 * 36 + 4 * 21
        f.close()
    e2e_total = max_over_ranks(sum(e2e_ms), dist, f"cuda:{local_rank}")
    e2e_value = ns_per_key(e2e_total, e2e_steps, n, world)

    if rank == 0:
        # ---- roofline of the dominant search kernel ----
        st = stats[-1]
        ms_search = st["ms_search"]
        dom = max(range(21), key=lambda s: ms_search[s])
        names = {17: "upper aggregation (k_search_aggr<16,17>)", 18: "lower aggregation (k_search_aggr<16,18>)",
                 19: "rotation leaves (k_search_leaf<16,true>)", 20: "brute-force leaves (k_search_leaf<16,false>)"}
        dom_name = names.get(dom, f"fanout-2 depth {dom} (k_search_higher)")
        achieved = st["evals_stage"][dom] / (ms_search[dom] * 1e-3) / 1e9
        peak_rates = [engine.probe_eval_rate()[0] for _ in range(3)]
        peak = max(peak_rates) / 1e9
        traffic = None
        if os.path.exists(PROFILE_TRAFFIC):
            traffic = json.load(open(PROFILE_TRAFFIC)).get(str(dom))
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline(args)
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_NS_PER_KEY, "dtype": "u64", "data": "synthetic",
            "config": workload_config(n, world),
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": d2h_bytes},
            "roofline": {"bound": "int", "kernel": dom_name, "achieved": achieved, "peak": peak, "unit": "Geval/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "peak_source": "rsb_probe_eval_rate: measured remixAndRemap32 evaluation ceiling on this GPU",
                         "evals": st["evals_stage"][dom], "ms": ms_search[dom]},
            "cpu_baseline": cpu,
            "clocks": clocks.summary(),
            "gpu_launches": sum(s["kernel_launches"] for s in stats),
            "bits_per_key": bits_per_key,
            "parity": parity,
            "stage_ms": {"partition": st["ms_partition"], "search": {str(i): round(v, 3) for i, v in
                                                                     enumerate(ms_search) if v > 0},
                         "encode": st["ms_encode"], "total": st["ms_total"]},
            "stage_geval_s": {str(i): round(st["evals_stage"][i] / (v * 1e-3) / 1e9, 1)
                              for i, v in enumerate(ms_search) if v > 0.05},
            "step_ms": [round(x, 3) for x in step_ms],
            "schedule": schedule_of(engine, LEAF, n),
            "windows_per_stage": {str(i): [st["windows_stage"][i], st["window_candidates"][i]]
                                  for i in (17, 18, 19) if st["windows_stage"][i]},
        }
        if world == 1 and not args.no_extras:
            # The other configurations, each with its own clock record, parity and timing
            # (one GPU; at N > 1 the line carries the headline only).
            del keys_dev, flush
            torch.cuda.empty_cache()
            # 1.2 ms per C1 build: 1000 timed steps keep the clock sampler (200 ms period) busy
            line["c1"] = measure_config("c1", engine, steps=1000, warmup=3, e2e_steps=20)
            line["c3"] = measure_config("c3", engine, steps=1, warmup=1, e2e_steps=1)
            line["c4_batch"] = measure_batch(args.sets, engine)
            line["c5_serve"] = measure_serve(args.requests, args.max_keys, args.hbm_budget, args.inflight, args.load)
        print(json.dumps(line), flush=True)
    engine.close()
    if dist is not None:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------
# Batched form: many independent key sets in one pipeline vs back-to-back plain builds
# ---------------------------------------------------------------------------------------
def batch_workload(nsets: int, seed0: int = 1000):
    """Set i: round(exp(U[ln 1e3, ln 1e6])) u64 keys from splitmix64 seeded seed0 + i."""
    rng = np.random.default_rng(7)
    sizes = np.rint(np.exp(rng.uniform(np.log(1e3), np.log(1e6), nsets))).astype(np.int64)
    offsets = np.zeros(nsets + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(sizes)
    keys = np.empty(int(offsets[-1]), dtype=np.uint64)
    for i in range(nsets):
        keys[offsets[i]:offsets[i + 1]] = splitmix64_keys(seed0 + i, int(sizes[i]))
    return keys, offsets


# ---------------------------------------------------------------------------------------
# Other plain configurations: C1 (string keys, l=8, b=100) and C3 (l=24)
# ---------------------------------------------------------------------------------------
def printable_strings(seed: int, n: int, min_len: int = 10, max_len: int = 50):
    """n printable strings from one splitmix64 stream started at `seed`: per key one output
    for the length (min_len + v % (max_len - min_len + 1)), then one output per byte
    (0x21 + v % 94)."""
    stream = splitmix64_keys(seed, n * (max_len + 1))
    span = np.uint64(max_len - min_len + 1)
    len_pos = np.empty(n, dtype=np.int64)
    lens = np.empty(n, dtype=np.int64)
    pos = 0
    for i in range(n):  # each length decides where the next one is drawn
        ln = min_len + int(stream[pos] % span)
        len_pos[i] = pos
        lens[i] = ln
        pos += 1 + ln
    is_byte = np.ones(pos, dtype=bool)
    is_byte[len_pos] = False
    data = (np.uint64(0x21) + stream[:pos][is_byte] % np.uint64(94)).astype(np.uint8)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    return data, offsets


CONFIGS = {
    # name: (key kind, seed, n, leaf, bucket, golden digest entry)
    "c1": ("strings", 42, 1_000_000, 8, 100, "strings_n1M_l8_b100"),
    "c3": ("u64", 43, 200_000, 24, 2000, "u64_n200k_l24_b2000"),
}


HAND_SET = {17: lambda leaf: 12 if leaf >= 12 else 8, 18: lambda leaf: 12 if leaf >= 12 else 8, 19: lambda leaf: 8}


def schedule_of(engine, leaf: int, keys: int) -> dict:
    """The engine's stage schedules for a build of `keys` keys: {stage: [per lane, occupancy %]}."""
    cls = 1 if keys >= (1 << 20) else 0
    return {str(st): list(engine.schedule(leaf, st, cls)) for st in (17, 18, 19)}


def set_hand_schedule(engine, leaf: int, keys: int, on: bool) -> None:
    """Overrides the tuned schedules with the fixed ones used before tuning (12 candidates per
    lane for aggregation at l >= 12, 8 otherwise, 8 bases for rotation leaves, full
    occupancy), or restores the tuned ones."""
    cls = 1 if keys >= (1 << 20) else 0
    for st, f in HAND_SET.items():
        engine.set_schedule(leaf, st, cls, f(leaf) if on else 0, 100)


def measure_config(name: str, engine=None, steps: int = 5, warmup: int = 3, e2e_steps: int = 2) -> dict:
    """Device build time of one plain configuration (keys resident in HBM, L2 flushed before
    every timed step), end-to-end time from host keys, and parity with the committed digest of
    the reference's build. Warm-up builds are of the same configuration; for l=24 (seconds per
    build) a single one-bucket build of the same leaf size loads the kernels instead."""
    import ctypes

    import torch
    import gpurecsplit_b200 as rsb

    kind, seed, n, leaf, b, golden = CONFIGS[name]
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    own = engine is None
    if own:
        engine = rsb.Engine(0, stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    L = rsb.lib()
    if kind == "strings":
        data, offsets = printable_strings(seed, n)
        d_data = torch.from_numpy(data).to("cuda")
        d_off = torch.from_numpy(offsets.view(np.int64)).to("cuda")
        # the end-to-end builds read the keys from pinned host memory
        host_keys = (torch.from_numpy(data).pin_memory().numpy(),
                     torch.from_numpy(offsets.view(np.int64)).pin_memory().numpy().view(np.uint64))
        flags = rsb.RSB_ROTATE | rsb.RSB_KEYS_ON_DEVICE | rsb.RSB_DEVICE_ONLY

        def device_build(count=n):
            h = ctypes.c_void_p()
            rsb._check(L.rsb_build_strings(engine.handle, ctypes.c_void_p(d_data.data_ptr()),
                                           ctypes.c_void_p(d_off.data_ptr()), count, b, leaf, flags,
                                           ctypes.byref(h)), "rsb_build_strings")
            return rsb.GPURecSplit(bucket_size=b, leaf_size=leaf, _handle=h)
        h2d = data.nbytes + offsets.nbytes
    else:
        keys = splitmix64_keys(seed, n)
        d_keys = torch.from_numpy(keys.view(np.int64)).to("cuda")
        host_keys = torch.from_numpy(keys.view(np.int64)).pin_memory().numpy().view(np.uint64)

        def device_build(count=n):
            return rsb.GPURecSplit.from_device(d_keys.data_ptr(), count, b, leaf, key_type="u64", engine=engine,
                                               device_only=True)
        h2d = keys.nbytes
    torch.cuda.synchronize()
    small_warmup = leaf >= 20
    for _ in range(warmup):
        flush.zero_()
        device_build(min(n, b) if small_warmup else n).close()
    times, stats = [], None
    blob = None
    with ClockSampler(0) as clocks:
        for _ in range(steps):
            flush.zero_()
            s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s0.record(stream)
            f = device_build()
            e0.record(stream)
            e0.synchronize()
            times.append(s0.elapsed_time(e0))
            stats = f.stats()
            blob = f.serialize()
            f.close()
        e2e = []
        for i in range(e2e_steps + (1 if e2e_steps > 1 else 0)):  # the first of several is untimed
            flush.zero_()
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            f = rsb.GPURecSplit(host_keys, bucket_size=b, leaf_size=leaf, key_type=kind, engine=engine)
            blob2 = f.serialize()
            if e2e_steps == 1 or i > 0:
                e2e.append(time.perf_counter() - t0)
            bits = f.get_bits()
            f.close()
    # the same timed steps with the fixed schedule used before tuning (same function)
    set_hand_schedule(engine, leaf, n, True)
    hand = []
    for _ in range(steps):
        flush.zero_()
        s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        f = device_build()
        e0.record(stream)
        e0.synchronize()
        hand.append(s0.elapsed_time(e0))
        same_hand = f.serialize() == blob
        f.close()
    set_hand_schedule(engine, leaf, n, False)
    parity = None
    if os.path.exists(GOLDEN):
        g = json.load(open(GOLDEN)).get(golden)
        if g is not None:
            parity = {"sha256_equals_reference": hashlib.sha256(blob).hexdigest() == g.get("ref_sha256")
                      and hashlib.sha256(blob2).hexdigest() == g.get("ref_sha256"), "golden": golden}
    ms = statistics.median(times)
    ms_search = stats["ms_search"]
    out = {
        "metric": f"build ns/key ({name}: {kind} keys, l={leaf}, b={b}, n={n})", "value": ms * 1e6 / n,
        "unit": "ns/key", "higher_is_better": False, "n_gpus": 1, "steps": steps,
        "warmup": warmup, "warmup_kind": f"one-bucket builds (l={leaf})" if small_warmup else "same configuration",
        "ms_per_step": ms, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"{kind} keys n={n} (splitmix64 seed {seed}"
                               + (", printable 10-50 B strings" if kind == "strings" else "")
                               + f"), l={leaf}, b={b}, rotation", "l2": "flushed before every timed step"},
        "e2e": {"value": statistics.median(e2e) * 1e9 / n, "unit": "ns/key", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": len(blob2), "steps": e2e_steps,
                "timing": "median host wall clock around the public-API build and serialization, keys in "
                          "pinned host memory" + (", after one untimed call" if e2e_steps > 1 else "")},
        "bits_per_key": bits / n, "parity": parity,
        "stage_ms": {"partition": stats["ms_partition"],
                     "search": {str(i): round(v, 3) for i, v in enumerate(ms_search) if v > 0},
                     "encode": stats["ms_encode"], "total": stats["ms_total"]},
        "stage_geval_s": {str(i): round(stats["evals_stage"][i] / (v * 1e-3) / 1e9, 1)
                          for i, v in enumerate(ms_search) if v > 0.05},
        "gpu_launches": stats["kernel_launches"] * steps, "clocks": clocks.summary(),
        "step_ms": [round(x, 3) for x in times],
        "schedule": schedule_of(engine, leaf, n),
        "untuned": {"ms_per_step": statistics.median(hand), "schedule": {str(s): [f(leaf), 100] for s, f in
                                                                       HAND_SET.items()},
                    "tuning_gain": statistics.median(hand) / ms, "identical": same_hand},
    }
    if own:
        engine.close()
    return out


def measure_batch(nsets: int, engine=None) -> dict:
    """Batched form: all sets in one pipeline vs back-to-back plain builds of the same sets on
    the same engine; every set's function must equal its plain build."""
    import torch
    import gpurecsplit_b200 as rsb

    leaf, b = 12, 1000
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream()
    own = engine is None
    if own:
        engine = rsb.Engine(0, stream.cuda_stream)
    keys, offsets = batch_workload(nsets)
    n = int(offsets[-1])
    keys_dev = torch.from_numpy(keys.view(np.int64)).to("cuda")
    torch.cuda.synchronize()
    base = keys_dev.data_ptr()

    def batched():
        funcs, st = rsb.build_batch(base, offsets, b, leaf, key_type="u64", engine=engine, keys_on_device=True)
        return funcs, st

    def plain_all():
        out = []
        for i in range(nsets):
            lo, hi = int(offsets[i]), int(offsets[i + 1])
            out.append(rsb.GPURecSplit.from_device(base + 8 * lo, hi - lo, b, leaf, key_type="u64", engine=engine,
                                                   device_only=False))
        return out

    def timed(fn):
        torch.cuda.synchronize()
        s0, e0 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s0.record(stream)
        r = fn()
        e0.record(stream)
        e0.synchronize()
        return r, s0.elapsed_time(e0)

    for f in batched()[0]:  # warm-up (sizes the engine's scratch)
        f.close()
    for f in plain_all():
        f.close()
    with ClockSampler(0) as clocks:
        (funcs, st), t_batch = timed(batched)
        plain, t_plain = timed(plain_all)
        set_hand_schedule(engine, leaf, n, True)
        (hand_funcs, _), t_hand = timed(batched)
        set_hand_schedule(engine, leaf, n, False)
    same = all(f.serialize() == p.serialize() for f, p in zip(funcs, plain))
    same_hand = all(f.serialize() == h.serialize() for f, h in zip(funcs, hand_funcs))
    for f in funcs + plain + hand_funcs:
        f.close()
    del keys_dev
    out = {
        "metric": "batched keys/s (log-uniform sets in [1e3,1e6], l=12, b=1000)", "value": n / (t_batch * 1e-3),
        "unit": "keys/s", "higher_is_better": True, "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": t_batch, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"{nsets} key sets, sizes round(exp(U[ln 1e3, ln 1e6])) (numpy seed 7), "
                               f"set i = splitmix64(seed 1000+i) u64 keys, l={leaf}, b={b}, rotation",
                   "sets": nsets, "keys": n, "l2": f"inputs ({8 * n / 1e9:.1f} GB) larger than L2"},
        "plain_back_to_back": {"keys_per_s": n / (t_plain * 1e-3), "ms": t_plain},
        "speedup_vs_plain": t_plain / t_batch,
        "identical_to_plain": same,
        "stage_ms": {"partition": st["ms_partition"], "search": {str(i): round(v, 3) for i, v in
                                                                 enumerate(st["ms_search"]) if v > 0},
                     "encode": st["ms_encode"], "total": st["ms_total"]},
        "stage_geval_s": {str(i): round(st["evals_stage"][i] / (v * 1e-3) / 1e9, 1)
                          for i, v in enumerate(st["ms_search"]) if v > 0.05},
        "gpu_launches": st["kernel_launches"], "clocks": clocks.summary(),
        "schedule": schedule_of(engine, leaf, n),
        "untuned": {"ms_per_step": t_hand, "schedule": {str(s): [f(leaf), 100] for s, f in HAND_SET.items()},
                    "tuning_gain": t_hand / t_batch, "identical": same_hand},
    }
    if own:
        engine.close()
    return out


# ---------------------------------------------------------------------------------------
# Serving form: continuous batching of string-key build requests under an HBM budget
# ---------------------------------------------------------------------------------------
SERVE_CLASSES = [(8, 100), (12, 1000), (16, 2000)]


def string_pool(n: int, seed: int = 2024):
    """n random byte strings of 10..50 bytes (numpy default_rng(seed)), concatenated."""
    rng = np.random.default_rng(seed)
    lens = rng.integers(10, 51, n)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    data = rng.integers(0, 256, int(offsets[-1]), dtype=np.uint8)
    return data, offsets


def serve_requests(nreq: int, pool_n: int, max_keys: int, seed: int = 11):
    """Request i: size round(exp(U[ln 100, ln max_keys])), class uniform over (l, b), a
    contiguous slice of the string pool at a uniform offset."""
    rng = np.random.default_rng(seed)
    sizes = np.rint(np.exp(rng.uniform(np.log(100), np.log(max_keys), nreq))).astype(np.int64)
    cls = rng.integers(0, len(SERVE_CLASSES), nreq)
    starts = [int(rng.integers(0, pool_n - s + 1)) for s in sizes]
    return [(int(st), int(sz), SERVE_CLASSES[c]) for st, sz, c in zip(starts, sizes, cls)]


def measure_serve(requests: int = 100, max_keys: int = 10_000_000, hbm_budget: int = 32 << 30, inflight: int = 2,
                  load: float = 0.75) -> dict:
    """Serving form: a saturated leg (every request queued at once: capacity), a Poisson leg at
    `load` x capacity (p50/p99 latency), and each request alone (identity and sequential rate)."""
    import threading

    import torch
    import gpurecsplit_b200 as rsb

    torch.cuda.set_device(0)
    data, offsets = string_pool(max_keys)
    reqs = serve_requests(requests, max_keys, max_keys)
    total_keys = sum(r[1] for r in reqs)

    def keys_of(r):
        st, n, _ = r
        return data, offsets[st:st + n + 1]

    def submit(srv, r):
        _, _, (leaf, b) = r
        return srv.submit_strings(keys_of(r), b, leaf)

    srv = rsb.Server(hbm_budget=hbm_budget, inflight=inflight)
    # Warm-up: 1M-key requests of every class on every worker size the engines' scratch.
    wn = min(1_000_000, max_keys)
    warm = [srv.submit_strings((data, offsets[:wn + 1]), b, leaf)
            for _ in range(inflight) for leaf, b in SERVE_CLASSES]
    for w in warm:
        srv.wait(w)

    with ClockSampler(0) as clocks:
        # Saturated leg: every request queued at once -> capacity.
        t0 = time.perf_counter()
        ids = [submit(srv, r) for r in reqs]
        sat = [srv.wait(i) for i in ids]
        t_sat = time.perf_counter() - t0
        capacity = total_keys / t_sat

        # Poisson leg at `load` x capacity (arrival rate in requests/s).
        rate = load * capacity / (total_keys / len(reqs))
        gaps = np.random.default_rng(5).exponential(1.0 / rate, len(reqs))
        ids = [None] * len(reqs)
        lag = []

        def submitter():
            start = time.perf_counter()
            t_next = 0.0
            for i, r in enumerate(reqs):
                t_next += gaps[i]
                d = t_next - (time.perf_counter() - start)
                if d > 0:
                    time.sleep(d)
                lag.append(max(0.0, -d))
                ids[i] = submit(srv, r)

        th = threading.Thread(target=submitter)
        t1 = time.perf_counter()
        th.start()
        th.join()
        poi = [srv.wait(i) for i in ids]
        t_poi = time.perf_counter() - t1
    srv.close()

    lat = np.array([(info["done_s"] - info["submit_s"]) * 1e3 for _, info in poi])
    qwait = np.array([(info["admit_s"] - info["submit_s"]) * 1e3 for _, info in poi])
    batch_req = np.array([info["batch_requests"] for _, info in poi])

    # Each request alone (plain build, one engine, back to back): identity + sequential rate.
    engine = rsb.Engine(0)
    same = True
    t2 = time.perf_counter()
    for r, (fs, _), (fp, _) in zip(reqs, sat, poi):
        _, _, (leaf, b) = r
        alone = rsb.GPURecSplit(keys_of(r), bucket_size=b, leaf_size=leaf, key_type="strings", engine=engine)
        blob = alone.serialize()
        same &= blob == fs.serialize() and blob == fp.serialize()
        alone.close()
    t_alone = time.perf_counter() - t2
    engine.close()

    per_class = {}
    for (st, n, (leaf, b)), l_ms in zip(reqs, lat):
        per_class.setdefault(f"l={leaf},b={b}", []).append(l_ms)
    # every function handed out by the server is closed here; the alone builds were closed above
    for f, _ in sat + poi:
        f.close()
    return {
        "metric": "serve keys/s (string requests, log-uniform [100,1e7] keys, mixed (l,b))",
        "value": capacity, "unit": "keys/s", "higher_is_better": True, "n_gpus": 1, "steps": 1, "warmup": 1,
        "ms_per_step": t_sat * 1e3, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"{len(reqs)} requests; size round(exp(U[ln 100, ln {max_keys:.0e}])), "
                               f"(l,b) uniform over {SERVE_CLASSES}, keys = slices of a pool of {max_keys} "
                               "random 10-50 byte strings (numpy seed 2024), rotation",
                   "requests": len(reqs), "keys": total_keys, "hbm_budget": hbm_budget,
                   "inflight": inflight, "timing": "host wall clock (server steady clock for latency)"},
        "saturated": {"keys_per_s": capacity, "s": t_sat,
                      "mean_batch_requests": float(np.mean([i["batch_requests"] for _, i in sat]))},
        "poisson": {"load": load, "rate_req_per_s": rate, "keys_per_s": total_keys / t_poi, "s": t_poi,
                    "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                    "queue_p50_ms": float(np.percentile(qwait, 50)), "queue_p99_ms": float(np.percentile(qwait, 99)),
                    "mean_batch_requests": float(batch_req.mean()), "max_submit_lag_ms": 1e3 * max(lag),
                    "p50_ms_by_class": {k: float(np.percentile(v, 50)) for k, v in per_class.items()},
                    "p99_ms_by_class": {k: float(np.percentile(v, 99)) for k, v in per_class.items()}},
        "alone_back_to_back": {"keys_per_s": total_keys / t_alone, "s": t_alone},
        "speedup_vs_alone": t_alone / t_sat,
        "identical_to_alone": bool(same),
        "clocks": clocks.summary(),
    }


def measure_pipeline(reps: int = 3) -> dict:
    """Stage kernels against pipeline mode (rsb_engine_set_pipeline) on the same builds: the
    device time of each build (CUDA events around the public call with device-resident keys,
    best of `reps`) and whether both modes serialize to the same bytes."""
    import torch
    import gpurecsplit_b200 as rsb
    torch.cuda.set_device(0)
    st = torch.cuda.current_stream()
    cases = [("u64 n=5M l=16 b=2000", 5_000_000, 16, 2000, 42), ("u64 n=1M l=12 b=1000", 1_000_000, 12, 1000, 42),
             ("u64 n=1M l=8 b=100", 1_000_000, 8, 100, 42), ("u64 n=200k l=20 b=2000", 200_000, 20, 2000, 43)]

    def best_ms(fn):
        out = []
        for _ in range(reps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(st)
            r = fn()
            b.record(st)
            b.synchronize()
            out.append(a.elapsed_time(b))
            for f in (r[0] if isinstance(r, tuple) else [r]):
                f.close()
        return round(min(out), 3)

    rows = {}
    for pipe in (False, True):
        e = rsb.Engine(0, st.cuda_stream)
        e.set_pipeline(pipe)
        for name, n, leaf, b, seed in cases:
            keys = torch.from_numpy(splitmix64_keys(seed, n).view(np.int64)).cuda()
            torch.cuda.synchronize()
            fn = (lambda k=keys, n=n, b=b, leaf=leaf:
                  rsb.GPURecSplit.from_device(k.data_ptr(), n, b, leaf, key_type="u64", engine=e, device_only=True))
            f = fn()
            blob = f.serialize()
            f.close()
            row = rows.setdefault(name, {})
            row["pipeline_ms" if pipe else "stages_ms"] = best_ms(fn)
            row["sha256_" + ("pipeline" if pipe else "stages")] = hashlib.sha256(blob).hexdigest()
            del keys
        k, off = batch_workload(1000)
        d = torch.from_numpy(k.view(np.int64)).cuda()
        torch.cuda.synchronize()
        fn = lambda: rsb.build_batch(d.data_ptr(), off, 1000, 12, key_type="u64", engine=e, keys_on_device=True)
        row = rows.setdefault("1000 sets (%d u64 keys) l=12 b=1000" % int(off[-1]), {})
        row["pipeline_ms" if pipe else "stages_ms"] = best_ms(fn)
        del d
        e.close()
    for row in rows.values():
        if "sha256_stages" in row:
            row["identical"] = row.pop("sha256_stages") == row.pop("sha256_pipeline")
    return {"mode": "pipeline", "unit": "ms", "workloads": rows}


def measure_builds(n: int, leaf: int, bucket: int, builds: int, pipeline: bool = False) -> dict:
    """`builds` plain builds of n splitmix64 u64 keys (seed 42) on one engine (in pipeline mode
    with `pipeline`), for profiling the search kernels on a chosen size: the per-stage
    evaluations, times and windows of the last build."""
    import gpurecsplit_b200 as rsb
    e = rsb.Engine(0)
    e.set_pipeline(pipeline)
    keys = splitmix64_keys(42, n)
    st = None
    for _ in range(builds):
        f = rsb.GPURecSplit(keys, bucket_size=bucket, leaf_size=leaf, key_type="u64", engine=e)
        st = f.stats()
        f.close()
    e.close()
    stages = {s: {"evals": int(st["evals_stage"][s]), "ms": round(st["ms_search"][s], 3),
                  "windows": int(st["windows_stage"][s])} for s in range(17, 21)}
    return {"mode": "build", "n": n, "leaf": leaf, "bucket": bucket, "builds": builds, "pipeline": pipeline,
            "stages": stages}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="rsb", choices=["rsb", "reference"])
    ap.add_argument("--n", type=int, default=N_KEYS)
    ap.add_argument("--cpu-fraction", type=int, default=5, help="CPU baseline sample: 1/N of the workload's buckets")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="plain", choices=["plain", "batch", "serve", "c1", "c3", "pipeline", "build"])
    ap.add_argument("--sets", type=int, default=1000)
    ap.add_argument("--leaf", type=int, default=16, help="--mode build: leaf size")
    ap.add_argument("--bucket", type=int, default=2000, help="--mode build: bucket size")
    ap.add_argument("--builds", type=int, default=2, help="--mode build: builds on one engine")
    ap.add_argument("--pipeline", action="store_true", help="--mode build: in pipeline mode")
    ap.add_argument("--requests", type=int, default=100)
    ap.add_argument("--max-keys", type=int, default=10_000_000)
    ap.add_argument("--hbm-budget", type=int, default=32 << 30)
    ap.add_argument("--inflight", type=int, default=2)
    ap.add_argument("--load", type=float, default=0.75)
    ap.add_argument("--no-extras", action="store_true", help="omit the c1/c3/c4_batch/c5_serve keys of the default line")
    args = ap.parse_args()
    if args.mode == "batch":
        print(json.dumps(measure_batch(args.sets)), flush=True)
        return
    if args.mode == "build":
        print(json.dumps(measure_builds(args.n, args.leaf, args.bucket, args.builds, args.pipeline)), flush=True)
        return
    if args.mode == "pipeline":
        print(json.dumps(measure_pipeline()), flush=True)
        return
    if args.mode == "serve":
        print(json.dumps(measure_serve(args.requests, args.max_keys, args.hbm_budget, args.inflight, args.load)),
              flush=True)
        return
    if args.mode in CONFIGS:
        print(json.dumps(measure_config(args.mode, steps=args.steps, warmup=max(args.warmup, 3))), flush=True)
        return
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
