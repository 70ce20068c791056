"""Autotuner of the seed-search stage schedules.

Every persistent search stage (17 upper aggregation, 18 lower aggregation, 19 rotation
leaves) has a schedule: candidates per lane of a search window (aggregation: 4, 8, 12 or
16 seeds; rotation leaves: 4, 8 or 12 bases) and the share of full occupancy its grid keeps.
Larger windows amortise a window's per-key work over more candidates; smaller ones overshoot
a node's minimum seed by less and keep more warps busy at the end of a stage. The best
choice depends on the leaf size (node sizes, seeds per node) and on the size of the build
(how long a stage's tail is), so the table is keyed by (leaf size, stage, size class), size
class 0 below 2^20 keys, 1 from 2^20 and 2 from 2^24 (tuned on 2^17 and 3 * 2^18, 2^20 and 2^24
keys).

For each leaf size and size class the tuner builds a synthetic workload (uniform random
64-bit keys, the bucket size usual for that leaf size) of each of the class's sizes with every
candidate schedule - all three stages take their k-th candidate in the same build, since each
stage is its own launch with its own CUDA-event time - keeps for each stage the schedule with
the least median stage time (over two sizes: the least summed time relative to each size's
fastest), and checks that every build's serialized function is identical to the build with the
built-in schedule (a schedule never changes the minimum seeds). Results go to
gpurecsplit_b200/schedules.json (measurements) and gpurecsplit_b200/csrc/rsb_schedules.inc
(the table compiled into librsb.so as its built-in schedules; rebuild after tuning); entries
of leaf sizes and classes not measured in this run are kept from the existing schedules.json.

    python -m gpurecsplit_b200.tune [--leaves 4-20] [--classes 0,1,2] [--repeats 3] [--out DIR]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
STAGES = {17: (4, 8, 12, 16), 18: (4, 8, 12, 16), 19: (4, 8, 12)}
OCCUPANCY = (100, 75)
# Workload sizes per class. Class 0 spans an 8x range of sizes below 2^20 over which a stage's
# best window changes (at 2^17 keys 12 bases per lane win the l = 8 leaves by 6 %, at 1M keys
# they lose by 25 %), so it is measured at both ends and each stage takes the schedule with
# the least summed relative time (time / fastest time at that size).
CLASS_KEYS = {0: (1 << 17, 3 << 18), 1: (1 << 20,), 2: (1 << 24,)}


def bucket_size_for(leaf: int) -> int:
    """The bucket size the workloads of a leaf size use (the reference's configurations:
    l=8 b=100, l=12 b=1000, l=16 b=2000, l=24 b=2000)."""
    return 100 if leaf <= 8 else (1000 if leaf <= 14 else 2000)


def keys_for(leaf: int, size_class: int) -> tuple:
    """Keys of the tuning workloads: the size class's sizes, fewer for slow leaf sizes of
    class 0 (l >= 20 needs tens of microseconds per key)."""
    if size_class == 0 and leaf >= 20:
        return (1 << 14,)
    if size_class == 0 and leaf >= 17:
        return CLASS_KEYS[0][:1]
    return CLASS_KEYS[size_class]


def splitmix64(seed: int, n: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def measure(rsb, engine, leaf: int, size_class: int, n: int, repeats: int) -> dict:
    """Median stage times {stage: {(candidates, occupancy): ms}} of every candidate schedule
    on one n-key workload; every build's bytes must equal the built-in schedule's."""
    import torch
    b = bucket_size_for(leaf)
    keys = torch.from_numpy(splitmix64(1000 + leaf, n).view(np.int64)).cuda()
    torch.cuda.synchronize()

    def build():
        f = rsb.GPURecSplit.from_device(keys.data_ptr(), n, b, leaf, key_type="u64", engine=engine,
                                        device_only=False)
        st, blob = f.stats(), f.serialize()
        f.close()
        return st, blob

    for stage in STAGES:
        engine.set_schedule(leaf, stage, size_class, 0)
    build()  # warm-up: kernels loaded, scratch sized
    _, reference = build()
    # the k-th build takes every stage's k-th candidate (a stage's last one once it has no more)
    configs = [(k, pct) for pct in OCCUPANCY for k in range(max(len(c) for c in STAGES.values()))]
    times = {stage: {} for stage in STAGES}
    for k, pct in configs:
        for stage, cands in STAGES.items():
            engine.set_schedule(leaf, stage, size_class, cands[min(k, len(cands) - 1)], pct)
        ms = {stage: [] for stage in STAGES}
        for _ in range(repeats):
            st, blob = build()
            if blob != reference:
                raise RuntimeError(f"schedule {k}/{pct} changed the function at l={leaf}")
            for stage in STAGES:
                ms[stage].append(st["ms_search"][stage])
        for stage, cands in STAGES.items():
            times[stage].setdefault((cands[min(k, len(cands) - 1)], pct), statistics.median(ms[stage]))
    for stage in STAGES:
        engine.set_schedule(leaf, stage, size_class, 0)
    return times


def choose(times_by_size: list) -> tuple:
    """The schedule of one stage from its median times at one or more workload sizes
    ([{(candidates, occupancy): ms}, ...], the same schedules at every size): the least summed
    time relative to each size's fastest. Returns (schedule, {schedule: score})."""
    score = {c: sum(t[c] / min(t.values()) for t in times_by_size) for c in times_by_size[0]}
    return min(score, key=score.get), score


def tune_one(rsb, engine, leaf: int, size_class: int, repeats: int, log) -> list:
    """Measures every candidate schedule for one (leaf, size class) at each of the class's
    sizes; returns table entries."""
    sizes = keys_for(leaf, size_class)
    per_size = {n: measure(rsb, engine, leaf, size_class, n, repeats) for n in sizes}
    out = []
    for stage in STAGES:
        default = engine.schedule(leaf, stage, size_class)
        t = per_size[sizes[0]][stage]
        best, score = choose([per_size[n][stage] for n in sizes])
        entry = {"leaf": leaf, "stage": stage, "size_class": size_class, "seeds_per_lane": best[0],
                 "occupancy_pct": best[1], "ms_best": round(t[best], 4), "ms_builtin": round(t.get(default, -1), 4),
                 "builtin": list(default), "keys": sizes[0], "bucket_size": bucket_size_for(leaf),
                 "ms": {f"{s}/{p}": round(v, 4) for (s, p), v in sorted(t.items())}}
        if len(sizes) > 1:  # the choice minimises the summed relative time over the sizes
            entry["score"] = {f"{s}/{p}": round(v, 4) for (s, p), v in sorted(score.items())}
            entry["ms_at"] = {str(n): {f"{s}/{p}": round(v, 4) for (s, p), v in sorted(per_size[n][stage].items())}
                              for n in sizes[1:]}
        out.append(entry)
        log(json.dumps(entry))
    return out


def write_table(entries: list, out_dir: str) -> None:
    old = os.path.join(out_dir, "schedules.json")
    if os.path.exists(old):  # keep the entries this run did not measure
        measured = {(e["leaf"], e["stage"], e["size_class"]) for e in entries}
        entries = entries + [e for e in json.load(open(old))["entries"]
                             if (e["leaf"], e["stage"], e["size_class"]) not in measured]
    entries = sorted(entries, key=lambda e: (e["leaf"], e["stage"], e["size_class"]))
    with open(os.path.join(out_dir, "schedules.json"), "w") as f:
        json.dump({"how": "python -m gpurecsplit_b200.tune", "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime()),
                   "entries": entries}, f, indent=1)
    lines = ["// Tuned stage schedules: {leaf size, stage, size class, candidates per lane, occupancy %}.",
             "// Written by gpurecsplit_b200/tune.py from measurements on one B200 (gpurecsplit_b200/schedules.json)."]
    for e in entries:
        lines.append(f"    {{{e['leaf']}, {e['stage']}, {e['size_class']}, {e['seeds_per_lane']}, {e['occupancy_pct']}}},")
    os.makedirs(os.path.join(out_dir, "csrc"), exist_ok=True)
    with open(os.path.join(out_dir, "csrc", "rsb_schedules.inc"), "w") as f:
        f.write("\n".join(lines) + "\n")


def parse_leaves(spec: str) -> list:
    out = []
    for part in spec.split(","):
        if "-" in part:
            a, b = part.split("-")
            out += list(range(int(a), int(b) + 1))
        else:
            out.append(int(part))
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--leaves", default="4-20")
    ap.add_argument("--classes", default="0,1,2")
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--out", default=HERE, help="directory holding schedules.json and csrc/rsb_schedules.inc")
    ap.add_argument("--log", default=None)
    args = ap.parse_args()
    import torch
    import gpurecsplit_b200 as rsb
    torch.cuda.set_device(0)
    engine = rsb.Engine(0, torch.cuda.current_stream().cuda_stream)
    logf = open(args.log, "a") if args.log else None

    def log(s):
        print(s, flush=True)
        if logf:
            logf.write(s + "\n")
            logf.flush()

    entries = []
    for leaf in parse_leaves(args.leaves):
        for c in [int(x) for x in args.classes.split(",")]:
            if (c == 1 and leaf > 18) or (c == 2 and leaf > 16):
                continue  # builds that take minutes each: they use the next smaller class's result
            entries += tune_one(rsb, engine, leaf, c, args.repeats, log)
    for e in [e for e in entries if e["size_class"] == 0 and e["leaf"] > 18]:
        entries.append(dict(e, size_class=1, copied_from_size_class=0))
    for e in [e for e in entries if e["size_class"] == 1 and e["leaf"] > 16]:
        entries.append(dict(e, size_class=2, copied_from_size_class=e.get("copied_from_size_class", 1)))
    engine.close()
    write_table(entries, args.out)


if __name__ == "__main__":
    main()
