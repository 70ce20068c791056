"""Autotuner of the seed-search stage schedules.

Every persistent search stage (17 upper aggregation, 18 lower aggregation, 19 rotation
leaves) has a schedule: candidates per lane of a search window (aggregation: 8, 12 or 16
seeds; rotation leaves: 4, 8 or 12 bases) and the share of full occupancy its grid keeps.
Larger windows amortise a window's per-key work over more candidates; smaller ones overshoot
a node's minimum seed by less and keep more warps busy at the end of a stage. The best
choice depends on the leaf size (node sizes, seeds per node) and on the size of the build
(how long a stage's tail is), so the table is keyed by (leaf size, stage, size class), size
class 0 below 2^20 keys, 1 from 2^20 and 2 from 2^24 (tuned on 2^17, 2^20 and 2^24 keys).

For each leaf size and size class the tuner builds one synthetic workload (uniform random
64-bit keys, the bucket size usual for that leaf size) with every candidate schedule - all
three stages take their k-th candidate in the same build, since each stage is its own launch
with its own CUDA-event time - keeps for each stage the schedule with the least median stage
time, and checks that every build's serialized function is identical to the build with the
built-in schedule (a schedule never changes the minimum seeds). Results go to
gpurecsplit_b200/schedules.json (measurements) and gpurecsplit_b200/csrc/rsb_schedules.inc
(the table compiled into librsb.so as its built-in schedules; rebuild after tuning).

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
STAGES = {17: (8, 12, 16), 18: (8, 12, 16), 19: (4, 8, 12)}
OCCUPANCY = (100, 75)
CLASS_KEYS = {0: 1 << 17, 1: 1 << 20, 2: 1 << 24}


def bucket_size_for(leaf: int) -> int:
    """The bucket size the workloads of a leaf size use (the reference's configurations:
    l=8 b=100, l=12 b=1000, l=16 b=2000, l=24 b=2000)."""
    return 100 if leaf <= 8 else (1000 if leaf <= 14 else 2000)


def keys_for(leaf: int, size_class: int) -> int:
    """Keys of the tuning workload: the size class's size, fewer for slow leaf sizes of
    class 0 (l >= 20 needs tens of microseconds per key)."""
    n = CLASS_KEYS[size_class]
    if size_class == 0 and leaf >= 20:
        n = 1 << 14
    return n


def splitmix64(seed: int, n: int) -> np.ndarray:
    with np.errstate(over="ignore"):
        i = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + i * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def tune_one(rsb, engine, leaf: int, size_class: int, repeats: int, log) -> list:
    """Measures every candidate schedule for one (leaf, size class); returns table entries."""
    import torch
    n, b = keys_for(leaf, size_class), bucket_size_for(leaf)
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
    configs = [(k, pct) for pct in OCCUPANCY for k in range(3)]
    times = {stage: {} for stage in STAGES}
    for k, pct in configs:
        for stage, cands in STAGES.items():
            engine.set_schedule(leaf, stage, size_class, cands[k], pct)
        ms = {stage: [] for stage in STAGES}
        for _ in range(repeats):
            st, blob = build()
            if blob != reference:
                raise RuntimeError(f"schedule {k}/{pct} changed the function at l={leaf}")
            for stage in STAGES:
                ms[stage].append(st["ms_search"][stage])
        for stage, cands in STAGES.items():
            times[stage][(cands[k], pct)] = statistics.median(ms[stage])
    for stage in STAGES:
        engine.set_schedule(leaf, stage, size_class, 0)
    out = []
    for stage, t in times.items():
        default = engine.schedule(leaf, stage, size_class)
        best = min(t, key=t.get)
        entry = {"leaf": leaf, "stage": stage, "size_class": size_class, "seeds_per_lane": best[0],
                 "occupancy_pct": best[1], "ms_best": round(t[best], 4), "ms_builtin": round(t.get(default, -1), 4),
                 "builtin": list(default), "keys": n, "bucket_size": b,
                 "ms": {f"{s}/{p}": round(v, 4) for (s, p), v in sorted(t.items())}}
        out.append(entry)
        log(json.dumps(entry))
    return out


def write_table(entries: list, out_dir: str) -> None:
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
