"""Generates tests/golden/golden_builds.json: SHA-256 digests of full-size reference builds.

Each entry names a seeded synthetic workload (key kind, seed, n, leaf size, bucket size,
rotation) and the SHA-256 of the serialized function that the reference's own SIMDRecSplit
(compiled from its sources into oracle/_ref/ by oracle/Makefile) builds for it. Where this
project's CPU oracle finishes in reasonable time it builds the workload too and the two
digests must be equal; the entry records which builds produced it. The GPU tests build the
same workloads on the device and compare digests, which checks full-size builds bit for bit
without running a CPU build on the GPU box.

    python tests/golden/make_golden.py [--no-oracle] [--simd] [--redo] [--threads=T] [name ...]

With no names every missing entry is made (--redo: every entry). --simd uses the oracle's
AVX-512 search loops (byte-identical to its scalar build) for the cross-check; --no-oracle
skips the cross-check (workloads the oracle needs hours for). The reference tree must be
present to build oracle/_ref (see oracle.reference_tree()).
"""
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle  # noqa: E402

OUT = os.path.join(HERE, "golden_builds.json")

# name -> (key kind, seed, n, leaf, bucket, rotate)
WORKLOADS = {
    "strings_n1M_l8_b100": ("strings", 42, 1_000_000, 8, 100, True),
    "u64_n5M_l16_b2000": ("u64", 42, 5_000_000, 16, 2000, True),
    "u64_n200k_l24_b2000": ("u64", 43, 200_000, 24, 2000, True),
    "hash128_n1M_l8_b100": ("hash128", 42, 1_000_000, 8, 100, True),
    "hash128_n100k_l12_b1000": ("hash128", 7, 100_000, 12, 1000, True),
    "hash128_n50k_l8_b2000_bf": ("hash128", 3, 50_000, 8, 2000, False),
    "u64_n100k_l16_b2000": ("u64", 42, 100_000, 16, 2000, True),
    # README.md:19-22 row (l=18, b=50, 5M keys, ~1.709 bits/key)
    "u64_n5M_l18_b50": ("u64", 44, 5_000_000, 18, 50, True),
    # small buckets: more than 12,288 buckets per build (the device's global-histogram path)
    "hash128_n1M_l8_b2": ("hash128", 45, 1_000_000, 8, 2, True),
    "hash128_n1M_l8_b5": ("hash128", 46, 1_000_000, 8, 5, True),
    "hash128_n1M_l5_b10": ("hash128", 47, 1_000_000, 5, 10, True),
    # the sizes of the reference's equivalence grid (test/GPUandSIMDequivalence.cu:8-11)
    "hash128_n12345678_l8_b100": ("hash128", 48, 12_345_678, 8, 100, True),
    "hash128_n10M_l4_b25": ("hash128", 49, 10_000_000, 4, 25, True),
    "hash128_n10M_l2_b2": ("hash128", 50, 10_000_000, 2, 2, True),
}


def keys_for(kind, seed, n):
    if kind == "hash128":
        return oracle.keygen_hash128(seed, n)
    if kind == "u64":
        return oracle.hash_u64(oracle.keygen_u64(seed, n))
    if kind == "strings":
        data, offsets = oracle.keygen_strings(seed, n)
        return oracle.hash_strings(data, offsets)
    raise ValueError(kind)


def main(args):
    flags = {a.split("=")[0] for a in args if a.startswith("--")}
    threads = int(next((a.split("=")[1] for a in args if a.startswith("--threads=")), 0)) or os.cpu_count()
    names = [a for a in args if not a.startswith("--")]
    oracle.build()
    if not oracle.ref_available():
        raise SystemExit("oracle/_ref is not built or this CPU cannot run it")
    db = json.load(open(OUT)) if os.path.exists(OUT) else {}
    todo = names or [k for k in WORKLOADS if "--redo" in flags or k not in db or "ref_sha256" not in db[k]]
    for name in todo:
        kind, seed, n, leaf, b, rot = WORKLOADS[name]
        keys = keys_for(kind, seed, n)
        t = time.time()
        ref = oracle.ref_build(keys, leaf, b, rot, threads=threads)
        t_ref = time.time() - t
        digest = hashlib.sha256(ref.tobytes()).hexdigest()
        entry = {
            "kind": kind, "seed": seed, "n": n, "leaf": leaf, "bucket": b, "rotate": rot,
            "sha256": digest, "ref_sha256": digest, "bytes": int(ref.size),
            "bits": oracle.ref_get_bits(ref, leaf, rot), "ref_seconds": round(t_ref, 1),
            "ref_threads": threads, "cpu": oracle.cpu_model(),
        }
        if "--no-oracle" not in flags:
            t = time.time()
            res = oracle.build_mphf(keys, leaf, b, rot, threads=threads, simd="--simd" in flags)
            entry["oracle_seconds"] = round(time.time() - t, 1)
            entry["oracle_build"] = "avx512 search loops" if "--simd" in flags else "scalar"
            entry["oracle_sha256"] = hashlib.sha256(res.bytes.tobytes()).hexdigest()
            entry["nodes"] = int(res.seeds.size)
            entry["evals_alg"] = res.evals_alg
            if entry["oracle_sha256"] != digest:
                raise SystemExit(f"{name}: the oracle's build differs from the reference's")
        elif name in db:
            old = db[name]
            if old.get("sha256") not in (None, digest):
                raise SystemExit(f"{name}: the reference's build differs from the recorded oracle digest")
            for k in ("oracle_seconds", "oracle_build", "oracle_threads", "nodes", "evals_alg"):
                if k in old:
                    entry[k] = old[k]
            if "sha256" in old:
                entry["oracle_sha256"] = old["sha256"]
        print(name, entry, flush=True)
        cur = json.load(open(OUT)) if os.path.exists(OUT) else {}
        cur[name] = entry
        with open(OUT, "w") as f:
            json.dump(cur, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
