"""Generates tests/golden/golden_builds.json: SHA-256 digests of oracle-built functions.

Each entry names a seeded synthetic workload (key kind, seed, n, leaf size, bucket size,
rotation) and the SHA-256 of the oracle's serialized function for it. The GPU tests build
the same workload on the device and compare digests, which checks full-size builds
bit for bit without running the scalar oracle on the GPU box.

    python tests/golden/make_golden.py [--simd] [name ...]   # default: every missing entry

--simd builds with the oracle's AVX-512 search loops (oracle/_build/libsimdrs.so), which
tests/test_oracle.py checks byte for byte against the scalar oracle; the entry records which
build produced it. It is used for workloads the scalar build needs hours for (l = 24).
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
    simd = "--simd" in args
    names = [a for a in args if a != "--simd"]
    db = json.load(open(OUT)) if os.path.exists(OUT) else {}
    todo = names or [k for k in WORKLOADS if k not in db]
    for name in todo:
        kind, seed, n, leaf, b, rot = WORKLOADS[name]
        t = time.time()
        keys = keys_for(kind, seed, n)
        res = oracle.build_mphf(keys, leaf, b, rot, simd=simd)
        dt = time.time() - t
        db[name] = {
            "kind": kind, "seed": seed, "n": n, "leaf": leaf, "bucket": b, "rotate": rot,
            "sha256": hashlib.sha256(res.bytes.tobytes()).hexdigest(), "bytes": int(res.bytes.size),
            "bits": oracle.get_bits(res.bytes), "nodes": int(res.seeds.size), "evals_alg": res.evals_alg,
            "oracle_seconds": round(dt, 1), "oracle_threads": os.cpu_count(),
            "oracle_build": "avx512 search loops" if simd else "scalar",
        }
        print(name, db[name], flush=True)
        cur = json.load(open(OUT)) if os.path.exists(OUT) else {}
        cur[name] = db[name]
        with open(OUT, "w") as f:
            json.dump(cur, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
