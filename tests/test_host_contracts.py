"""Host-side contracts that need no GPU: the C++ drop-in header compiles and links against
librsb.so as a program written for the reference would, and the CPU reference arm of
bench.py prints the JSON line the benchmark driver reads."""
import json
import os
import shutil
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_dropin_compiles_and_links(tmp_path, rsb):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    lib_dir = os.path.dirname(rsb.LIB_PATH)
    exe = tmp_path / "dropin_test"
    subprocess.run([cxx, "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_test.cpp"), "-L", lib_dir, "-lrsb",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    assert exe.exists()


def test_reference_arm_json_contract():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "2",
                        "--warmup", "3", "--n", "40000"], capture_output=True, text=True, timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "dtype", "data", "config", "impl", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference"
    assert line["unit"] == "ns/key" and line["higher_is_better"] is False
    assert line["value"] > 0 and line["e2e"]["value"] == line["value"]
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    # the reference line's config is the GPU arm's config, so the two are the same workload
    sys.path.insert(0, ROOT)
    import bench
    assert line["config"] == bench.workload_config(40000, 1)


def test_cpu_bucket_ranges_rebuild_the_full_builds_searches(oracle_mod):
    """bench.py times CPU builds on contiguous bucket ranges of the workload: each range,
    built as its own function, must have the full build's bucket sizes and DFS seeds for those
    buckets, so that ranges covering the workload do its search work exactly once."""
    sys.path.insert(0, ROOT)
    import bench
    import numpy as np
    n = 40_000
    simd = oracle_mod.simd_supported()
    work = bench.CpuWorkload(n)
    full = oracle_mod.build_mphf(oracle_mod.hash_u64(bench.splitmix64_keys(bench.SEED, n)), bench.LEAF,
                                 bench.BUCKET, simd=simd)
    seeds = []
    for lo, hi in work.ranges(3):
        keys, b = work.range_keys(lo, hi)
        part = oracle_mod.build_mphf(keys, bench.LEAF, b, simd=simd)
        assert np.array_equal(np.diff(part.bucket_size_acc), np.diff(full.bucket_size_acc)[lo:hi])
        seeds.append(part.seeds)
    assert np.array_equal(np.concatenate(seeds), full.seeds)
