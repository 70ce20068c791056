"""The C++ drop-in class (include/function/GPURecSplit.cuh) compiled from a program written
against the reference's API: it builds on the GPU, round-trips through operator<< / >>,
rejects duplicates with an exception, and its serialized bytes equal the oracle's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpp_dropin(tmp_path, oracle_mod, rsb):
    cxx = shutil.which("g++") or shutil.which("c++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    lib_dir = os.path.dirname(rsb.LIB_PATH)
    exe = tmp_path / "dropin_test"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "dropin_test.cpp"), "-L", lib_dir, "-lrsb",
                    f"-Wl,-rpath,{lib_dir}", "-o", str(exe)], check=True)
    out = tmp_path / "f.bin"
    r = subprocess.run([str(exe), str(out)], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "dropin ok" in r.stdout
    keys = oracle_mod.keygen_hash128(0x5603141978c51071, 100000)
    ref = oracle_mod.build_mphf(keys, 8, 100)
    assert out.read_bytes() == ref.bytes.tobytes()
    if oracle_mod.ref_available():
        # getBits() as the reference's own SIMDRecSplit reports it for the same bytes
        bits = int(next(l for l in r.stdout.splitlines() if l.startswith("getBits ")).split()[1])
        assert bits == oracle_mod.ref_get_bits(ref.bytes, 8)
