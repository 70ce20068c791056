"""Pins the CPU oracle to the reference's own code (CPU only, no GPU).

oracle/_ref/libref_simdrs.so is GpuRecSplit's SIMDRecSplit compiled from its unmodified
sources (include/function/SIMDRecSplit.hpp, AbstractParallelRecSplit.hpp, RiceBitVector.hpp,
DoubleEF.hpp, golombRiceMemo.hpp, support/common.hpp) with stand-ins for its empty
submodules. These tests check, byte for byte, that the oracle builds what the reference
builds over the reference's correctness grid (test/correctness.hpp:24-27, sizes capped so
the suite stays short), that the reference's operator>> / operator() read the oracle's
functions as the oracle does, and that the reference's own encoders (RiceBitVector::Builder,
DoubleEF) turn the oracle's seeds into the oracle's bytes. The GPU tests then compare the
device with both.
"""
import hashlib
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden", "golden_builds.json")
SEED = 0x5603141978c51071  # the reference tests' key seed (test/correctness.hpp:40)


@pytest.fixture(scope="module")
def ref(oracle_mod):
    if not oracle_mod.ref_available():
        if oracle_mod.reference_tree() is not None and oracle_mod.simd_supported():
            pytest.fail("the reference tree is present but oracle/_ref was not built")
        pytest.skip("oracle/_ref is not built here or this CPU lacks AVX-512")
    return oracle_mod


def _grid(leaf):
    """(bucket size, n) pairs of the correctness grid, capped by leaf size for CPU time."""
    sizes = [1, 10, 100, 123]
    if leaf <= 14:
        sizes.append(2000)
    if leaf > 20:
        sizes = [1, 10, 123]
    for b in (2, 5, 10, 25, 100, 483, 2000):
        for n in sizes:
            yield b, n


@pytest.mark.parametrize("leaf", range(2, 25))
def test_reference_builds_what_the_oracle_builds(ref, leaf):
    for b, n in _grid(leaf):
        keys = ref.keygen_hash128(SEED + 1000 * leaf + n, n)
        want = ref.build_mphf(keys, leaf, b, simd=leaf >= 15 and ref.simd_supported()).bytes
        got = ref.ref_build(keys, leaf, b)
        assert np.array_equal(got, want), (leaf, b, n)


@pytest.mark.parametrize("leaf,b,n", [(8, 2000, 5000), (5, 3, 3000), (12, 100, 1000), (16, 2000, 4000)])
def test_reference_without_rotation(ref, leaf, b, n):
    keys = ref.keygen_hash128(SEED ^ n, n)
    assert np.array_equal(ref.ref_build(keys, leaf, b, rotate=False), ref.build_mphf(keys, leaf, b, False).bytes)


def test_reference_larger_builds(ref):
    for leaf, b, n, kind in [(8, 100, 300_000, "hash128"), (12, 1000, 200_000, "u64"), (16, 2000, 20_000, "u64"),
                             (4, 2, 100_000, "hash128"), (10, 7, 50_000, "hash128")]:
        keys = ref.keygen_hash128(7 + n, n) if kind == "hash128" else ref.hash_u64(ref.keygen_u64(7 + n, n))
        want = ref.build_mphf(keys, leaf, b, simd=ref.simd_supported()).bytes
        assert np.array_equal(ref.ref_build(keys, leaf, b), want), (leaf, b, n)


def test_empty_set_differs_only_in_the_undefined_field(ref):
    """n = 0: the reference computes bits_per_key_fixed_point as 2^20 * (0 / 0.0) and
    converts the NaN to uint64_t (DoubleEF.hpp:144), which C++ leaves undefined; its AVX-512
    build yields 2^64 - 1, SSE/AVX2 builds 2^63 (this project's value). Every other byte is
    the same."""
    keys = np.zeros((0, 2), dtype=np.uint64)
    got = ref.ref_build(keys, 8, 100).view(np.uint64).copy()
    want = ref.build_mphf(keys, 8, 100).bytes.view(np.uint64).copy()
    assert got.size == want.size
    field = 10  # leaf, bucket, keys, descriptor count + 1 word, then five EF scalars
    assert want[field] == 1 << 63 and got[field] in (1 << 63, (1 << 64) - 1)
    got[field] = want[field] = 0
    assert np.array_equal(got, want)


def test_reference_query_reads_oracle_functions(ref):
    for leaf, b, n, rot in [(8, 100, 20000, True), (16, 2000, 6000, True), (12, 10, 5000, False), (3, 2, 777, True),
                            (24, 2000, 100, True)]:
        keys = ref.keygen_hash128(11 * n + leaf, n)
        f = ref.build_mphf(keys, leaf, b, rot, simd=ref.simd_supported())
        got = ref.ref_query(f.bytes, leaf, keys, rot)
        assert np.array_equal(got, ref.query(f.bytes, keys, rot))
        assert np.array_equal(np.sort(got), np.arange(n, dtype=np.uint64))


def test_reference_encoders_turn_oracle_seeds_into_oracle_bytes(ref):
    for leaf, b, n, rot in [(8, 100, 100_000, True), (16, 2000, 20_000, True), (5, 2, 10_000, True),
                            (12, 1000, 50_000, False), (24, 50, 300, True), (2, 7, 1, True), (8, 3000, 2999, True)]:
        keys = ref.keygen_hash128(13 * n + leaf, n)
        f = ref.build_mphf(keys, leaf, b, rot, simd=ref.simd_supported())
        bucket_keys = np.diff(f.bucket_size_acc)
        got = ref.ref_encode(bucket_keys, b, leaf, f.seeds, f.sizes, rot)
        assert np.array_equal(got, f.bytes), (leaf, b, n)


def test_checked_reference_build_self_verifies(ref):
    """The reference built with assertions (its DoubleEF checks every bucket after building,
    DoubleEF.hpp:351-364, and the searches assert their invariants) in a child process, so a
    failed assertion cannot end the test run: same bytes as the release build."""
    if not ref.ref_available(checked=True):
        pytest.skip("checked reference build missing")
    code = (
        "import sys, numpy as np; sys.path.insert(0, %r); import oracle\n"
        "for leaf, b, n in [(8, 100, 50000), (16, 2000, 6000), (4, 3, 20000), (11, 500, 4000)]:\n"
        "    k = oracle.keygen_hash128(n + leaf, n)\n"
        "    a = oracle.ref_build(k, leaf, b, checked=True)\n"
        "    f = oracle.build_mphf(k, leaf, b)\n"
        "    assert np.array_equal(a, oracle.ref_build(k, leaf, b)) and np.array_equal(a, f.bytes)\n"
        "    e = oracle.ref_encode(np.diff(f.bucket_size_acc), b, leaf, f.seeds, f.sizes, checked=True)\n"
        "    assert np.array_equal(e, f.bytes)\n"
        "print('checked ok')\n" % ROOT)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0 and "checked ok" in r.stdout, r.stdout + r.stderr


def test_golden_digests_come_from_the_reference(ref):
    """Every committed full-size digest was made by the reference's own build (and, where
    recorded, equals the oracle's); the quick ones are rebuilt here."""
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden
    db = json.load(open(GOLDEN))
    for name, g in db.items():
        assert g.get("ref_sha256") == g["sha256"], name
        if "oracle_sha256" in g:
            assert g["oracle_sha256"] == g["sha256"], name
    for name in ("hash128_n100k_l12_b1000", "hash128_n50k_l8_b2000_bf", "hash128_n1M_l8_b100", "strings_n1M_l8_b100",
                 "hash128_n1M_l8_b2"):
        kind, seed, n, leaf, b, rot = make_golden.WORKLOADS[name]
        blob = ref.ref_build(make_golden.keys_for(kind, seed, n), leaf, b, rot)
        assert hashlib.sha256(blob.tobytes()).hexdigest() == db[name]["sha256"], name


def test_reference_object_size_is_the_drop_in_constant(ref):
    # include/rsb/GPURecSplit.hpp adds kReferenceObjectBytes = 224 bytes in getBits()
    for leaf in (2, 8, 16, 24):
        assert ref.ref_object_size(leaf) == 224
