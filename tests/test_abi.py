"""CPU checks of the C-ABI library (no device compute): it loads, exports every entry point
that include/rsb.h declares, and its host-side code (tables, deserialization, host queries,
serialization) agrees with the oracle on oracle-built functions."""
import hashlib
import json
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SEED = 0x5603141978c51071


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "rsb.h")).read()
    return sorted(set(re.findall(r"\b(rsb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(rsb):
    L = rsb.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s


def test_strerror_and_version(rsb):
    assert rsb.lib().rsb_version().startswith(b"rsb")
    for code in range(11):
        assert rsb.lib().rsb_strerror(code)


@pytest.mark.parametrize("leaf", range(2, 25))
def test_engine_memo_matches_reference_table(rsb, leaf):
    d = json.load(open(os.path.join(ROOT, "tests", "golden", "memo_digests.json")))["leaf"][str(leaf)]
    assert hashlib.sha256(rsb.golomb_memo(leaf).astype("<u4").tobytes()).hexdigest() == d["sha256"]


@pytest.mark.parametrize("n,leaf,b,rot", [(10000, 8, 100, True), (1000, 5, 3, True), (2000, 16, 2000, True),
                                          (5000, 8, 100, False), (1, 8, 100, True), (123, 2, 2, True),
                                          (0, 8, 100, True), (3000, 10, 231, True)])
def test_host_paths_agree_with_oracle(rsb, oracle_mod, n, leaf, b, rot):
    keys = oracle_mod.keygen_hash128(SEED, n)
    ref = oracle_mod.build_mphf(keys, leaf, b, rot)
    f = rsb.GPURecSplit.deserialize(ref.bytes.tobytes(), leaf, rot)
    assert f.serialize() == ref.bytes.tobytes()
    assert f.get_bits() == oracle_mod.get_bits(ref.bytes)
    if n:
        assert np.array_equal(f.query(keys), oracle_mod.query(ref.bytes, keys, rot))


def test_deserialize_rejects_wrong_leaf_and_truncation(rsb, oracle_mod):
    keys = oracle_mod.keygen_hash128(SEED, 500)
    blob = oracle_mod.build_mphf(keys, 8, 100).bytes.tobytes()
    with pytest.raises(rsb.RSBError) as e:
        rsb.GPURecSplit.deserialize(blob, 9)
    assert e.value.name == "FORMAT"
    for cut in (0, 7, 30, len(blob) - 1):
        with pytest.raises(rsb.RSBError):
            rsb.GPURecSplit.deserialize(blob[:cut], 8)


def test_engine_without_device_fails_cleanly(rsb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(rsb.RSBError) as e:
        rsb.Engine(0)
    assert e.value.name in ("NO_DEVICE", "CUDA")


def test_server_argument_checks(rsb):
    import ctypes
    L = rsb.lib()
    h = ctypes.c_void_p()
    assert L.rsb_server_create(0, 1 << 30, 0, 0, ctypes.byref(h)) == 1  # no workers
    assert L.rsb_server_create(0, 0, 1, 0, ctypes.byref(h)) == 1        # no budget
    assert L.rsb_server_create(0, 1 << 30, 1, 0, None) == 1
    rid = ctypes.c_uint64()
    assert L.rsb_server_submit_hash128(None, None, 0, 100, 8, 1, ctypes.byref(rid)) == 1
    assert L.rsb_server_wait(None, 1, 0.0, ctypes.byref(h), None) == 1
    assert L.rsb_server_destroy(None) == 1


def test_server_without_device_fails_cleanly(rsb):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(rsb.RSBError) as e:
        rsb.Server(hbm_budget=1 << 30, inflight=2)
    assert e.value.name in ("NO_DEVICE", "CUDA")


def test_engine_occupancy_argument_checks(rsb):
    L = rsb.lib()
    assert L.rsb_engine_set_occupancy(None, 50) == 1
