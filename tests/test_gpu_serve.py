"""Serving loop (rsb_server_*): every request's function equals its plain build, whatever
batch it was admitted into; admission respects the HBM budget; one bad request fails alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _string_keys(rng, n, lo=10, hi=50):
    lens = rng.integers(lo, hi + 1, n)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    offsets[1:] = np.cumsum(lens)
    data = rng.integers(0, 256, int(offsets[-1]), dtype=np.uint8)
    return data, offsets


def _plain(rsb, engine, req):
    kind, keys, b, leaf, rot = req
    if kind == "strings":
        return rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, rotate=rot, key_type="strings", engine=engine)
    return rsb.GPURecSplit(keys, bucket_size=b, leaf_size=leaf, rotate=rot, key_type="hash128", engine=engine)


def test_serve_mix_equals_plain(rsb, oracle_mod, engine):
    rng = np.random.default_rng(17)
    classes = [(100, 8), (1000, 12), (2000, 16)]
    reqs = []
    for i in range(36):
        b, leaf = classes[i % 3]
        n = int(np.exp(rng.uniform(np.log(100), np.log(30000 if leaf < 16 else 8000))))
        if i in (4, 9):
            n = i - 4  # empty and tiny requests
        if i % 4 == 3:
            reqs.append(("hash128", oracle_mod.keygen_hash128(1000 + i, n), b, leaf, True))
        else:
            reqs.append(("strings", _string_keys(rng, n), b, leaf, i % 7 != 0))
    with rsb.Server(hbm_budget=2 << 30, inflight=2) as srv:
        ids = []
        for kind, keys, b, leaf, rot in reqs:
            if kind == "strings":
                ids.append(srv.submit_strings(keys, b, leaf, rotate=rot))
            else:
                ids.append(srv.submit_hash128(keys, b, leaf, rotate=rot))
        results = [srv.wait(i) for i in ids]
    batched = 0
    for req, (f, info) in zip(reqs, results):
        assert info["submit_s"] <= info["admit_s"] <= info["done_s"]
        batched += info["batch_requests"] > 1
        assert f.serialize() == _plain(rsb, engine, req).serialize()
    assert batched > 0, "no request was batched with another"


def test_serve_matches_oracle_strings(rsb, oracle_mod):
    rng = np.random.default_rng(5)
    data, offsets = _string_keys(rng, 4000)
    with rsb.Server(hbm_budget=1 << 30, inflight=1) as srv:
        f, _ = srv.wait(srv.submit_strings((data, offsets), 100, 8))
    h = oracle_mod.hash_strings(data, offsets)
    ref = oracle_mod.build_mphf(h, 8, 100)
    assert f.serialize() == ref.bytes.tobytes()


def test_serve_budget_rejects_oversize_request(rsb, oracle_mod):
    # 64 MiB over 2 workers: each worker may hold ~32 MiB, so 1M keys (~70 MB) cannot fit.
    with rsb.Server(hbm_budget=64 << 20, inflight=2) as srv:
        big = srv.submit_hash128(oracle_mod.keygen_hash128(1, 1_000_000), 1000, 12)
        small = srv.submit_hash128(oracle_mod.keygen_hash128(2, 50_000), 1000, 12)
        with pytest.raises(rsb.RSBError) as e:
            srv.wait(big)
        assert e.value.name == "OOM"
        f, info = srv.wait(small)
        assert f.query(oracle_mod.keygen_hash128(2, 50_000)).max() == 49_999


def test_serve_budget_splits_batches(rsb, oracle_mod):
    # Budget for one worker fits about two of these requests at a time, never all ten.
    keys = [oracle_mod.keygen_hash128(300 + i, 100_000) for i in range(10)]
    with rsb.Server(hbm_budget=20 << 20, inflight=1) as srv:
        ids = [srv.submit_hash128(k, 1000, 12) for k in keys]
        out = [srv.wait(i) for i in ids]
    for k, (f, info) in zip(keys, out):
        assert info["batch_requests"] <= 2
        assert info["batch_keys"] <= 200_000
        q = f.query(k)
        assert np.array_equal(np.sort(q), np.arange(len(k), dtype=np.uint64))


def test_serve_duplicate_fails_alone(rsb, oracle_mod, engine):
    good = [oracle_mod.keygen_hash128(40 + i, 3000) for i in range(4)]
    bad = oracle_mod.keygen_hash128(99, 3000)
    bad[10] = bad[20]
    with rsb.Server(hbm_budget=1 << 30, inflight=1) as srv:
        # A large first request keeps the worker busy so that the next five share a batch.
        first = srv.submit_hash128(oracle_mod.keygen_hash128(7, 400_000), 100, 8)
        ids = [srv.submit_hash128(k, 100, 8) for k in good[:2]]
        bid = srv.submit_hash128(bad, 100, 8)
        ids += [srv.submit_hash128(k, 100, 8) for k in good[2:]]
        srv.wait(first)
        with pytest.raises(rsb.RSBError) as e:
            srv.wait(bid)
        assert e.value.name == "DUPLICATE_KEY"
        for k, i in zip(good, ids):
            f, _ = srv.wait(i)
            plain = rsb.GPURecSplit(k, bucket_size=100, leaf_size=8, engine=engine)
            assert f.serialize() == plain.serialize()


def test_serve_wait_timeout_and_unknown_id(rsb, oracle_mod):
    with rsb.Server(hbm_budget=1 << 30, inflight=1) as srv:
        rid = srv.submit_hash128(oracle_mod.keygen_hash128(3, 2_000_000), 2000, 16)
        try:
            srv.wait(rid, timeout_s=0.0)
        except rsb.RSBError as e:
            assert e.name == "TIMEOUT"
        f, _ = srv.wait(rid)
        assert f.get_bits() > 0
        with pytest.raises(rsb.RSBError) as e:
            srv.wait(rid)  # already collected
        assert e.value.name == "BAD_ARG"


def test_serve_batch_strings_entry(rsb, oracle_mod, engine):
    rng = np.random.default_rng(11)
    sizes = [0, 1, 500, 2500, 40]
    parts = [_string_keys(rng, n) for n in sizes]
    data = np.concatenate([p[0] for p in parts])
    offs = [np.uint64(0)]
    base = 0
    for d, o in parts:
        offs.extend((o[1:] + base).tolist())
        base += len(d)
    key_offsets = np.array(offs, dtype=np.uint64)
    set_offsets = np.zeros(len(sizes) + 1, dtype=np.uint64)
    set_offsets[1:] = np.cumsum(sizes)
    funcs, _ = rsb.build_batch((data, key_offsets), set_offsets, 100, 8, key_type="strings", engine=engine)
    for (d, o), f in zip(parts, funcs):
        plain = rsb.GPURecSplit((d, o), bucket_size=100, leaf_size=8, key_type="strings", engine=engine)
        assert f.serialize() == plain.serialize()


def test_serve_holds_its_budget(rsb, oracle_mod):
    import torch
    torch.cuda.init()
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    budget = 3 << 30
    with rsb.Server(hbm_budget=budget, inflight=3) as srv:
        free1, _ = torch.cuda.mem_get_info()
        rng = np.random.default_rng(8)
        ids = []
        for i in range(24):
            b, leaf = [(100, 8), (1000, 12), (2000, 16)][i % 3]
            n = int(rng.integers(1000, 400_000 if leaf < 16 else 100_000))
            ids.append(srv.submit_strings(_string_keys(rng, n), b, leaf))
        for i in ids:
            srv.wait(i)
        free2, _ = torch.cuda.mem_get_info()
    reserved = free0 - free1
    assert reserved <= budget + (256 << 20), reserved     # reservation ~ budget (+ streams, tables)
    assert free1 - free2 <= 64 << 20, free1 - free2        # serving allocates no more scratch


def test_engine_reserve_then_build(rsb, oracle_mod):
    eng = rsb.Engine(0)
    eng.reserve(200_000, 100, 0, 4)
    keys = oracle_mod.keygen_hash128(12, 150_000)
    f = rsb.GPURecSplit(keys, bucket_size=100, leaf_size=8, engine=eng)
    assert f.serialize() == oracle_mod.build_mphf(keys, 8, 100).bytes.tobytes()
    with pytest.raises(rsb.RSBError) as e:
        eng.reserve(10, 0)
    assert e.value.name == "BAD_ARG"
    eng.close()
