"""B200-native RecSplit construction engine (Python binding of librsb.so).

Mirrors the construction API of ByteHamster/GpuRecSplit
(``GPURecSplit<LEAF_SIZE, AT, USE_BIJECTIONS_ROTATE>``, include/function/GPURecSplit.cuh:409-505):

    f = GPURecSplit(keys, bucket_size=2000, leaf_size=16)   # keys: hash128 array, strings or bytes
    f(key)                                                   # operator()
    f.get_bits()                                             # getBits()
    blob = f.serialize(); g = GPURecSplit.deserialize(blob, leaf_size=16)   # operator<< / >>

All construction runs in CUDA kernels for sm_100a through the C ABI of ``include/rsb.h``.
There is no CPU fallback: without the built library or a B200 every call raises.
"""
from __future__ import annotations

import ctypes
import os
from typing import Iterable, Optional, Sequence, Union

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# RSB_LIBRARY selects another build of librsb.so (e.g. one compiled with different flags).
LIB_PATH = os.environ.get("RSB_LIBRARY") or os.path.join(_HERE, "_lib", "librsb.so")

RSB_ROTATE = 1
RSB_KEYS_ON_DEVICE = 2
RSB_DEVICE_ONLY = 4
RSB_KEEP_SEEDS = 8
RSB_VERIFY = 16

STATUS_NAMES = {
    0: "OK", 1: "BAD_ARG", 2: "CUDA", 3: "OOM", 4: "DUPLICATE_KEY", 5: "SEARCH_BUDGET",
    6: "BUCKET_TOO_LARGE", 7: "TIMEOUT", 8: "FORMAT", 9: "INTERNAL", 10: "NO_DEVICE",
}

_lib = None


class RSBError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        msg = lib().rsb_strerror(status).decode()
        super().__init__(f"{what}: rsb status {status} ({STATUS_NAMES.get(status, '?')}): {msg}")
        self.status = status
        self.name = STATUS_NAMES.get(status, "?")


class Stats(ctypes.Structure):
    _fields_ = [
        ("keys", ctypes.c_uint64), ("buckets", ctypes.c_uint64), ("nodes", ctypes.c_uint64),
        ("nodes_per_stage", ctypes.c_uint64 * 21), ("evals_alg", ctypes.c_uint64),
        ("descriptor_bits", ctypes.c_uint64), ("ms_total", ctypes.c_double), ("ms_partition", ctypes.c_double),
        ("ms_search", ctypes.c_double * 21), ("ms_encode", ctypes.c_double),
        ("evals_stage", ctypes.c_uint64 * 21), ("kernel_launches", ctypes.c_uint64),
        ("windows_stage", ctypes.c_uint64 * 21), ("window_candidates", ctypes.c_uint64 * 21),
    ]

    def as_dict(self) -> dict:
        return {
            "keys": self.keys, "buckets": self.buckets, "nodes": self.nodes,
            "nodes_per_stage": list(self.nodes_per_stage), "evals_alg": self.evals_alg,
            "descriptor_bits": self.descriptor_bits, "ms_total": self.ms_total,
            "ms_partition": self.ms_partition, "ms_search": list(self.ms_search), "ms_encode": self.ms_encode,
            "evals_stage": list(self.evals_stage), "kernel_launches": self.kernel_launches,
            "windows_stage": list(self.windows_stage), "window_candidates": list(self.window_candidates),
        }


class RequestInfo(ctypes.Structure):
    _fields_ = [("submit_s", ctypes.c_double), ("admit_s", ctypes.c_double), ("done_s", ctypes.c_double),
                ("batch_requests", ctypes.c_uint32), ("batch_keys", ctypes.c_uint64)]


def build_library() -> str:
    from . import build as _build
    return _build.build()


def lib():
    """Loads librsb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m gpurecsplit_b200.build` first")
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, u32, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int
        pp = ctypes.POINTER(ctypes.c_void_p)
        sig = {
            "rsb_engine_create": ([i32, vp, pp], i32),
            "rsb_engine_destroy": ([vp], i32),
            "rsb_engine_set_budget": ([vp, u32, u64], i32),
            "rsb_engine_reserve": ([vp, u64, u64, u64, u32], i32),
            "rsb_engine_set_occupancy": ([vp, u32], i32),
            "rsb_build_hash128": ([vp, vp, u64, u64, u32, u32, pp], i32),
            "rsb_build_strings": ([vp, vp, vp, u64, u64, u32, u32, pp], i32),
            "rsb_build_u64": ([vp, vp, u64, u64, u32, u32, pp], i32),
            "rsb_query_hash128": ([vp, vp, u64, vp], i32),
            "rsb_query_strings": ([vp, vp, vp, u64, vp], i32),
            "rsb_query_device": ([vp, vp, vp, u64, vp], i32),
            "rsb_get_bits": ([vp, ctypes.POINTER(u64)], i32),
            "rsb_serialize": ([vp, vp, ctypes.POINTER(ctypes.c_size_t)], i32),
            "rsb_deserialize": ([vp, ctypes.c_size_t, u32, u32, pp], i32),
            "rsb_seeds": ([vp, vp, vp, ctypes.POINTER(ctypes.c_size_t)], i32),
            "rsb_get_stats": ([vp, ctypes.POINTER(Stats)], i32),
            "rsb_free": ([vp], i32),
            "rsb_hash_strings": ([vp, vp, vp, u64, u32, vp], i32),
            "rsb_hash_u64": ([vp, vp, u64, u32, vp], i32),
            "rsb_strerror": ([i32], ctypes.c_char_p),
            "rsb_version": ([], ctypes.c_char_p),
            "rsb_golomb_memo": ([u32, vp], i32),
            "rsb_probe_eval_rate": ([vp, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)], i32),
            "rsb_hash_strings_static": ([vp, vp, u64, vp, vp], i32),
            "rsb_build_batch_hash128": ([vp, vp, vp, u32, u64, u32, u32, vp, ctypes.POINTER(Stats)], i32),
            "rsb_build_batch_u64": ([vp, vp, vp, u32, u64, u32, u32, vp, ctypes.POINTER(Stats)], i32),
            "rsb_build_batch_strings": ([vp, vp, vp, vp, u32, u64, u32, u32, vp, ctypes.POINTER(Stats)], i32),
            "rsb_build_part_hash128": ([vp, vp, u64, u64, u64, u64, u64, u32, u32, pp], i32),
            "rsb_part_export": ([vp, vp, ctypes.POINTER(ctypes.c_size_t)], i32),
            "rsb_engine_set_schedule": ([vp, u32, u32, u32, u32, u32], i32),
            "rsb_engine_set_pipeline": ([vp, u32], i32),
            "rsb_engine_set_watchdog": ([vp, ctypes.c_double], i32),
            "rsb_engine_get_schedule": ([vp, u32, u32, u32, ctypes.POINTER(u32), ctypes.POINTER(u32)], i32),
            "rsb_merge_parts": ([vp, vp, vp, u32, u32, u32, pp], i32),
            "rsb_server_create": ([i32, u64, u32, u64, pp], i32),
            "rsb_server_submit_strings": ([vp, vp, vp, u64, u64, u32, u32, ctypes.POINTER(u64)], i32),
            "rsb_server_submit_hash128": ([vp, vp, u64, u64, u32, u32, ctypes.POINTER(u64)], i32),
            "rsb_server_wait": ([vp, u64, ctypes.c_double, pp, ctypes.POINTER(RequestInfo)], i32),
            "rsb_server_destroy": ([vp], i32),
        }
        for name, (args, res) in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def _check(status: int, what: str) -> None:
    if status != 0:
        raise RSBError(status, what)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def golomb_memo(leaf_size: int) -> np.ndarray:
    """The engine's Golomb-Rice table (AbstractParallelRecSplit.hpp:191-227) for one leaf size."""
    out = np.zeros(3000, dtype=np.uint32)
    _check(lib().rsb_golomb_memo(leaf_size, _ptr(out)), "rsb_golomb_memo")
    return out


class Engine:
    """A device context (stream + cached scratch); one per GPU and host thread."""

    def __init__(self, device: int = 0, stream: Optional[int] = None):
        h = ctypes.c_void_p()
        _check(lib().rsb_engine_create(device, ctypes.c_void_p(stream or 0), ctypes.byref(h)), "rsb_engine_create")
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def set_budget(self, shift: int, min_candidates: int = 1 << 16) -> None:
        _check(lib().rsb_engine_set_budget(self._h, shift, min_candidates), "rsb_engine_set_budget")

    def reserve(self, keys: int, bucket_size: int, string_bytes: int = 0, sets: int = 1) -> None:
        """Pre-sizes the device scratch for builds of up to `keys` keys (rsb_engine_reserve)."""
        _check(lib().rsb_engine_reserve(self._h, keys, bucket_size, string_bytes, sets), "rsb_engine_reserve")

    def set_occupancy(self, percent: int) -> None:
        """Runs the persistent search kernels at `percent` of full occupancy (rsb_engine_set_occupancy)."""
        _check(lib().rsb_engine_set_occupancy(self._h, percent), "rsb_engine_set_occupancy")

    def set_pipeline(self, on: bool) -> None:
        """Runs the aggregation and leaf searches of every build as one persistent launch with
        device work queues (rsb_engine_set_pipeline); the functions are the same."""
        _check(lib().rsb_engine_set_pipeline(self._h, 1 if on else 0), "rsb_engine_set_pipeline")

    def set_watchdog(self, seconds: float) -> None:
        """Upper bound on one pipeline-mode launch (rsb_engine_set_watchdog); 0: none."""
        _check(lib().rsb_engine_set_watchdog(self._h, float(seconds)), "rsb_engine_set_watchdog")

    def set_schedule(self, leaf_size: int, stage: int, size_class: int, seeds_per_lane: int,
                     occupancy_pct: int = 100) -> None:
        """Schedule of one search stage (rsb_engine_set_schedule): 17/18 aggregation levels
        (4, 8, 12 or 16 seeds per lane), 19 rotation leaves (4, 8 or 12 bases per lane); size class
        0 below 2^20 keys, 1 from 2^20, 2 from 2^24. seeds_per_lane 0 restores the built-in schedule."""
        _check(lib().rsb_engine_set_schedule(self._h, leaf_size, stage, size_class, seeds_per_lane, occupancy_pct),
               "rsb_engine_set_schedule")

    def schedule(self, leaf_size: int, stage: int, size_class: int):
        """(seeds per lane, occupancy %) this engine uses for the stage (rsb_engine_get_schedule)."""
        s, p = ctypes.c_uint32(), ctypes.c_uint32()
        _check(lib().rsb_engine_get_schedule(self._h, leaf_size, stage, size_class, ctypes.byref(s), ctypes.byref(p)),
               "rsb_engine_get_schedule")
        return s.value, p.value

    def probe_eval_rate(self):
        """(evaluations per second, ms) of the synthetic remixAndRemap32 ceiling kernel."""
        r, ms = ctypes.c_double(), ctypes.c_double()
        _check(lib().rsb_probe_eval_rate(self._h, ctypes.byref(r), ctypes.byref(ms)), "rsb_probe_eval_rate")
        return r.value, ms.value

    def close(self) -> None:
        if self._h:
            lib().rsb_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_engines: dict = {}


def default_engine(device: int = 0) -> Engine:
    e = _default_engines.get(device)
    if e is None:
        e = Engine(device)
        _default_engines[device] = e
    return e


def _strings_to_arrays(keys: Sequence[Union[str, bytes]]):
    bs = [k.encode() if isinstance(k, str) else bytes(k) for k in keys]
    offsets = np.zeros(len(bs) + 1, dtype=np.uint64)
    if bs:
        offsets[1:] = np.cumsum([len(b) for b in bs], dtype=np.uint64)
    data = np.frombuffer(b"".join(bs), dtype=np.uint8) if bs else np.zeros(0, dtype=np.uint8)
    return np.ascontiguousarray(data), offsets


class GPURecSplit:
    """Minimal perfect hash function built on the GPU (drop-in for the reference class).

    ``keys`` may be a uint64 array of shape (n, 2) holding hash128 (first, second) pairs,
    a sequence of str/bytes (hashed with SpookyHash V2 like the reference's string
    constructor), or — with ``key_type="u64"`` — a uint64 array of 64-bit keys.
    """

    def __init__(self, keys=None, bucket_size: int = 100, leaf_size: int = 8, rotate: bool = True,
                 engine: Optional[Engine] = None, key_type: Optional[str] = None, keep_seeds: bool = False,
                 device_only: bool = False, verify: bool = False, _handle=None):
        self.leaf_size = leaf_size
        self.bucket_size = bucket_size
        self.rotate = rotate
        self._h = _handle
        if _handle is not None:
            return
        eng = engine or default_engine()
        flags = (RSB_ROTATE if rotate else 0) | (RSB_KEEP_SEEDS if keep_seeds else 0) | \
            (RSB_DEVICE_ONLY if device_only else 0) | (RSB_VERIFY if verify else 0)
        h = ctypes.c_void_p()
        L = lib()
        if key_type is None:
            if isinstance(keys, np.ndarray):
                key_type = "hash128" if keys.ndim == 2 else "u64"
            else:
                key_type = "strings"
        if key_type == "hash128":
            k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1, 2)
            st = L.rsb_build_hash128(eng.handle, _ptr(k), k.shape[0], bucket_size, leaf_size, flags, ctypes.byref(h))
        elif key_type == "u64":
            k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1)
            st = L.rsb_build_u64(eng.handle, _ptr(k), k.size, bucket_size, leaf_size, flags, ctypes.byref(h))
        elif key_type == "strings":
            if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], np.ndarray):
                data, offsets = keys
            else:
                data, offsets = _strings_to_arrays(keys)
            data = np.ascontiguousarray(data, dtype=np.uint8)
            offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
            st = L.rsb_build_strings(eng.handle, _ptr(data), _ptr(offsets), offsets.size - 1, bucket_size, leaf_size,
                                     flags, ctypes.byref(h))
        else:
            raise ValueError(f"unknown key_type {key_type!r}")
        _check(st, "build")
        self._h = h

    # ---- device-resident construction (torch CUDA tensors or raw device pointers) ----
    @classmethod
    def from_device(cls, keys_ptr: int, n: int, bucket_size: int, leaf_size: int, rotate: bool = True,
                    key_type: str = "hash128", engine: Optional[Engine] = None, device_only: bool = True,
                    keep_seeds: bool = False) -> "GPURecSplit":
        eng = engine or default_engine()
        flags = RSB_KEYS_ON_DEVICE | (RSB_ROTATE if rotate else 0) | (RSB_DEVICE_ONLY if device_only else 0) | \
            (RSB_KEEP_SEEDS if keep_seeds else 0)
        h = ctypes.c_void_p()
        L = lib()
        if key_type == "hash128":
            st = L.rsb_build_hash128(eng.handle, ctypes.c_void_p(keys_ptr), n, bucket_size, leaf_size, flags, ctypes.byref(h))
        elif key_type == "u64":
            st = L.rsb_build_u64(eng.handle, ctypes.c_void_p(keys_ptr), n, bucket_size, leaf_size, flags, ctypes.byref(h))
        else:
            raise ValueError(key_type)
        _check(st, "build (device keys)")
        return cls(bucket_size=bucket_size, leaf_size=leaf_size, rotate=rotate, _handle=h)

    # ---- queries ----
    def __call__(self, key) -> int:
        if isinstance(key, (str, bytes)):
            return int(self.query_strings([key])[0])
        k = np.asarray(key, dtype=np.uint64).reshape(1, 2)
        return int(self.query(k)[0])

    def query(self, keys128: np.ndarray) -> np.ndarray:
        k = np.ascontiguousarray(keys128, dtype=np.uint64).reshape(-1, 2)
        out = np.zeros(k.shape[0], dtype=np.uint64)
        _check(lib().rsb_query_hash128(self._h, _ptr(k), k.shape[0], _ptr(out)), "query")
        return out

    def query_strings(self, keys) -> np.ndarray:
        if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], np.ndarray):
            data, offsets = keys
        else:
            data, offsets = _strings_to_arrays(keys)
        data = np.ascontiguousarray(data, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        out = np.zeros(offsets.size - 1, dtype=np.uint64)
        _check(lib().rsb_query_strings(self._h, _ptr(data), _ptr(offsets), offsets.size - 1, _ptr(out)), "query_strings")
        return out

    def query_device(self, keys_ptr: int, n: int, out_ptr: int, engine: Optional[Engine] = None) -> None:
        eng = engine or default_engine()
        _check(lib().rsb_query_device(eng.handle, self._h, ctypes.c_void_p(keys_ptr), n, ctypes.c_void_p(out_ptr)),
               "query_device")

    # ---- accessors ----
    def get_bits(self, object_bytes: int = 0) -> int:
        b = ctypes.c_uint64()
        _check(lib().rsb_get_bits(self._h, ctypes.byref(b)), "get_bits")
        return b.value + 8 * object_bytes

    def serialize(self) -> bytes:
        n = ctypes.c_size_t(0)
        _check(lib().rsb_serialize(self._h, None, ctypes.byref(n)), "serialize")
        buf = np.zeros(n.value, dtype=np.uint8)
        _check(lib().rsb_serialize(self._h, _ptr(buf), ctypes.byref(n)), "serialize")
        return buf[: n.value].tobytes()

    @classmethod
    def deserialize(cls, blob: bytes, leaf_size: int, rotate: bool = True) -> "GPURecSplit":
        b = np.frombuffer(blob, dtype=np.uint8).copy()
        h = ctypes.c_void_p()
        _check(lib().rsb_deserialize(_ptr(b), b.size, leaf_size, RSB_ROTATE if rotate else 0, ctypes.byref(h)),
               "deserialize")
        return cls(leaf_size=leaf_size, rotate=rotate, _handle=h)

    def seeds(self):
        n = ctypes.c_size_t(0)
        _check(lib().rsb_seeds(self._h, None, None, ctypes.byref(n)), "seeds")
        s = np.zeros(n.value, dtype=np.uint64)
        z = np.zeros(n.value, dtype=np.uint32)
        if n.value:
            _check(lib().rsb_seeds(self._h, _ptr(s), _ptr(z), ctypes.byref(n)), "seeds")
        return s, z

    def stats(self) -> dict:
        s = Stats()
        _check(lib().rsb_get_stats(self._h, ctypes.byref(s)), "stats")
        return s.as_dict()

    def close(self) -> None:
        if self._h:
            lib().rsb_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_part(keys, nbuckets_total: int, bucket_lo: int, bucket_hi: int, bucket_size: int, leaf_size: int,
               rotate: bool = True, engine: Optional[Engine] = None, n: Optional[int] = None) -> bytes:
    """Builds the part of an ``nbuckets_total``-bucket function over buckets [bucket_lo,
    bucket_hi) (rsb_build_part_hash128) and returns it exported (rsb_part_export).

    ``keys`` are the (n, 2) uint64 hash128 keys of exactly those buckets, as a host array or
    (with ``n``) a device pointer.
    """
    eng = engine or default_engine()
    L = lib()
    flags = RSB_ROTATE if rotate else 0
    if isinstance(keys, np.ndarray):
        k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1, 2)
        ptr, count = _ptr(k), k.shape[0]
    else:
        ptr, count = ctypes.c_void_p(int(keys)), int(n)
        flags |= RSB_KEYS_ON_DEVICE
    h = ctypes.c_void_p()
    _check(L.rsb_build_part_hash128(eng.handle, ptr, count, nbuckets_total, bucket_lo, bucket_hi, bucket_size,
                                    leaf_size, flags, ctypes.byref(h)), "build_part")
    try:
        size = ctypes.c_size_t(0)
        _check(L.rsb_part_export(h, None, ctypes.byref(size)), "part_export")
        buf = ctypes.create_string_buffer(size.value)
        _check(L.rsb_part_export(h, buf, ctypes.byref(size)), "part_export")
        return buf.raw[:size.value]
    finally:
        L.rsb_free(h)


def merge_parts(parts, leaf_size: int, rotate: bool = True, engine: Optional[Engine] = None) -> "GPURecSplit":
    """Merges exported parts that tile all buckets of one function, in bucket order
    (rsb_merge_parts); the result equals the plain build of all their keys."""
    eng = engine or default_engine()
    parts = [bytes(p) for p in parts]
    bufs = [ctypes.create_string_buffer(p, len(p)) for p in parts]
    ptrs = (ctypes.c_void_p * len(parts))(*[ctypes.cast(b, ctypes.c_void_p) for b in bufs])
    lens = (ctypes.c_size_t * len(parts))(*[len(p) for p in parts])
    h = ctypes.c_void_p()
    _check(lib().rsb_merge_parts(eng.handle, ptrs, lens, len(parts), leaf_size, RSB_ROTATE if rotate else 0,
                                 ctypes.byref(h)), "merge_parts")
    bucket_size = int(np.frombuffer(parts[0][64:72], dtype=np.uint64)[0])  # header word 8
    return GPURecSplit(bucket_size=bucket_size, leaf_size=leaf_size, rotate=rotate, _handle=h)


def build_batch(keys: np.ndarray, set_offsets, bucket_size: int, leaf_size: int, rotate: bool = True,
                key_type: Optional[str] = None, engine: Optional[Engine] = None, keys_on_device: bool = False,
                n_keys: Optional[int] = None):
    """Builds one function per key set in a single device pipeline (rsb_build_batch_*).

    Set s is keys[set_offsets[s]:set_offsets[s+1]]. ``keys`` is a (n, 2) uint64 hash128 array,
    (``key_type="u64"``) a uint64 array, (``key_type="strings"``) a (bytes, offsets) pair of
    uint8/uint64 arrays or a sequence of str/bytes, or with ``keys_on_device`` a device
    pointer (int). Returns (list of GPURecSplit, stats dict); each function equals the plain
    build of its set.
    """
    eng = engine or default_engine()
    offsets = np.ascontiguousarray(set_offsets, dtype=np.uint64)
    nsets = offsets.size - 1
    outs = (ctypes.c_void_p * max(nsets, 1))()
    stats = Stats()
    flags = (RSB_ROTATE if rotate else 0) | (RSB_KEYS_ON_DEVICE if keys_on_device else 0)
    L = lib()
    if key_type == "strings":
        if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], np.ndarray):
            data, key_offsets = keys
        else:
            data, key_offsets = _strings_to_arrays(keys)
        data = np.ascontiguousarray(data, dtype=np.uint8)
        key_offsets = np.ascontiguousarray(key_offsets, dtype=np.uint64)
        st = L.rsb_build_batch_strings(eng.handle, _ptr(data), _ptr(key_offsets), _ptr(offsets), nsets, bucket_size,
                                       leaf_size, flags & RSB_ROTATE, outs, ctypes.byref(stats))
        _check(st, "build_batch")
        funcs = [GPURecSplit(bucket_size=bucket_size, leaf_size=leaf_size, rotate=rotate,
                             _handle=ctypes.c_void_p(outs[i])) for i in range(nsets)]
        return funcs, stats.as_dict()
    if keys_on_device:
        kp = ctypes.c_void_p(keys)
        if key_type is None:
            key_type = "hash128"
    else:
        if key_type is None:
            key_type = "hash128" if keys.ndim == 2 else "u64"
        keys = np.ascontiguousarray(keys, dtype=np.uint64)
        kp = _ptr(keys)
    if key_type == "hash128":
        st = L.rsb_build_batch_hash128(eng.handle, kp, _ptr(offsets), nsets, bucket_size, leaf_size, flags, outs,
                                       ctypes.byref(stats))
    elif key_type == "u64":
        st = L.rsb_build_batch_u64(eng.handle, kp, _ptr(offsets), nsets, bucket_size, leaf_size, flags, outs,
                                   ctypes.byref(stats))
    else:
        raise ValueError(key_type)
    _check(st, "build_batch")
    funcs = [GPURecSplit(bucket_size=bucket_size, leaf_size=leaf_size, rotate=rotate, _handle=ctypes.c_void_p(outs[i]))
             for i in range(nsets)]
    return funcs, stats.as_dict()


class Server:
    """Continuous batching of build requests (rsb_server_*).

    ``inflight`` workers, each with its own engine, take the oldest queued request plus
    every queued request of the same (leaf size, bucket size, rotate, key kind) class while
    the batch's estimated device working set fits ``hbm_budget / inflight`` bytes, and build
    them as one batched pipeline. ``submit_*`` copies the keys and returns an id at once;
    ``wait(id)`` returns (GPURecSplit, info dict) with the request's timestamps.
    """

    def __init__(self, hbm_budget: int, inflight: int = 2, max_batch_keys: int = 0, device: int = 0):
        h = ctypes.c_void_p()
        _check(lib().rsb_server_create(device, hbm_budget, inflight, max_batch_keys, ctypes.byref(h)),
               "rsb_server_create")
        self._h = h
        self._params = {}

    def submit_strings(self, keys, bucket_size: int, leaf_size: int, rotate: bool = True) -> int:
        if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], np.ndarray):
            data, offsets = keys
        else:
            data, offsets = _strings_to_arrays(keys)
        data = np.ascontiguousarray(data, dtype=np.uint8)
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        rid = ctypes.c_uint64()
        _check(lib().rsb_server_submit_strings(self._h, _ptr(data), _ptr(offsets), offsets.size - 1, bucket_size,
                                               leaf_size, RSB_ROTATE if rotate else 0, ctypes.byref(rid)),
               "rsb_server_submit_strings")
        self._params[rid.value] = (bucket_size, leaf_size, rotate)
        return rid.value

    def submit_hash128(self, keys: np.ndarray, bucket_size: int, leaf_size: int, rotate: bool = True) -> int:
        k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1, 2)
        rid = ctypes.c_uint64()
        _check(lib().rsb_server_submit_hash128(self._h, _ptr(k), k.shape[0], bucket_size, leaf_size,
                                               RSB_ROTATE if rotate else 0, ctypes.byref(rid)),
               "rsb_server_submit_hash128")
        self._params[rid.value] = (bucket_size, leaf_size, rotate)
        return rid.value

    def wait(self, rid: int, timeout_s: float = -1.0):
        out = ctypes.c_void_p()
        info = RequestInfo()
        st = lib().rsb_server_wait(self._h, rid, timeout_s, ctypes.byref(out), ctypes.byref(info))
        if st == 7:  # still running: the request stays queued
            raise RSBError(st, "rsb_server_wait")
        b, leaf, rot = self._params.pop(rid, (0, 0, True))
        _check(st, "rsb_server_wait")
        f = GPURecSplit(bucket_size=b, leaf_size=leaf, rotate=rot, _handle=out)
        return f, {"submit_s": info.submit_s, "admit_s": info.admit_s, "done_s": info.done_s,
                   "batch_requests": info.batch_requests, "batch_keys": info.batch_keys}

    def close(self) -> None:
        if self._h:
            lib().rsb_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def hash_strings(keys, engine: Optional[Engine] = None) -> np.ndarray:
    """Device SpookyHash V2 of string keys -> (n, 2) uint64 (first, second)."""
    eng = engine or default_engine()
    if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], np.ndarray):
        data, offsets = keys
    else:
        data, offsets = _strings_to_arrays(keys)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    n = offsets.size - 1
    out = np.zeros((n, 2), dtype=np.uint64)
    _check(lib().rsb_hash_strings(eng.handle, _ptr(data), _ptr(offsets), n, 0, _ptr(out)), "hash_strings")
    return out


def hash_strings_static(keys, stream: Optional[int] = None) -> np.ndarray:
    """Device SpookyHash V2 of string keys without any device allocation (rsb_hash_strings_static).

    For callers that cannot allocate device memory; at most 32,768 keys and 1 MiB of key
    bytes per call. Runs on the current CUDA device.
    """
    if isinstance(keys, tuple) and len(keys) == 2 and isinstance(keys[0], np.ndarray):
        data, offsets = keys
    else:
        data, offsets = _strings_to_arrays(keys)
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    n = offsets.size - 1
    out = np.zeros((n, 2), dtype=np.uint64)
    _check(lib().rsb_hash_strings_static(_ptr(data), _ptr(offsets), n, _ptr(out), ctypes.c_void_p(stream or 0)),
           "hash_strings_static")
    return out


def hash_u64(keys: np.ndarray, engine: Optional[Engine] = None) -> np.ndarray:
    """Device 64->128-bit key mixer -> (n, 2) uint64 (first, second)."""
    eng = engine or default_engine()
    k = np.ascontiguousarray(keys, dtype=np.uint64).reshape(-1)
    out = np.zeros((k.size, 2), dtype=np.uint64)
    _check(lib().rsb_hash_u64(eng.handle, _ptr(k), k.size, 0, _ptr(out)), "hash_u64")
    return out


__all__ = ["GPURecSplit", "Engine", "Server", "build_batch", "build_part", "merge_parts", "RSBError", "lib", "build_library", "golomb_memo", "hash_strings", "hash_u64",
           "default_engine", "LIB_PATH"]
