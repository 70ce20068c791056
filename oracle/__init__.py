"""CPU oracle for RecSplit construction — TEST INFRASTRUCTURE ONLY.

A scalar C++ restatement of ByteHamster/GpuRecSplit's SIMDRecSplit construction
(``oracle/recsplit_oracle.cpp``), loaded through ctypes. Only ``tests/``, ``bench.py``
(its ``cpu_baseline`` leg and ``--impl reference`` arm) and ``__graft_entry__.smoke()``
may import this module, and only as the checker or the timed CPU baseline; the
``gpurecsplit_b200`` product never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
# Same source with the seed searches in AVX-512 intrinsics (SIMDRecSplit's lane layout):
# the timed CPU baseline only. Loaded on request and only on CPUs that have the features.
_SIMD_LIB_PATH = os.path.join(_HERE, "_build", "libsimdrs.so")
_SIMD_FLAGS = ("avx512f", "avx512dq", "avx512bw", "avx512vl", "avx512_vpopcntdq")
_lib = None
_simd_lib = None

STATUS = {0: "OK", 1: "BAD_ARG", 2: "DUPLICATE_KEY", 3: "BUCKET_TOO_LARGE", 4: "FORMAT"}


# The reference's own SIMDRecSplit compiled from its sources (oracle/ref_harness.cpp with the
# stand-ins in oracle/_ref_shim/); built only where the reference tree is present, used
# prebuilt elsewhere.
_REF_LIB_PATH = os.path.join(_HERE, "_ref", "libref_simdrs.so")
_REF_CHECKED_LIB_PATH = os.path.join(_HERE, "_ref", "libref_simdrs_checked.so")
_REF_FLAGS = ("avx2", "bmi2", "avx512f", "avx512cd", "avx512dq", "avx512bw", "avx512vl", "avx512_vpopcntdq")
_ref_libs = {}


def reference_tree():
    """The GpuRecSplit source tree to compile oracle/_ref from, or None when absent."""
    root = os.environ.get("RSB_REFERENCE_ROOT", "/root/reference")
    return root if os.path.isfile(os.path.join(root, "include", "function", "SIMDRecSplit.hpp")) else None


def build() -> str:
    """Compiles the oracle libraries with the committed Makefile (no-op when up to date), and
    the reference's own SIMDRecSplit into oracle/_ref/ when the reference tree is present."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    ref = reference_tree()
    if ref is not None:
        subprocess.run(["make", "-s", "-j2", "-C", _HERE, "ref", f"REF={ref}"], check=True)
    return _LIB_PATH


def simd_supported() -> bool:
    """True when this CPU has the AVX-512 features libsimdrs.so is compiled for."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    return all(x in flags for x in _SIMD_FLAGS)
    except OSError:
        pass
    return False


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def simd_lib():
    """The AVX-512 build (raises if this CPU lacks the features)."""
    global _simd_lib
    if _simd_lib is None:
        if not simd_supported():
            raise RuntimeError("this CPU lacks AVX-512 F/DQ/BW/VL/VPOPCNTDQ")
        if not os.path.exists(_SIMD_LIB_PATH):
            build()
        _simd_lib = _configure(ctypes.CDLL(_SIMD_LIB_PATH))
    return _simd_lib


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = _configure(ctypes.CDLL(_LIB_PATH))
    return _lib


def _configure(L):
    u64p = ctypes.POINTER(ctypes.c_uint64)
    L.orc_memo.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    L.orc_build.restype = ctypes.c_void_p
    L.orc_build.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64,
                            ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    L.orc_build_buckets.restype = ctypes.c_void_p
    L.orc_build_buckets.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                    ctypes.POINTER(ctypes.c_int)]
    L.orc_result_len.restype = ctypes.c_uint64
    L.orc_result_len.argtypes = [ctypes.c_void_p, ctypes.c_int]
    L.orc_result_copy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    L.orc_free.argtypes = [ctypes.c_void_p]
    L.orc_query.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int, ctypes.c_void_p,
                            ctypes.c_uint64, ctypes.c_void_p]
    L.orc_get_bits.restype = ctypes.c_uint64
    L.orc_get_bits.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64]
    L.orc_keygen_hash128.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
    L.orc_keygen_u64.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_void_p]
    L.orc_hash_u64.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    L.orc_keygen_strings.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                     ctypes.c_void_p, ctypes.c_void_p]
    L.orc_hash_strings.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.c_void_p]
    L.orc_search_aggr.restype = ctypes.c_uint64
    L.orc_search_aggr.argtypes = [ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64]
    L.orc_remap16.restype = ctypes.c_uint32
    L.orc_remap16.argtypes = [ctypes.c_uint64, ctypes.c_uint32]
    return L


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleError(RuntimeError):
    def __init__(self, status: int):
        super().__init__(f"oracle status {status} ({STATUS.get(status, '?')})")
        self.status = status


def memo(leaf: int):
    out = np.zeros(3000, dtype=np.uint32)
    lo, up = ctypes.c_uint32(), ctypes.c_uint32()
    st = lib().orc_memo(leaf, _ptr(out), ctypes.byref(lo), ctypes.byref(up))
    if st:
        raise OracleError(st)
    return out, lo.value, up.value


class Build:
    """Result of one oracle build: serialized bytes, DFS seeds, node sizes, EF inputs."""

    def __init__(self, handle, L=None):
        L = L or lib()
        self.bytes = self._get(L, handle, 0, np.uint8)
        self.seeds = self._get(L, handle, 1, np.uint64)
        self.sizes = self._get(L, handle, 2, np.uint32)
        self.bucket_size_acc = self._get(L, handle, 3, np.uint64)
        self.bucket_pos_acc = self._get(L, handle, 4, np.uint64)
        self.evals_alg = int(self._get(L, handle, 5, np.uint64)[0])
        L.orc_free(handle)

    @staticmethod
    def _get(L, handle, which, dtype):
        n = L.orc_result_len(handle, which)
        a = np.zeros(n, dtype=dtype)
        if n:
            L.orc_result_copy(handle, which, _ptr(a))
        return a


def build_mphf(keys128: np.ndarray, leaf: int, bucket_size: int, rotate: bool = True, threads: int = 0,
               simd: bool = False) -> Build:
    """keys128: uint64 array of shape (n, 2) holding (first, second). ``simd`` selects the
    AVX-512 build of the searches (same output; the timed CPU baseline)."""
    keys128 = np.ascontiguousarray(keys128, dtype=np.uint64).reshape(-1, 2)
    threads = threads or os.cpu_count() or 1
    L = simd_lib() if simd else lib()
    st = ctypes.c_int(0)
    h = L.orc_build(_ptr(keys128), keys128.shape[0], leaf, bucket_size, int(rotate), threads, ctypes.byref(st))
    if not h:
        raise OracleError(st.value)
    return Build(h, L)


def bucket_seeds(keys128: np.ndarray, leaf: int, bucket_size: int, buckets, rotate: bool = True,
                 threads: int = 0) -> Build:
    """Seeds (DFS order) of the selected buckets only; nothing is encoded."""
    keys128 = np.ascontiguousarray(keys128, dtype=np.uint64).reshape(-1, 2)
    sel = np.ascontiguousarray(buckets, dtype=np.uint64)
    threads = threads or os.cpu_count() or 1
    st = ctypes.c_int(0)
    h = lib().orc_build_buckets(_ptr(keys128), keys128.shape[0], leaf, bucket_size, int(rotate), threads,
                                _ptr(sel), sel.size, ctypes.byref(st))
    if not h:
        raise OracleError(st.value)
    return Build(h)


def query(serialized: np.ndarray, keys128: np.ndarray, rotate: bool = True) -> np.ndarray:
    serialized = np.ascontiguousarray(serialized, dtype=np.uint8)
    keys128 = np.ascontiguousarray(keys128, dtype=np.uint64).reshape(-1, 2)
    out = np.zeros(keys128.shape[0], dtype=np.uint64)
    st = lib().orc_query(_ptr(serialized), serialized.size, int(rotate), _ptr(keys128), keys128.shape[0], _ptr(out))
    if st:
        raise OracleError(st)
    return out


def get_bits(serialized: np.ndarray, object_bytes: int = 0) -> int:
    serialized = np.ascontiguousarray(serialized, dtype=np.uint8)
    return int(lib().orc_get_bits(_ptr(serialized), serialized.size, object_bytes))


def keygen_hash128(seed: int, n: int) -> np.ndarray:
    out = np.zeros((n, 2), dtype=np.uint64)
    lib().orc_keygen_hash128(seed, n, _ptr(out))
    return out


def keygen_u64(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=np.uint64)
    lib().orc_keygen_u64(seed, n, _ptr(out))
    return out


def hash_u64(keys: np.ndarray) -> np.ndarray:
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    out = np.zeros((keys.size, 2), dtype=np.uint64)
    lib().orc_hash_u64(_ptr(keys), keys.size, _ptr(out))
    return out


def keygen_strings(seed: int, n: int, min_len: int = 10, max_len: int = 50):
    offsets = np.zeros(n + 1, dtype=np.uint64)
    lib().orc_keygen_strings(seed, n, min_len, max_len, _ptr(offsets), None)
    data = np.zeros(int(offsets[-1]), dtype=np.uint8)
    lib().orc_keygen_strings(seed, n, min_len, max_len, _ptr(offsets), _ptr(data))
    return data, offsets


def hash_strings(data: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    data = np.ascontiguousarray(data, dtype=np.uint8)
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    n = offsets.size - 1
    out = np.zeros((n, 2), dtype=np.uint64)
    lib().orc_hash_strings(_ptr(data), _ptr(offsets), n, _ptr(out))
    return out


def search_aggr(seconds: np.ndarray, split: int, seed: int, simd: bool = False) -> int:
    """Minimum seed (from `seed`) splitting the keys into parts of `split` keys (the last part
    the rest), by the scalar or the AVX-512 search loop."""
    k = np.ascontiguousarray(seconds, dtype=np.uint64)
    L = simd_lib() if simd else lib()
    return int(L.orc_search_aggr(_ptr(k), k.size, split, seed))


def remap16(x: int, n: int) -> int:
    return int(lib().orc_remap16(x, n))


# ---------------------------------------------------------------------------------------
# The reference's own SIMDRecSplit (oracle/_ref), compiled from its unmodified sources
# ---------------------------------------------------------------------------------------
def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def ref_available(checked: bool = False) -> bool:
    """True when oracle/_ref holds the reference build and this CPU can run it."""
    path = _REF_CHECKED_LIB_PATH if checked else _REF_LIB_PATH
    return os.path.exists(path) and all(x in _cpu_flags() for x in _REF_FLAGS)


def ref_lib(checked: bool = False):
    """The reference's SIMDRecSplit build (release, or with assertions when `checked`)."""
    if checked not in _ref_libs:
        path = _REF_CHECKED_LIB_PATH if checked else _REF_LIB_PATH
        if not os.path.exists(path):
            raise RuntimeError(f"{path} is missing: build it with oracle.build() where the reference tree is present")
        if not all(x in _cpu_flags() for x in _REF_FLAGS):
            raise RuntimeError("this CPU lacks the AVX-512 features the reference build needs")
        L = ctypes.CDLL(path)
        L.ref_build.restype = ctypes.c_void_p
        L.ref_build.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                                ctypes.c_int]
        L.ref_encode.restype = ctypes.c_void_p
        L.ref_encode.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32,
                                 ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                 ctypes.POINTER(ctypes.c_int)]
        L.ref_blob_len.restype = ctypes.c_uint64
        L.ref_blob_len.argtypes = [ctypes.c_void_p]
        L.ref_blob_copy.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        L.ref_blob_free.argtypes = [ctypes.c_void_p]
        L.ref_query.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p,
                                ctypes.c_uint64, ctypes.c_void_p]
        L.ref_get_bits.restype = ctypes.c_uint64
        L.ref_get_bits.argtypes = [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int]
        L.ref_object_size.restype = ctypes.c_uint64
        L.ref_object_size.argtypes = [ctypes.c_uint32, ctypes.c_int]
        _ref_libs[checked] = L
    return _ref_libs[checked]


def _ref_blob(L, h) -> np.ndarray:
    n = L.ref_blob_len(h)
    a = np.zeros(n, dtype=np.uint8)
    if n:
        L.ref_blob_copy(h, _ptr(a))
    L.ref_blob_free(h)
    return a


def ref_build(keys128: np.ndarray, leaf: int, bucket_size: int, rotate: bool = True, threads: int = 0,
              checked: bool = False) -> np.ndarray:
    """Serialized function built by the reference's SIMDRecSplit<leaf, MALLOC, rotate> from
    `keys128` (uint64 (n, 2): first, second) with `threads` threads."""
    keys128 = np.ascontiguousarray(keys128, dtype=np.uint64).reshape(-1, 2)
    threads = threads or os.cpu_count() or 1
    L = ref_lib(checked)
    h = L.ref_build(_ptr(keys128), keys128.shape[0], leaf, bucket_size, int(rotate), threads)
    if not h:
        raise RuntimeError("ref_build: bad arguments")
    return _ref_blob(L, h)


def ref_encode(bucket_keys: np.ndarray, bucket_size: int, leaf: int, seeds: np.ndarray, sizes: np.ndarray,
               rotate: bool = True, checked: bool = False) -> np.ndarray:
    """Serialized function made by the reference's RiceBitVector::Builder, DoubleEF and
    operator<< from given DFS seeds and node sizes; `bucket_keys` holds the key count of
    every bucket."""
    bk = np.ascontiguousarray(bucket_keys, dtype=np.uint64)
    sd = np.ascontiguousarray(seeds, dtype=np.uint64)
    sz = np.ascontiguousarray(sizes, dtype=np.uint32)
    L = ref_lib(checked)
    err = ctypes.c_int(0)
    h = L.ref_encode(_ptr(bk), bk.size, int(bk.sum()), bucket_size, leaf, int(rotate), _ptr(sd), _ptr(sz), sd.size,
                     ctypes.byref(err))
    if not h:
        raise RuntimeError(f"ref_encode failed ({err.value})")
    return _ref_blob(L, h)


def ref_query(serialized: np.ndarray, leaf: int, keys128: np.ndarray, rotate: bool = True) -> np.ndarray:
    """The reference's operator>> then operator()(hash128_t) for every key."""
    serialized = np.ascontiguousarray(serialized, dtype=np.uint8)
    keys128 = np.ascontiguousarray(keys128, dtype=np.uint64).reshape(-1, 2)
    out = np.zeros(keys128.shape[0], dtype=np.uint64)
    st = ref_lib().ref_query(_ptr(serialized), serialized.size, leaf, int(rotate), _ptr(keys128), keys128.shape[0],
                             _ptr(out))
    if st:
        raise RuntimeError(f"ref_query: cannot read the function (status {st})")
    return out


def ref_get_bits(serialized: np.ndarray, leaf: int, rotate: bool = True) -> int:
    serialized = np.ascontiguousarray(serialized, dtype=np.uint8)
    return int(ref_lib().ref_get_bits(_ptr(serialized), serialized.size, leaf, int(rotate)))


def ref_object_size(leaf: int, rotate: bool = True) -> int:
    """sizeof(SIMDRecSplit<leaf, MALLOC, rotate>) in the reference build."""
    return int(ref_lib().ref_object_size(leaf, int(rotate)))
