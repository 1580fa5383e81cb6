"""ctypes access to the oracle (oracle/build/liborc.so) and, where it was built,
to the reference's own host code (oracle/_ref/libphobic_ref.so).

Test infrastructure only: the oracle is the checker for the CUDA path.  It is
loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

ORACLE = Path(__file__).resolve().parent
ORC_LIB = ORACLE / "build" / "liborc.so"
REF_LIB = ORACLE / "_ref" / "libphobic_ref.so"
P = C.c_void_p

_orc = None
_ref = None


class Stats(C.Structure):
    _fields_ = [
        ("hash_evals", C.c_uint64),
        ("probe_words", C.c_uint64),
        ("k_retries", C.c_uint64),
        ("max_bucket", C.c_uint32),
        ("max_partition", C.c_uint32),
        ("max_k", C.c_uint32),
        ("err_partition", C.c_uint32),
        ("pad", C.c_uint32),
        ("probe_keys", C.c_uint64),
    ]


class U128(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_uint64)]


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORC_LIB.exists():
            subprocess.run(["make", "-C", str(ORACLE), "oracle"], check=True, capture_output=True)
        lib = C.CDLL(str(ORC_LIB))
        lib.orc_xxh3_128.argtypes = [C.c_char_p, C.c_size_t, C.c_uint64, C.POINTER(U128)]
        lib.orc_xxh3_128.restype = C.c_int
        lib.orc_hash_u64.argtypes = [P, C.c_uint64, P, C.c_int]
        lib.orc_hash_pairs.argtypes = [P, C.c_uint64, P, C.c_int]
        lib.orc_hash_keys16.argtypes = [P, C.c_uint64, P, C.c_int]
        lib.orc_hash_bytes.argtypes = [P, P, C.c_uint64, P, C.c_int]
        lib.orc_buckets_per_partition.argtypes = [C.c_double, C.c_uint32, C.c_int]
        lib.orc_buckets_per_partition.restype = C.c_uint32
        lib.orc_fulcrums.argtypes = [C.c_int, C.c_double, C.c_uint32, C.c_uint32, P]
        lib.orc_max_partition_size.argtypes = [C.c_uint32]
        lib.orc_max_partition_size.restype = C.c_uint32
        lib.orc_build.argtypes = [P, C.c_uint64, C.c_uint32, C.c_uint32, P, P, P, P, P, P, P, C.c_uint32, C.c_int,
                                  C.c_int, C.POINTER(Stats)]
        lib.orc_build.restype = C.c_int
        lib.orc_query.argtypes = [P, C.c_uint64, C.c_uint32, C.c_uint32, P, P, P, P, C.c_int]
        lib.orc_is_bijection.argtypes = [P, C.c_uint64]
        lib.orc_is_bijection.restype = C.c_int
        lib.orc_splitmix64.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, P, C.c_int]
        lib.orc_pilot_hash.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32]
        lib.orc_pilot_hash.restype = C.c_uint32
        _orc = lib
    return _orc


def ref_available() -> bool:
    return REF_LIB.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        lib = C.CDLL(str(REF_LIB))
        lib.ref_hash_u64.argtypes = [P, C.c_uint64, P]
        lib.ref_hash_pairs.argtypes = [P, C.c_uint64, P]
        lib.ref_hash_keys16.argtypes = [P, C.c_uint64, P]
        lib.ref_hash_strings.argtypes = [P, P, C.c_uint64, P]
        lib.ref_config.argtypes = [C.c_double, C.c_uint32, C.c_int, C.c_int, P, P]
        lib.ref_config.restype = C.c_uint32
        lib.ref_encode.argtypes = [C.c_int, C.c_int, P, P, C.c_uint32, C.c_double, C.c_uint32, C.c_float, P,
                                   C.c_size_t, C.POINTER(C.c_double)]
        lib.ref_encode.restype = C.c_size_t
        lib.ref_query_u64.argtypes = [P, P, C.c_uint32, C.c_double, C.c_uint32, P, C.c_uint64, P]
        _ref = lib
    return _ref


# ------------------------------------------------------------------ wrappers

def xxh3_128(b: bytes) -> int:
    o = U128()
    assert orc().orc_xxh3_128(b, len(b), 0, C.byref(o)) == 0
    return (o.hi << 64) | o.lo


def splitmix64(seed: int, n: int, start: int = 0, threads: int = 0) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    orc().orc_splitmix64(seed, start, n, out.ctypes.data, threads)
    return out


def hash_keys(keys, kind: str = "u64", threads: int = 0) -> np.ndarray:
    """4-word Keys (n, 4) uint32 for u64 / pairs / keys16 / strings (bytes, offsets)."""
    if kind == "strings":
        data, offs = keys
        n = len(offs) - 1
        out = np.zeros((n, 4), np.uint32)
        data = np.ascontiguousarray(data, np.uint8)
        orc().orc_hash_bytes(data.ctypes.data if data.size else None, offs.ctypes.data, n, out.ctypes.data, threads)
        return out
    a = np.ascontiguousarray(keys)
    n = a.shape[0]
    out = np.zeros((n, 4), np.uint32)
    fn = {"u64": orc().orc_hash_u64, "pairs": orc().orc_hash_pairs, "keys16": orc().orc_hash_keys16}[kind]
    fn(a.ctypes.data if n else None, n, out.ctypes.data, threads)
    return out


def config(lam: float, P_: int, bucketer: int = 0, use_round: bool = False):
    B = orc().orc_buckets_per_partition(lam, P_, int(use_round))
    f = np.zeros(2048, np.uint32)
    orc().orc_fulcrums(bucketer, lam, P_, B, f.ctypes.data)
    return B, f


def build(keys4: np.ndarray, P_: int, B: int, fulcs: np.ndarray, intermediates: bool = False, max_k: int = 0,
          naive: bool = False, threads: int = 0):
    """Oracle build: returns dict with status, pilots, offsets (+ intermediates) and stats."""
    keys4 = np.ascontiguousarray(keys4, np.uint32)
    n = keys4.shape[0]
    parts = (n + P_ - 1) // P_
    pil = np.zeros(max(B * parts, 1), np.uint32)
    off = np.zeros(parts + 1, np.uint32)
    inter = {}
    ptrs = [None] * 4
    if intermediates:
        inter = {
            "bucket_sizes": np.zeros(max(parts * B, 1), np.uint32),
            "histo": np.zeros(max(parts * 256, 1), np.uint32),
            "perm": np.zeros(max(parts * B, 1), np.uint32),
            "sorted_lowers": np.zeros(max(2 * n, 1), np.uint32),
        }
        ptrs = [inter[k].ctypes.data for k in ("bucket_sizes", "histo", "perm", "sorted_lowers")]
    st = Stats()
    rc = orc().orc_build(keys4.ctypes.data if n else None, n, P_, B, fulcs.ctypes.data, pil.ctypes.data,
                         off.ctypes.data, *ptrs, max_k, int(naive), threads, C.byref(st))
    out = {"status": rc, "pilots": pil[: B * parts], "offsets": off, "partitions": parts, "stats": st}
    if intermediates:
        out["bucket_sizes"] = inter["bucket_sizes"][: parts * B].reshape(parts, B)
        out["histo"] = inter["histo"][: parts * 256].reshape(parts, 256)
        out["perm"] = inter["perm"][: parts * B].reshape(parts, B)
        out["sorted_lowers"] = inter["sorted_lowers"][: 2 * n].reshape(n, 2)
    return out


def query(keys4: np.ndarray, parts: int, B: int, fulcs, pilots, offsets, threads: int = 0) -> np.ndarray:
    keys4 = np.ascontiguousarray(keys4, np.uint32)
    n = keys4.shape[0]
    out = np.zeros(max(n, 1), np.uint32)
    orc().orc_query(keys4.ctypes.data if n else None, n, parts, B, fulcs.ctypes.data, pilots.ctypes.data,
                    offsets.ctypes.data, out.ctypes.data, threads)
    return out[:n]


def is_bijection(pos: np.ndarray) -> bool:
    n = len(pos)
    return n == 0 or bool((np.sort(pos) == np.arange(n, dtype=pos.dtype)).all())
