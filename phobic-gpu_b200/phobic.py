"""Python binding of libphobic_b200.so (the C ABI in include/phobic_b200.h).

Mirrors the reference's build surface (stefanfred/PHOBIC-GPU,
include/phobicGpu/mphf_builder.h and mphf_config.h):

    cfg = MPHFconfig(7.0, 2500)          # MPHFconfig(double λ, uint32_t P)
    builder = MPHFbuilder(cfg)           # MPHFbuilder(MPHFconfig)
    res = builder.build(keys)            # pilots[B * partitions], partition offsets[partitions + 1]

Keys are numpy arrays (uint64 keys, or (n, 2) uint64 / (n, 4) uint32 records), lists
of bytes (strings), or CUDA tensors (device-resident keys).  The library must be
built (``python phobic-gpu_b200/build.py``); there is no CPU fallback: every call
goes through the CUDA kernels or raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parent
# PHOBIC_LIBRARY=checked selects the bounds-checked build of the same library.
LIB_PATH = PKG / "lib" / ("libphobic_b200_checked.so" if os.environ.get("PHOBIC_LIBRARY") == "checked"
                          else "libphobic_b200.so")
FULCRUMS = 2048

OK, ERR_INVALID, ERR_OOM, ERR_BUCKET_OVERFLOW, ERR_PARTITION_OVERFLOW = 0, 1, 2, 3, 4
ERR_SEARCH_LIMIT, ERR_TIMEOUT, ERR_CUDA, ERR_DUPLICATE_KEY, ERR_BUDGET = 5, 6, 7, 8, 9
ERR_BUSY, ERR_NO_DEVICE, ERR_NOT_FOUND, ERR_KEYS_CHANGED = 10, 11, 12, 13
KEYS_U64, KEYS_BYTES16, KEYS_PREHASHED, KEYS_STRINGS = 0, 1, 2, 3
BUCKETER_OPT, BUCKETER_UNIFORM, BUCKETER_SKEW = 0, 1, 2


class Params(C.Structure):
    _fields_ = [
        ("partition_size", C.c_uint32),
        ("buckets", C.c_uint32),
        ("max_partition_size", C.c_uint32),
        ("max_pilot_counter", C.c_uint32),
        ("fulcrums", C.c_uint32 * FULCRUMS),
    ]


class Keys(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("on_device", C.c_int32),
        ("n", C.c_uint64),
        ("data", C.c_void_p),
        ("offsets", C.c_void_p),
    ]


class Result(C.Structure):
    _fields_ = [("on_device", C.c_int32), ("pilots", C.c_void_p), ("partition_offsets", C.c_void_p)]


class Timings(C.Structure):
    _fields_ = [
        ("input_transfer", C.c_float),
        ("bucket_sizes", C.c_float),
        ("partition_offsets", C.c_float),
        ("key_redistribution", C.c_float),
        ("search", C.c_float),
        ("result_transfer", C.c_float),
        ("total", C.c_float),
        ("kernels", C.c_uint32),
        ("graph_replays", C.c_uint32),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_}


class Tuning(C.Structure):
    _fields_ = [("search_group", C.c_uint32), ("search_pipeline", C.c_uint32), ("graphs_off", C.c_uint32),
                ("reserved", C.c_uint32 * 5)]


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("streams", C.c_uint32),
        ("queue_capacity", C.c_uint32),
        ("max_batch_sets", C.c_uint32),
        ("budget_bytes", C.c_uint64),
    ]


class ServerStats(C.Structure):
    _fields_ = [
        ("completed", C.c_uint64),
        ("failed", C.c_uint64),
        ("keys", C.c_uint64),
        ("p50_ms", C.c_double),
        ("p99_ms", C.c_double),
        ("max_ms", C.c_double),
        ("busy_ms", C.c_double),
        ("peak_bytes", C.c_uint64),
        ("max_batch_requests", C.c_uint32),
        ("max_batches_in_flight", C.c_uint32),
        ("max_device_overlap", C.c_uint32),
        ("pad", C.c_uint32),
    ]


class PhobicError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        name = _lib().phobic_status_string(status).decode() if _LIB else str(status)
        super().__init__(f"{name}{': ' + detail if detail else ''} (status {status})")


_LIB: C.CDLL | None = None
P = C.c_void_p
PP = C.POINTER(C.c_void_p)
U32, U64, I32 = C.c_uint32, C.c_uint64, C.c_int


def _lib() -> C.CDLL:
    """Load the in-tree library (raises if it was not built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise RuntimeError(f"{LIB_PATH} is missing: run python phobic-gpu_b200/build.py")
    lib = C.CDLL(str(LIB_PATH))
    sig = {
        "phobic_status_string": (C.c_char_p, [I32]),
        "phobic_partitions": (U32, [U64, U32]),
        "phobic_config": (I32, [C.c_double, U32, I32, I32, C.POINTER(Params)]),
        "phobic_ctx_create": (I32, [I32, PP]),
        "phobic_ctx_destroy": (I32, [P]),
        "phobic_last_error": (C.c_char_p, [P]),
        "phobic_ctx_device_bytes": (U64, [P]),
        "phobic_ctx_stream": (P, [P]),
        "phobic_ctx_set_memory_limit": (I32, [P, U64]),
        "phobic_build_bytes_needed": (U64, [C.POINTER(Keys), C.POINTER(Params)]),
        "phobic_build": (I32, [P, C.POINTER(Keys), C.POINTER(Params), C.POINTER(Result), C.POINTER(Timings)]),
        "phobic_build_u64": (I32, [P, P, U64, C.POINTER(Params), P, P, C.POINTER(Timings)]),
        "phobic_build_strings": (I32, [P, P, P, U64, C.POINTER(Params), P, P, C.POINTER(Timings)]),
        "phobic_build_batch": (I32, [P, C.POINTER(Keys), U32, C.POINTER(Params), C.POINTER(Result), C.POINTER(I32),
                                     C.POINTER(Timings)]),
        "phobic_query": (I32, [P, C.POINTER(Keys), C.POINTER(Params), U32, C.POINTER(Result), P]),
        "phobic_verify": (I32, [P, C.POINTER(Keys), C.POINTER(Params), C.POINTER(Result), C.POINTER(U64)]),
        "phobic_debug_build": (I32, [P, C.POINTER(Keys), C.POINTER(Params), C.POINTER(Result), P, P]),
        "phobic_debug_stalled_wait": (I32, [P, U32, C.POINTER(I32)]),
        "phobic_debug_checks": (I32, [P, C.POINTER(I32), C.POINTER(U32), I32]),
        "phobic_encode": (I32, [I32, I32, P, P, U32, C.POINTER(Params), C.c_float, P, C.c_size_t,
                                C.POINTER(C.c_size_t), C.POINTER(C.c_double)]),
        "phobic_encode_gpu": (I32, [P, I32, I32, C.POINTER(Result), U32, C.POINTER(Params), P, C.c_size_t, I32,
                                    C.POINTER(C.c_size_t), C.POINTER(C.c_double)]),
        "phobic_ctx_result": (I32, [P, U32, U32, C.POINTER(Result)]),
        "phobic_build_noalloc": (I32, [C.POINTER(Keys), C.POINTER(Params), C.POINTER(Result), P]),
        "phobic_debug_change_key": (I32, [U64, U64]),
        "phobic_measure_int_peak": (I32, [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
        "phobic_ctx_kernel_arch": (I32, [P, C.POINTER(I32)]),
        "phobic_ctx_set_tuning": (I32, [P, C.POINTER(Tuning)]),
        "phobic_autotune": (I32, [P, C.POINTER(Params), C.c_char_p, C.POINTER(U32)]),
        "phobic_server_create": (I32, [C.POINTER(ServerConfig), PP]),
        "phobic_server_submit": (I32, [P, C.POINTER(Keys), C.POINTER(Params), C.POINTER(Result), C.POINTER(U64)]),
        "phobic_server_poll": (I32, [P, U64, C.POINTER(I32), C.POINTER(I32)]),
        "phobic_server_wait": (I32, [P, U64, U32, C.POINTER(I32)]),
        "phobic_server_drain": (I32, [P, U32]),
        "phobic_server_reserve": (I32, [P, U64, U64]),
        "phobic_server_stats_get": (I32, [P, C.POINTER(ServerStats)]),
        "phobic_server_destroy": (I32, [P]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype, fn.argtypes = res, args
    _LIB = lib
    return lib


def lib() -> C.CDLL:
    return _lib()


def check(status: int, ctx: "Context | None" = None) -> None:
    if status != OK:
        detail = _lib().phobic_last_error(ctx.handle).decode() if ctx is not None and ctx.handle else ""
        raise PhobicError(status, detail)


# ------------------------------------------------------------------ configuration

class MPHFconfig:
    """MPHFconfig(λ, P) (mphf_config.h:26-34); bucketer_ctor=True mirrors MPHFconfig(Bucketer*, λ, P)."""

    def __init__(self, average_bucket_size: float = 8.0, partition_size: int = 2048,
                 bucketer: int = BUCKETER_OPT, bucketer_ctor: bool = False):
        self.params = Params()
        check(_lib().phobic_config(float(average_bucket_size), int(partition_size), int(bucketer),
                                   int(bool(bucketer_ctor)), C.byref(self.params)))
        self.m_averageBucketSize = float(average_bucket_size)
        self.partitionSize = int(partition_size)
        self.bucketCountPerPartition = int(self.params.buckets)
        self.sortingBins = 256

    def getFulcs(self) -> np.ndarray:
        return np.ctypeslib.as_array(self.params.fulcrums).copy()

    def partitionMaxSize(self) -> int:
        return self.partitionSize + self.partitionSize // 2

    def partitions(self, n: int) -> int:
        return int(_lib().phobic_partitions(int(n), self.partitionSize))


# ------------------------------------------------------------------ keys

@dataclass
class KeySet:
    """A key set in the layout the C ABI expects; keeps its buffers alive."""
    kind: int
    n: int
    data: object
    offsets: object = None
    on_device: bool = False
    _keep: list = field(default_factory=list)

    def struct(self) -> Keys:
        return Keys(self.kind, int(self.on_device), self.n, _ptr(self.data), _ptr(self.offsets))


def _ptr(x) -> int | None:
    if x is None:
        return None
    if isinstance(x, np.ndarray):
        return x.ctypes.data if x.size else None
    if hasattr(x, "data_ptr"):
        return x.data_ptr() if x.numel() else None
    if isinstance(x, int):
        return x
    raise TypeError(f"unsupported buffer {type(x)}")


def keyset(keys, kind: int | None = None) -> KeySet:
    """Wrap keys: uint64 array -> U64; (n,2) uint64 -> BYTES16; (n,4) uint32 -> PREHASHED unless kind given;
    list of bytes/str -> STRINGS; a (bytes, offsets) tuple -> STRINGS; CUDA tensors stay on the device."""
    if isinstance(keys, KeySet):
        return keys
    if isinstance(keys, tuple) and len(keys) == 2:
        data, offs = keys
        on_dev = hasattr(data, "is_cuda") and data.is_cuda
        if not on_dev:
            data = np.ascontiguousarray(np.frombuffer(data, np.uint8) if isinstance(data, (bytes, bytearray)) else data,
                                        dtype=np.uint8)
            offs = np.ascontiguousarray(offs, dtype=np.uint64)
        return KeySet(KEYS_STRINGS, int(len(offs) - 1), data, offs, on_dev)
    if isinstance(keys, list):
        enc = [k.encode() if isinstance(k, str) else bytes(k) for k in keys]
        offs = np.zeros(len(enc) + 1, np.uint64)
        np.cumsum([len(e) for e in enc], out=offs[1:])
        data = np.frombuffer(b"".join(enc), np.uint8) if enc else np.zeros(0, np.uint8)
        return KeySet(KEYS_STRINGS, len(enc), np.ascontiguousarray(data), offs)
    if hasattr(keys, "is_cuda") and keys.is_cuda:
        if keys.dim() == 1:
            return KeySet(KEYS_U64 if kind is None else kind, int(keys.shape[0]), keys.contiguous(), None, True)
        return KeySet(KEYS_BYTES16 if kind is None else kind, int(keys.shape[0]), keys.contiguous(), None, True)
    a = np.ascontiguousarray(keys)
    if a.dtype == np.int64:  # the same 8 bytes per key: a view, not a copy (a pinned buffer stays pinned)
        a = a.view(np.uint64)
    if a.ndim == 1:
        return KeySet(KEYS_U64 if kind is None else kind, a.shape[0], a.astype(np.uint64, copy=False))
    if a.ndim == 2 and a.dtype == np.uint64 and a.shape[1] == 2:
        return KeySet(KEYS_BYTES16 if kind is None else kind, a.shape[0], a)
    if a.ndim == 2 and a.dtype == np.uint32 and a.shape[1] == 4:
        return KeySet(KEYS_PREHASHED if kind is None else kind, a.shape[0], a)
    raise TypeError("keys must be uint64[n], uint64[n,2], uint32[n,4], list of bytes, or (bytes, offsets)")


# ------------------------------------------------------------------ context

@dataclass
class BuildResult:
    pilots: object             # [buckets * partitions] (bucket-major)
    partition_offsets: object  # [partitions + 1]
    partitions: int
    buckets: int
    timings: dict | None = None


class Context:
    """A phobic_ctx on one CUDA device."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        check(_lib().phobic_ctx_create(int(device), C.byref(h)))
        self.handle = h.value
        self.device = device

    def close(self) -> None:
        if self.handle:
            _lib().phobic_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_error(self) -> str:
        return _lib().phobic_last_error(self.handle).decode()

    def device_bytes(self) -> int:
        return int(_lib().phobic_ctx_device_bytes(self.handle))

    def stream_handle(self) -> int:
        """cudaStream_t of this context (all of its kernels run on it)."""
        return int(_lib().phobic_ctx_stream(self.handle) or 0)

    def _result(self, cfg: MPHFconfig, n: int, out=None):
        parts = cfg.partitions(n)
        if out is not None:
            pil, off = out
            return Result(int(_is_cuda(pil)), _ptr(pil), _ptr(off)), pil, off, parts
        pil = np.zeros(cfg.bucketCountPerPartition * parts, np.uint32)
        off = np.zeros(parts + 1, np.uint32)
        return Result(0, _ptr(pil), _ptr(off)), pil, off, parts

    def build(self, keys, cfg: MPHFconfig, out=None, kind: int | None = None) -> BuildResult:
        ks = keyset(keys, kind)
        res, pil, off, parts = self._result(cfg, ks.n, out)
        _torch_first(self, ks.data, ks.offsets, pil, off)
        t = Timings()
        k = ks.struct()
        check(_lib().phobic_build(self.handle, C.byref(k), C.byref(cfg.params), C.byref(res), C.byref(t)), self)
        return BuildResult(pil, off, parts, cfg.bucketCountPerPartition, t.as_dict())

    def debug_build(self, keys, cfg: MPHFconfig, kind: int | None = None):
        ks = keyset(keys, kind)
        res, pil, off, parts = self._result(cfg, ks.n)
        keys4 = np.zeros((max(ks.n, 1), 4), np.uint32)
        sizes = np.zeros(max(parts * cfg.bucketCountPerPartition, 1), np.uint32)
        _torch_first(self, ks.data, ks.offsets)
        k = ks.struct()
        check(_lib().phobic_debug_build(self.handle, C.byref(k), C.byref(cfg.params), C.byref(res),
                                        keys4.ctypes.data, sizes.ctypes.data), self)
        return (BuildResult(pil, off, parts, cfg.bucketCountPerPartition), keys4[: ks.n],
                sizes[: parts * cfg.bucketCountPerPartition].reshape(parts, cfg.bucketCountPerPartition))

    def query(self, keys, cfg: MPHFconfig, built: BuildResult, kind: int | None = None):
        """Slot of every key: a numpy uint32 array for host keys, an int32 CUDA tensor on the
        keys' device for device-resident keys (phobic_query writes positions where the keys are)."""
        ks = keyset(keys, kind)
        if ks.on_device:
            import torch
            pos = torch.empty(max(ks.n, 1), dtype=torch.int32, device=ks.data.device)
            ptr = pos.data_ptr()
        else:
            pos = np.zeros(max(ks.n, 1), np.uint32)
            ptr = pos.ctypes.data
        res = Result(int(_is_cuda(built.pilots)), _ptr(built.pilots), _ptr(built.partition_offsets))
        _torch_first(self, ks.data, ks.offsets, built.pilots, built.partition_offsets, pos)
        k = ks.struct()
        check(_lib().phobic_query(self.handle, C.byref(k), C.byref(cfg.params), built.partitions, C.byref(res),
                                  ptr), self)
        return pos[: ks.n]

    def set_memory_limit(self, nbytes: int) -> None:
        """Cap the device memory of this context's build pool (0 = no cap)."""
        check(_lib().phobic_ctx_set_memory_limit(self.handle, nbytes), self)

    def checks(self, reset: bool = False) -> tuple[bool, list[int]]:
        """(checked library?, source lines of the first failed bounds check in the
        key-mapping, partition and search kernels; 0 = none)."""
        compiled = C.c_int32()
        lines = (U32 * 3)()
        check(_lib().phobic_debug_checks(self.handle, C.byref(compiled), lines, int(reset)), self)
        return bool(compiled.value), list(lines)

    def stalled_wait(self, wait_ms: int) -> int:
        """Status recorded by a kernel whose bounded wait on a never-set flag ran out."""
        st = C.c_int()
        check(_lib().phobic_debug_stalled_wait(self.handle, wait_ms, C.byref(st)), self)
        return int(st.value)

    def set_tuning(self, search_group: int = 0, search_pipeline: int = 0, graphs_off: int = 0) -> None:
        """Launch shapes of later builds: warps per partition of the search (0 = automatic),
        whether a group pipelines small buckets (1) or splits pilot counters (0), and whether a
        build that repeats the previous build's launches may replay them as a CUDA graph (0)
        or always launches its stages one by one (1)."""
        t = Tuning()
        t.search_group = search_group
        t.search_pipeline = search_pipeline
        t.graphs_off = graphs_off
        check(_lib().phobic_ctx_set_tuning(self.handle, C.byref(t)), self)

    def autotune(self, cfg: "MPHFconfig", path: str | None = None) -> int:
        """Time the search shapes for a ladder of sizes at cfg's parameters and write the
        fastest per size class to the tuning table (phobic_autotune); returns lines written."""
        n = C.c_uint32()
        check(_lib().phobic_autotune(self.handle, C.byref(cfg.params), path.encode() if path else None,
                                     C.byref(n)), self)
        return int(n.value)

    def int_peak(self) -> tuple[float, float]:
        """(32-bit integer ops per second, kernel ms) of the pilot hash's mixing round on this
        device, all SMs at full occupancy (phobic_measure_int_peak)."""
        ops, ms = C.c_double(), C.c_double()
        check(_lib().phobic_measure_int_peak(self.handle, C.byref(ops), C.byref(ms)), self)
        return float(ops.value), float(ms.value)

    def kernel_arch(self) -> int:
        """cudaFuncAttributes::binaryVersion of the library's kernels (100 = sm_100)."""
        v = C.c_int()
        check(_lib().phobic_ctx_kernel_arch(self.handle, C.byref(v)), self)
        return int(v.value)

    def verify(self, keys, cfg: MPHFconfig, built: BuildResult, kind: int | None = None) -> int:
        """Number of keys whose slot is out of range or taken twice (0 = bijection)."""
        ks = keyset(keys, kind)
        res = Result(int(_is_cuda(built.pilots)), _ptr(built.pilots), _ptr(built.partition_offsets))
        bad = C.c_uint64()
        _torch_first(self, ks.data, ks.offsets, built.pilots, built.partition_offsets)
        k = ks.struct()
        check(_lib().phobic_verify(self.handle, C.byref(k), C.byref(cfg.params), C.byref(res), C.byref(bad)), self)
        return int(bad.value)


def debug_change_key(index: int, xor_mask: int) -> None:
    """Arm phobic_debug_change_key: the next build of one set of device-visible u64 keys
    flips key `index` by `xor_mask` between its counting and placing passes."""
    check(_lib().phobic_debug_change_key(index, xor_mask))


def _is_cuda(x) -> bool:
    return bool(getattr(x, "is_cuda", False))


def _torch_first(ctx: "Context", *bufs) -> None:
    """Work queued on torch's current stream may still be writing these device tensors
    (keys made on the GPU, outputs just zeroed).  The context's stream waits for it, by
    an event (no host synchronisation).  The library's calls return once their work is
    done, so later torch work sees complete results."""
    if any(_is_cuda(b) for b in bufs):
        import torch
        torch.cuda.ExternalStream(ctx.stream_handle()).wait_stream(torch.cuda.current_stream())


class MPHFbuilder:
    """MPHFbuilder(MPHFconfig) (mphf_builder.h:36-48): build(keys) -> BuildResult."""

    def __init__(self, config: MPHFconfig | None = None, device: int = 0):
        self.config = config or MPHFconfig()
        self.ctx = Context(device)

    def build(self, keys, out=None) -> BuildResult:
        return self.ctx.build(keys, self.config, out)


# ------------------------------------------------------------------ encoding

PILOT_ENCODERS = {"interleaved_compact": 0, "interleaved_dictionary": 1, "interleaved_rice": 2, "mono_compact": 3,
                  "mono_dictionary": 4, "dual_rice_compact": 5, "interleaved_elias_fano": 6, "interleaved_sdc": 7,
                  "mono_rice": 8}
OFFSET_ENCODERS = {"diff": 0, "direct": 1}


def encode(built: BuildResult, cfg: MPHFconfig, pilot_encoder: str = "interleaved_compact",
           offset_encoder: str = "diff", tradeoff: float = 0.5) -> tuple[bytes, float]:
    """Mphf::setData on the host (the reference's encoders, same bytes): (serialised bytes, bits per key)."""
    pil = np.ascontiguousarray(built.pilots, np.uint32)
    off = np.ascontiguousarray(built.partition_offsets, np.uint32)
    size, bpk = C.c_size_t(), C.c_double()
    args = (PILOT_ENCODERS[pilot_encoder], OFFSET_ENCODERS[offset_encoder], pil.ctypes.data, off.ctypes.data,
            built.partitions, C.byref(cfg.params), tradeoff)
    # One pass into a buffer sized for every encoder (at most 8 bytes per pilot and
    # offset plus headers); a second pass only if the encoding is larger.
    cap = 8 * (pil.size + off.size) + 64 * (built.buckets + 2) + (1 << 16)
    buf = np.empty(cap, np.uint8)
    check(_lib().phobic_encode(*args, buf.ctypes.data, cap, C.byref(size), C.byref(bpk)))
    if size.value > cap:
        buf = np.empty(size.value, np.uint8)
        check(_lib().phobic_encode(*args, buf.ctypes.data, size.value, C.byref(size), C.byref(bpk)))
    return buf[: size.value].tobytes(), bpk.value


def encode_gpu(ctx: "Context", built: BuildResult, cfg: MPHFconfig, pilot_encoder: str = "interleaved_compact",
               offset_encoder: str = "diff", out=None) -> tuple[bytes | None, float, int]:
    """Mphf::setData on the GPU for the compact-vector encoders (interleaved_compact or
    mono_compact pilots, diff or direct offsets): (serialised bytes, bits per key, size).
    The bytes equal encode()'s.  built's arrays may be torch CUDA tensors (read in
    place) or numpy arrays.  With out (a torch CUDA uint8 tensor) the bytes are
    written there and None is returned in their place."""
    res = Result(int(_is_cuda(built.pilots)), _ptr(built.pilots), _ptr(built.partition_offsets))
    _torch_first(ctx, built.pilots, built.partition_offsets, out)
    size, bpk = C.c_size_t(), C.c_double()
    args = (ctx.handle, PILOT_ENCODERS[pilot_encoder], OFFSET_ENCODERS[offset_encoder], C.byref(res),
            built.partitions, C.byref(cfg.params))
    if out is not None:
        check(_lib().phobic_encode_gpu(*args, _ptr(out), out.numel(), 1, C.byref(size), C.byref(bpk)), ctx)
        return None, bpk.value, size.value
    check(_lib().phobic_encode_gpu(*args, None, 0, 0, C.byref(size), C.byref(bpk)), ctx)
    buf = np.zeros(max(size.value, 1), np.uint8)
    check(_lib().phobic_encode_gpu(*args, buf.ctypes.data, size.value, 0, C.byref(size), C.byref(bpk)), ctx)
    return buf[: size.value].tobytes(), bpk.value, size.value


# ------------------------------------------------------------------ pilot-layout files

_LAYOUT_MAGIC = b"PHBLAYT1"


def save_layout(path, built: BuildResult, cfg: MPHFconfig) -> None:
    """Write a build's pilots and partition offsets (before any encoding) in the file
    layout of the C++ layer's savePilotLayout: magic, n, partitions, buckets, P, then
    the bucket-major pilots and the offsets, all little-endian."""
    pil = np.ascontiguousarray(_host(built.pilots), np.uint32).reshape(-1)
    off = np.ascontiguousarray(_host(built.partition_offsets), np.uint32).reshape(-1)
    if pil.size != built.buckets * built.partitions or off.size != built.partitions + 1:
        raise ValueError("result arrays do not match their partition and bucket counts")
    head = np.array([built.partitions, built.buckets, cfg.partitionSize, 0], "<u4")
    with open(path, "wb") as f:
        f.write(_LAYOUT_MAGIC)
        f.write(np.array([int(off[-1])], "<u8").tobytes())
        f.write(head.tobytes())
        f.write(pil.astype("<u4", copy=False).tobytes())
        f.write(off.astype("<u4", copy=False).tobytes())


def load_layout(path) -> tuple[BuildResult, int]:
    """Read a file written by save_layout (or savePilotLayout): (result, partition size)."""
    data = open(path, "rb").read()
    if data[:8] != _LAYOUT_MAGIC or len(data) < 32:
        raise ValueError("not a pilot-layout file")
    n = int(np.frombuffer(data, "<u8", 1, 8)[0])
    parts, buckets, psize, _ = (int(x) for x in np.frombuffer(data, "<u4", 4, 16))
    npil = parts * buckets
    if len(data) != 32 + 4 * (npil + parts + 1):
        raise ValueError("pilot-layout file size does not match its header")
    pil = np.frombuffer(data, "<u4", npil, 32).astype(np.uint32)
    off = np.frombuffer(data, "<u4", parts + 1, 32 + 4 * npil).astype(np.uint32)
    if off[0] != 0 or int(off[-1]) != n:
        raise ValueError("pilot-layout file has inconsistent partition offsets")
    return BuildResult(pil, off, parts, buckets), psize


def _host(x):
    return x.cpu().numpy().view(np.uint32) if hasattr(x, "cpu") else x


# ------------------------------------------------------------------ batch and serving

def build_batch(ctx: Context, key_sets: list, cfg: MPHFconfig, kind: int | None = None, outs_in: list | None = None):
    """Build many key sets in one pass of the kernels; returns (results, statuses).
    outs_in: optional (pilots, offsets) per set (e.g. CUDA tensors for device results)."""
    kss = [keyset(k, kind) for k in key_sets]
    arr = (Keys * len(kss))(*[k.struct() for k in kss])
    outs, res_structs = [], []
    for i, ks in enumerate(kss):
        r, pil, off, parts = ctx._result(cfg, ks.n, outs_in[i] if outs_in else None)
        outs.append(BuildResult(pil, off, parts, cfg.bucketCountPerPartition))
        res_structs.append(r)
    rarr = (Result * len(kss))(*res_structs)
    _torch_first(ctx, *[b for ks in kss for b in (ks.data, ks.offsets)], *[b for o in outs for b in (o.pilots, o.partition_offsets)])
    st = (C.c_int * len(kss))()
    t = Timings()
    rc = _lib().phobic_build_batch(ctx.handle, arr, len(kss), C.byref(cfg.params), rarr, st, C.byref(t))
    for o in outs:
        o.timings = t.as_dict()
    if rc not in (OK,) and all(s == OK for s in st):
        check(rc, ctx)
    return outs, [int(s) for s in st]


# numpy images of phobic_keys and phobic_result (one row per set), for batches of many sets.
_KEYS_DT = np.dtype({"names": ["kind", "on_device", "n", "data", "offsets"],
                     "formats": [np.int32, np.int32, np.uint64, np.uint64, np.uint64],
                     "offsets": [0, 4, 8, 16, 24], "itemsize": 32})
_RESULT_DT = np.dtype({"names": ["on_device", "pilots", "partition_offsets"],
                       "formats": [np.int32, np.uint64, np.uint64], "offsets": [0, 8, 16], "itemsize": 24})


def batch_layout(sizes, cfg: MPHFconfig) -> tuple[np.ndarray, np.ndarray]:
    """Start of every set's pilots and partition offsets in flat result arrays (one more
    entry than sets: the totals), for build_batch_flat."""
    sizes = np.asarray(sizes, dtype=np.int64)
    parts = (sizes + cfg.partitionSize - 1) // cfg.partitionSize
    pstart = np.zeros(len(sizes) + 1, np.int64)
    np.cumsum(parts * cfg.bucketCountPerPartition, out=pstart[1:])
    ostart = np.zeros(len(sizes) + 1, np.int64)
    np.cumsum(parts + 1, out=ostart[1:])
    return pstart, ostart


def build_batch_flat(ctx: Context, keys, sizes, cfg: MPHFconfig, pilots=None, offsets=None,
                     kind: int = KEYS_U64) -> tuple[object, object, np.ndarray, dict]:
    """Batched build of consecutive sets of one flat key array: set i is the next sizes[i]
    keys (u64, or 16-byte records with kind BYTES16 / PREHASHED).  Results go to flat arrays
    (created like the keys when None): set i's pilots start at batch_layout(...)[0][i] and its
    partition offsets at batch_layout(...)[1][i].  The C structs of all sets are built as
    numpy arrays, so the host cost does not grow with a Python call per set.  Returns
    (pilots, offsets, statuses, timings)."""
    sizes = np.asarray(sizes, dtype=np.int64)
    nsets = len(sizes)
    pstart, ostart = batch_layout(sizes, cfg)
    width = 8 if kind == KEYS_U64 else 16
    on_dev = _is_cuda(keys)
    if pilots is None or offsets is None:
        if on_dev:
            import torch
            pilots = torch.empty(max(int(pstart[-1]), 1), dtype=torch.int32, device=keys.device)
            offsets = torch.empty(int(ostart[-1]), dtype=torch.int32, device=keys.device)
        else:
            pilots = np.zeros(max(int(pstart[-1]), 1), np.uint32)
            offsets = np.zeros(int(ostart[-1]), np.uint32)
    kstart = np.zeros(nsets, np.int64)
    if nsets > 1:
        np.cumsum(sizes[:-1], out=kstart[1:])
    karr = np.zeros(nsets, _KEYS_DT)
    karr["kind"] = kind
    karr["on_device"] = int(on_dev)
    karr["n"] = sizes
    karr["data"] = np.uint64(_ptr(keys) or 0) + (kstart * width).astype(np.uint64)
    rarr = np.zeros(nsets, _RESULT_DT)
    rarr["on_device"] = int(_is_cuda(pilots))
    rarr["pilots"] = np.uint64(_ptr(pilots) or 0) + (pstart[:-1] * 4).astype(np.uint64)
    rarr["partition_offsets"] = np.uint64(_ptr(offsets)) + (ostart[:-1] * 4).astype(np.uint64)
    st = np.zeros(nsets, np.int32)
    _torch_first(ctx, keys, pilots, offsets)
    t = Timings()
    rc = _lib().phobic_build_batch(ctx.handle, C.cast(karr.ctypes.data, C.POINTER(Keys)), nsets,
                                   C.byref(cfg.params), C.cast(rarr.ctypes.data, C.POINTER(Result)),
                                   C.cast(st.ctypes.data, C.POINTER(C.c_int)), C.byref(t))
    if rc != OK and (st == OK).all():
        check(rc, ctx)
    return pilots, offsets, st, t.as_dict()


class Server:
    """phobic_server: continuous-batching build server on one device."""

    def __init__(self, device: int = 0, streams: int = 2, budget_bytes: int = 8 << 30, queue_capacity: int = 65536,
                 max_batch_sets: int = 0):
        cfg = ServerConfig(device, streams, queue_capacity, max_batch_sets, budget_bytes)
        h = C.c_void_p()
        check(_lib().phobic_server_create(C.byref(cfg), C.byref(h)))
        self.handle = h.value
        self._live = {}

    def submit(self, keys, cfg: MPHFconfig, kind: int | None = None, out=None) -> int:
        """Queue one build; out = (pilots, offsets) arrays (host numpy or CUDA tensors) or None."""
        ks = keyset(keys, kind)
        parts = cfg.partitions(ks.n)
        if out is None:
            pil = np.zeros(max(cfg.bucketCountPerPartition * parts, 1), np.uint32)
            off = np.zeros(parts + 1, np.uint32)
        else:
            pil, off = out
        res = Result(int(_is_cuda(pil)), _ptr(pil), _ptr(off))
        if any(_is_cuda(b) for b in (ks.data, ks.offsets, pil, off)):
            # The worker stream that will run the build is chosen later: let torch's
            # queued writes to these tensors finish first.
            import torch
            torch.cuda.current_stream().synchronize()
        k = ks.struct()
        t = C.c_uint64()
        check(_lib().phobic_server_submit(self.handle, C.byref(k), C.byref(cfg.params), C.byref(res), C.byref(t)))
        self._live[t.value] = (ks, k, res, BuildResult(pil[: cfg.bucketCountPerPartition * parts] if out is None else pil,
                                                        off, parts, cfg.bucketCountPerPartition))
        return int(t.value)

    def wait(self, ticket: int, timeout_ms: int = 600_000) -> tuple[int, BuildResult]:
        st = C.c_int()
        check(_lib().phobic_server_wait(self.handle, ticket, timeout_ms, C.byref(st)))
        return int(st.value), self._live.pop(ticket)[3]

    def poll(self, ticket: int) -> tuple[bool, int]:
        done, st = C.c_int(), C.c_int()
        check(_lib().phobic_server_poll(self.handle, ticket, C.byref(done), C.byref(st)))
        return bool(done.value), int(st.value)

    def drain(self, timeout_ms: int = 600_000) -> None:
        check(_lib().phobic_server_drain(self.handle, timeout_ms))

    def reserve(self, device_bytes: int, pinned_bytes: int = 0) -> None:
        """Size every stream's device arena and pinned result stage now (phobic_server_reserve)."""
        check(_lib().phobic_server_reserve(self.handle, device_bytes, pinned_bytes))

    @staticmethod
    def bytes_for(keys, cfg: MPHFconfig, kind: int | None = None) -> tuple[int, int]:
        """(device_bytes, pinned_bytes) one request for these keys needs: the arena of
        phobic_build_bytes_needed and the stage for results bound for pageable memory."""
        ks = keyset(keys, kind)
        k = ks.struct()
        dev = int(_lib().phobic_build_bytes_needed(C.byref(k), C.byref(cfg.params)))
        parts = cfg.partitions(ks.n)
        return dev, 4 * (cfg.bucketCountPerPartition * parts + parts + 1) + 512

    def stats(self) -> dict:
        s = ServerStats()
        check(_lib().phobic_server_stats_get(self.handle, C.byref(s)))
        return {name: getattr(s, name) for name, _ in s._fields_}

    def close(self) -> None:
        if self.handle:
            _lib().phobic_server_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
