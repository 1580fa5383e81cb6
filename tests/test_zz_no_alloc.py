"""phobic_build_noalloc: the build entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc: a framework that owns the device memory pool
and only hands out buffers it sized itself, a latency-critical path that cannot
pay for an allocation's implicit synchronisation, or a plugin host that forbids
allocation in its callbacks.  phobic_build_noalloc takes all its scratch memory
from one static device array inside the library instead.

These tests call it through the C ABI on device-resident keys, several times in a
row with different key sets (larger builds before smaller ones, so leftovers of a
larger call would show), and require its pilots and partition offsets to equal,
bit for bit, those of the regular phobic_build entry point on the same inputs.
The file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import keygen

pytestmark = pytest.mark.gpu


def _fn(phobic):
    fn = phobic.lib().phobic_build_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(phobic.Keys), C.POINTER(phobic.Params), C.POINTER(phobic.Result), C.c_void_p]
    return fn


def _device_build(phobic, fn_noalloc, keys, kind, cfg, torch, stream_handle):
    """Run phobic_build_noalloc into fresh device arrays and return them on the host."""
    n = len(keys)
    flat = np.ascontiguousarray(keys).view(np.int64).reshape(-1)
    dk = torch.from_numpy(flat.copy()).cuda() if flat.size else torch.zeros(1, dtype=torch.int64, device="cuda")
    parts = cfg.partitions(n)
    dp = torch.full((max(parts * cfg.bucketCountPerPartition, 1),), -1, dtype=torch.int32, device="cuda")
    do = torch.full((parts + 1,), -1, dtype=torch.int32, device="cuda")
    k = phobic.Keys(kind, 1, n, dk.data_ptr(), None)
    r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
    torch.cuda.synchronize()
    status = fn_noalloc(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream_handle))
    pil = dp.cpu().numpy().view(np.uint32)[: parts * cfg.bucketCountPerPartition]
    return status, pil, do.cpu().numpy().view(np.uint32)


def test_noalloc_matches_regular_build_twice_in_a_row(phobic):
    torch = pytest.importorskip("torch")
    fn = _fn(phobic)
    stream = torch.cuda.Stream()
    cases = [(keygen.splitmix64(2, 300_000), phobic.MPHFconfig(7.0, 2500)),
             (keygen.splitmix64(1, 1_000_000), phobic.MPHFconfig(5.0, 2048))]
    with phobic.Context(0) as ctx:
        for keys, cfg in cases:
            status, pil, off = _device_build(phobic, fn, keys, phobic.KEYS_U64, cfg, torch, stream.cuda_stream)
            assert status == phobic.OK
            want = ctx.build(keys, cfg)
            assert np.array_equal(pil, want.pilots)
            assert np.array_equal(off, want.partition_offsets)


def test_noalloc_many_partitions_then_smaller_and_every_kind(phobic):
    """5,000 partitions (more than one 4096-entry tile of the in-place scan), then smaller
    builds of 16-byte records, prehashed Keys and no keys at all, each equal to the
    regular build; a larger call's leftovers must not reach a smaller one."""
    torch = pytest.importorskip("torch")
    fn = _fn(phobic)
    stream = torch.cuda.Stream()
    cases = [
        (keygen.splitmix64(31, 1_000_000), phobic.KEYS_U64, phobic.MPHFconfig(7.0, 200)),
        (keygen.splitmix64(32, 2 * 400_000).reshape(400_000, 2), phobic.KEYS_BYTES16, phobic.MPHFconfig(6.0, 2048)),
        (keygen.splitmix64(33, 2 * 70_000).view(np.uint32).reshape(70_000, 4), phobic.KEYS_PREHASHED,
         phobic.MPHFconfig(5.0, 1024)),
        (np.zeros(0, np.uint64), phobic.KEYS_U64, phobic.MPHFconfig(7.0, 2500)),
        (keygen.splitmix64(34, 3000), phobic.KEYS_U64, phobic.MPHFconfig(7.0, 2500)),
    ]
    assert cases[0][2].partitions(1_000_000) > 4096
    with phobic.Context(0) as ctx:
        for keys, kind, cfg in cases:
            status, pil, off = _device_build(phobic, fn, keys, kind, cfg, torch, stream.cuda_stream)
            assert status == phobic.OK, (kind, len(keys))
            want = ctx.build(keys, cfg, kind=kind)
            assert np.array_equal(pil, want.pilots), (kind, len(keys))
            assert np.array_equal(off, want.partition_offsets), (kind, len(keys))


def test_noalloc_reports_keys_changed_between_passes(phobic):
    """A key rewritten between the counting and the placing pass (injected from the host)
    must give PHOBIC_ERR_KEYS_CHANGED; the next call builds correctly."""
    torch = pytest.importorskip("torch")
    fn = _fn(phobic)
    stream = torch.cuda.Stream()
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(35, 200_000)
    phobic.debug_change_key(12_345, 0x5A5A_0000_FFFF_0001)
    status, _, _ = _device_build(phobic, fn, keys, phobic.KEYS_U64, cfg, torch, stream.cuda_stream)
    assert status == phobic.ERR_KEYS_CHANGED
    status, pil, off = _device_build(phobic, fn, keys, phobic.KEYS_U64, cfg, torch, stream.cuda_stream)
    assert status == phobic.OK
    with phobic.Context(0) as ctx:
        want = ctx.build(keys, cfg)
    assert np.array_equal(pil, want.pilots) and np.array_equal(off, want.partition_offsets)


def test_noalloc_rejects_builds_larger_than_its_scratch(phobic):
    torch = pytest.importorskip("torch")
    fn = _fn(phobic)
    cfg = phobic.MPHFconfig(7.0, 2500)
    n = (1 << 20) + 1
    dk = torch.zeros(n, dtype=torch.int64, device="cuda")
    parts = cfg.partitions(n)
    dp = torch.zeros(parts * cfg.bucketCountPerPartition, dtype=torch.int32, device="cuda")
    do = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
    k = phobic.Keys(phobic.KEYS_U64, 1, n, dk.data_ptr(), None)
    r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
    assert fn(C.byref(k), C.byref(cfg.params), C.byref(r), None) == phobic.ERR_BUDGET
