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


def test_noalloc_timeout_then_busy_until_the_work_drains(phobic, monkeypatch):
    """A call whose work cannot finish within PHOBIC_TIMEOUT_MS returns PHOBIC_ERR_TIMEOUT
    and leaves its work queued; until that work has run, the static array is in use and
    another call returns PHOBIC_ERR_BUSY without queueing anything.  Once the stream has
    drained, calls build correctly again.  The work is held back by a bounded sleep kernel
    queued ahead of it on the same stream (about 50 ms), not by anything that can hang."""
    import time

    torch = pytest.importorskip("torch")
    fn = _fn(phobic)
    stream = torch.cuda.Stream()
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(36, 100_000)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    parts = cfg.partitions(len(keys))
    dp = torch.zeros(parts * cfg.bucketCountPerPartition, dtype=torch.int32, device="cuda")
    do = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
    k = phobic.Keys(phobic.KEYS_U64, 1, len(keys), dk.data_ptr(), None)
    r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
    torch.cuda.synchronize()
    assert fn(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream.cuda_stream)) == phobic.OK
    monkeypatch.setenv("PHOBIC_TIMEOUT_MS", "1")
    with torch.cuda.stream(stream):
        torch.cuda._sleep(100_000_000)  # ~50 ms of spinning on the build's stream
    assert fn(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream.cuda_stream)) == phobic.ERR_TIMEOUT
    assert fn(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream.cuda_stream)) == phobic.ERR_BUSY
    monkeypatch.delenv("PHOBIC_TIMEOUT_MS")
    stream.synchronize()
    status = phobic.ERR_BUSY
    for _ in range(200):  # the release runs as a host function behind the drained work
        status = fn(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream.cuda_stream))
        if status != phobic.ERR_BUSY:
            break
        time.sleep(0.01)
    assert status == phobic.OK
    with phobic.Context(0) as ctx:
        want = ctx.build(keys, cfg)
    assert np.array_equal(dp.cpu().numpy().view(np.uint32), want.pilots)
    assert np.array_equal(do.cpu().numpy().view(np.uint32), want.partition_offsets)


def test_noalloc_refuses_a_capturing_stream(phobic):
    """The call is synchronous, so it must not be captured into a CUDA graph: on a stream
    that is capturing it returns PHOBIC_ERR_INVALID and queues nothing (the graph stays
    empty); the same call outside the capture builds normally."""
    torch = pytest.importorskip("torch")
    fn = _fn(phobic)
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(37, 50_000)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    parts = cfg.partitions(len(keys))
    dp = torch.zeros(parts * cfg.bucketCountPerPartition, dtype=torch.int32, device="cuda")
    do = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
    k = phobic.Keys(phobic.KEYS_U64, 1, len(keys), dk.data_ptr(), None)
    r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
    torch.cuda.synchronize()
    import warnings

    stream = torch.cuda.Stream()
    graph = torch.cuda.CUDAGraph()
    with warnings.catch_warnings():
        warnings.filterwarnings("ignore", message="The CUDA Graph is empty")  # nothing was queued, by design
        with torch.cuda.graph(graph, stream=stream):
            status = fn(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream.cuda_stream))
    assert status == phobic.ERR_INVALID
    assert fn(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream.cuda_stream)) == phobic.OK
    with phobic.Context(0) as ctx:
        want = ctx.build(keys, cfg)
    assert np.array_equal(dp.cpu().numpy().view(np.uint32), want.pilots)
