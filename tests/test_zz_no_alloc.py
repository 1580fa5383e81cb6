"""phobic_build_noalloc: the build entry point for callers that cannot allocate.

Some callers cannot call cudaMalloc: a framework that owns the device memory pool
and only hands out buffers it sized itself, a latency-critical path that cannot
pay for an allocation's implicit synchronisation, or a plugin host that forbids
allocation in its callbacks.  phobic_build_noalloc takes all its scratch memory
from one static device array inside the library instead.

These tests call it through the C ABI on device-resident keys, twice in a row with
different key sets, and require its pilots and partition offsets to equal, bit
for bit, those of the regular phobic_build entry point on the same inputs.  The
file is named so that pytest collects it last.
"""
import ctypes as C

import numpy as np
import pytest

import keygen

pytestmark = pytest.mark.gpu


def _device_build(phobic, fn_noalloc, keys, cfg, torch, stream_handle):
    """Run phobic_build_noalloc into fresh device arrays and return them on the host."""
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    parts = cfg.partitions(len(keys))
    dp = torch.full((max(parts * cfg.bucketCountPerPartition, 1),), -1, dtype=torch.int32, device="cuda")
    do = torch.full((parts + 1,), -1, dtype=torch.int32, device="cuda")
    k = phobic.Keys(phobic.KEYS_U64, 1, len(keys), dk.data_ptr(), None)
    r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
    torch.cuda.synchronize()
    status = fn_noalloc(C.byref(k), C.byref(cfg.params), C.byref(r), C.c_void_p(stream_handle))
    pil = dp.cpu().numpy().view(np.uint32)[: parts * cfg.bucketCountPerPartition]
    return status, pil, do.cpu().numpy().view(np.uint32)


def test_noalloc_matches_regular_build_twice_in_a_row(phobic):
    torch = pytest.importorskip("torch")
    lib = phobic.lib()
    fn = lib.phobic_build_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(phobic.Keys), C.POINTER(phobic.Params), C.POINTER(phobic.Result), C.c_void_p]
    stream = torch.cuda.Stream()
    cases = [(keygen.splitmix64(2, 300_000), phobic.MPHFconfig(7.0, 2500)),
             (keygen.splitmix64(1, 1_000_000), phobic.MPHFconfig(5.0, 2048))]
    with phobic.Context(0) as ctx:
        for keys, cfg in cases:
            status, pil, off = _device_build(phobic, fn, keys, cfg, torch, stream.cuda_stream)
            assert status == phobic.OK
            want = ctx.build(keys, cfg)
            assert np.array_equal(pil, want.pilots)
            assert np.array_equal(off, want.partition_offsets)


def test_noalloc_rejects_builds_larger_than_its_scratch(phobic):
    torch = pytest.importorskip("torch")
    fn = phobic.lib().phobic_build_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(phobic.Keys), C.POINTER(phobic.Params), C.POINTER(phobic.Result), C.c_void_p]
    cfg = phobic.MPHFconfig(7.0, 2500)
    n = (1 << 20) + 1
    dk = torch.zeros(n, dtype=torch.int64, device="cuda")
    parts = cfg.partitions(n)
    dp = torch.zeros(parts * cfg.bucketCountPerPartition, dtype=torch.int32, device="cuda")
    do = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
    k = phobic.Keys(phobic.KEYS_U64, 1, n, dk.data_ptr(), None)
    r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
    assert fn(C.byref(k), C.byref(cfg.params), C.byref(r), None) == phobic.ERR_BUDGET
