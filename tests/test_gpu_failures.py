"""Failure detection on the GPU without faulting it: a kernel wait that nothing
releases must give up after its bound and report a status the host reads, and the
context must keep working afterwards."""
import time

import pytest

import keygen

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(phobic):
    with phobic.Context(0) as ctx:
        t0 = time.perf_counter()
        observed = ctx.stalled_wait(300)
        elapsed = time.perf_counter() - t0
        assert observed == phobic.ERR_TIMEOUT
        assert 0.25 < elapsed < 30
        cfg = phobic.MPHFconfig(7.0, 2500)
        keys = keygen.splitmix64(3, 200_000)
        got = ctx.build(keys, cfg)
        assert ctx.verify(keys, cfg, got) == 0


def test_errors_leave_other_sets_of_a_batch_intact(phobic):
    """A failing set (duplicate keys) in a batch reports its own status; the other
    sets' results are complete and correct."""
    cfg = phobic.MPHFconfig(6.0, 2048)
    good = [keygen.splitmix64(60 + i, 20_000) for i in range(3)]
    bad = keygen.splitmix64(70, 20_000)
    bad[11] = bad[5]
    with phobic.Context(0) as ctx:
        outs, st = phobic.build_batch(ctx, [good[0], bad, good[1], good[2]], cfg)
        assert st == [0, phobic.ERR_DUPLICATE_KEY, 0, 0]
        for keys, res in zip(good, [outs[0], outs[2], outs[3]]):
            assert ctx.verify(keys, cfg, res) == 0


def test_memory_limit_gives_oom_and_context_survives(phobic):
    """An allocation failure injected on the host: the context's memory cap makes the
    build fail with PHOBIC_ERR_OOM before cudaMalloc is called; lifting the cap, the
    same context builds the same keys correctly."""
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(61, 200_000)
    with phobic.Context(0) as c:
        c.set_memory_limit(1 << 20)
        with pytest.raises(phobic.PhobicError) as e:
            c.build(keys, cfg)
        assert e.value.status == phobic.ERR_OOM
        assert c.device_bytes() <= 1 << 20
        c.set_memory_limit(0)
        got = c.build(keys, cfg)
        assert c.verify(keys, cfg, got) == 0


def test_keys_changed_between_passes_is_reported(phobic):
    """Device keys rewritten between the counting pass and the placing pass (injected from
    the host by a one-thread kernel on the build's stream) give PHOBIC_ERR_KEYS_CHANGED,
    with every store kept inside the build's arrays; the context then builds the restored
    keys correctly."""
    torch = pytest.importorskip("torch")
    import numpy as np

    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(62, 500_000)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    with phobic.Context(0) as c:
        phobic.debug_change_key(499_999, 0xFFFF_0000_0000_0000)
        with pytest.raises(phobic.PhobicError) as e:
            c.build(dk, cfg)
        assert e.value.status == phobic.ERR_KEYS_CHANGED
        dk.copy_(torch.from_numpy(keys.view(np.int64)))  # the injected change, undone
        got = c.build(dk, cfg)
        assert c.verify(dk, cfg, got) == 0
        again = c.build(keys, cfg)
        assert (again.pilots == got.pilots).all() and (again.partition_offsets == got.partition_offsets).all()
