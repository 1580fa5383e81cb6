"""Batched builds and the build server through the C ABI: every set's result
equals the plain build of that set alone (bit-exact pilots and offsets), and
every set is a bijection."""
import numpy as np
import pytest

import keygen
import oracle_lib as O

pytestmark = pytest.mark.gpu


def oracle(keys4, cfg):
    r = O.build(keys4, cfg.partitionSize, cfg.bucketCountPerPartition, cfg.getFulcs())
    assert r["status"] == 0
    return r


def test_batch_equals_plain_builds(phobic, ctx):
    cfg = phobic.MPHFconfig(6.0, 2048)
    sizes = [0, 1, 5, 2047, 2048, 2049, 10_000, 1000, 77_777, 3]
    sets = [keygen.splitmix64(100 + i, n) for i, n in enumerate(sizes)]
    outs, st = phobic.build_batch(ctx, sets, cfg)
    assert st == [0] * len(sets)
    for keys, got in zip(sets, outs):
        want = oracle(O.hash_keys(keys, "u64"), cfg)
        assert (got.pilots == want["pilots"]).all()
        assert (got.partition_offsets == want["offsets"]).all()
        if len(keys):
            assert ctx.verify(keys, cfg, got) == 0


def test_flat_batch_equals_list_batch(phobic, ctx):
    """build_batch_flat (one key buffer, set sizes, flat results; device and host keys)
    gives every set the result of build_batch and of the oracle."""
    torch = pytest.importorskip("torch")
    cfg = phobic.MPHFconfig(6.0, 2048)
    sizes = np.array([0, 1, 5, 2047, 2048, 2049, 10_000, 0, 77_777, 3])
    keys = keygen.splitmix64(900, int(sizes.sum()))
    starts = np.concatenate([[0], np.cumsum(sizes)])
    sets = [keys[starts[i]:starts[i + 1]] for i in range(len(sizes))]
    outs, st = phobic.build_batch(ctx, sets, cfg)
    assert st == [0] * len(sets)
    pstart, ostart = phobic.batch_layout(sizes, cfg)
    for flat_keys in (torch.from_numpy(keys.view(np.int64)).cuda(), keys):
        fp, fo, fst, _ = phobic.build_batch_flat(ctx, flat_keys, sizes, cfg)
        assert (fst == 0).all()
        fp = fp.cpu().numpy().view(np.uint32) if hasattr(fp, "cpu") else fp
        fo = fo.cpu().numpy().view(np.uint32) if hasattr(fo, "cpu") else fo
        for i, got in enumerate(outs):
            assert (fp[pstart[i]:pstart[i + 1]] == got.pilots).all(), i
            assert (fo[ostart[i]:ostart[i + 1]] == got.partition_offsets).all(), i
    for i in (2, 5, 8):
        want = oracle(O.hash_keys(sets[i], "u64"), cfg)
        assert (outs[i].pilots == want["pilots"]).all()


def test_batch_many_small_sets_log_uniform(phobic, ctx):
    cfg = phobic.MPHFconfig(6.0, 2048)
    sizes = keygen.set_sizes(4, 300, 1000, 200_000)
    sets = [keygen.splitmix64(10_000 + i, int(n)) for i, n in enumerate(sizes)]
    outs, st = phobic.build_batch(ctx, sets, cfg)
    assert all(s == 0 for s in st)
    for i in range(0, len(sets), 37):
        want = oracle(O.hash_keys(sets[i], "u64"), cfg)
        assert (outs[i].pilots == want["pilots"]).all()
    for keys, got in zip(sets, outs):
        assert ctx.verify(keys, cfg, got) == 0


def test_batch_strings_and_mixed_kinds(phobic, ctx):
    cfg = phobic.MPHFconfig(6.0, 2048)
    s1 = keygen.strings(31, 5000)
    s2 = keygen.strings(32, 12_000)
    u = keygen.splitmix64(33, 9000)
    outs, st = phobic.build_batch(ctx, [s1, u, s2], cfg)
    assert st == [0, 0, 0]
    for keys, kind, got in ((s1, "strings", outs[0]), (u, "u64", outs[1]), (s2, "strings", outs[2])):
        want = oracle(O.hash_keys(keys, kind), cfg)
        assert (got.pilots == want["pilots"]).all()


def test_batch_reports_per_set_errors(phobic, ctx):
    cfg = phobic.MPHFconfig(6.0, 2048)
    good = keygen.splitmix64(40, 5000)
    dup = keygen.splitmix64(41, 5000)
    dup[7] = dup[3]
    outs, st = phobic.build_batch(ctx, [good, dup, good.copy()], cfg)
    assert st[0] == 0 and st[2] == 0 and st[1] == phobic.ERR_DUPLICATE_KEY
    assert ctx.verify(good, cfg, outs[0]) == 0 and ctx.verify(good, cfg, outs[2]) == 0


def test_server_results_equal_alone(phobic):
    """Continuous batching: two large requests occupy both streams while 40 small ones
    arrive; the small ones are built in batches of several requests, two batches are on
    the device at once, and every result equals the oracle's (and the plain build's)."""
    cfg = phobic.MPHFconfig(7.0, 2048)
    rng = np.random.default_rng(5)
    big = [keygen.splitmix64(498, 20_000_000), keygen.splitmix64(499, 20_000_000)]
    reqs = []
    for i in range(40):
        n = int(np.exp(rng.uniform(np.log(1e3), np.log(3e5))))
        reqs.append(keygen.strings(500 + i, n) if i % 3 == 2 else keygen.splitmix64(500 + i, n))
    with phobic.Server(0, streams=2, budget_bytes=16 << 30) as srv:
        big_tickets = [srv.submit(k, cfg) for k in big]
        tickets = [srv.submit(k, cfg) for k in reqs]
        big_results = [srv.wait(t) for t in big_tickets]
        results = [srv.wait(t) for t in tickets]
        stats = srv.stats()
    assert stats["completed"] == len(reqs) + len(big) and stats["failed"] == 0
    assert stats["p50_ms"] > 0 and stats["p99_ms"] >= stats["p50_ms"]
    assert stats["peak_bytes"] <= 16 << 30
    assert stats["max_batch_requests"] > 1, stats     # requests were batched together
    assert stats["max_batches_in_flight"] > 1, stats  # on more than one stream at once
    assert stats["max_device_overlap"] > 1, stats     # and their device work overlapped
    for i, (keys, (st, got)) in enumerate(zip(reqs, results)):
        assert st == 0
        want = oracle(O.hash_keys(keys, "strings" if i % 3 == 2 else "u64"), cfg)
        assert (got.pilots == want["pilots"]).all() and (got.partition_offsets == want["offsets"]).all()
    with phobic.Context(0) as alone:
        for keys, (st, got) in zip(big, big_results):
            assert st == 0
            ref = alone.build(keys, cfg)
            assert (got.pilots == ref.pilots).all() and (got.partition_offsets == ref.partition_offsets).all()


def test_server_budget_admission(phobic):
    cfg = phobic.MPHFconfig(7.0, 2048)
    big = keygen.splitmix64(9, 2_000_000)
    small = keygen.splitmix64(10, 10_000)
    need = phobic.lib().phobic_build_bytes_needed(
        __import__("ctypes").byref(phobic.keyset(big).struct()), __import__("ctypes").byref(cfg.params))
    with phobic.Server(0, streams=2, budget_bytes=need + (1 << 20)) as srv:
        with pytest.raises(phobic.PhobicError) as e:
            srv.submit(keygen.splitmix64(11, 3_000_000), cfg)
        assert e.value.status == phobic.ERR_BUDGET
        t1 = srv.submit(big, cfg)
        t2 = srv.submit(big.copy(), cfg)
        t3 = srv.submit(small, cfg)
        for t in (t1, t2, t3):
            st, _ = srv.wait(t)
            assert st == 0
        assert srv.stats()["peak_bytes"] <= need + (1 << 20)


def test_server_reserve_sizes_every_stream(phobic):
    """phobic_server_reserve sizes each stream's arena up front; requests up to that size
    then build without growing it, and the results equal the plain builds."""
    cfg = phobic.MPHFconfig(7.0, 2048)
    big = keygen.splitmix64(12, 3_000_000)
    dev, pinned = phobic.Server.bytes_for(big, cfg)
    with phobic.Server(0, streams=3, budget_bytes=3 * dev + (1 << 20)) as srv:
        with pytest.raises(phobic.PhobicError) as e:
            srv.reserve(dev + (1 << 21), pinned)
        assert e.value.status == phobic.ERR_BUDGET
        srv.reserve(dev, pinned)
        assert srv.stats()["peak_bytes"] == 0
        reqs = [big, keygen.splitmix64(13, 1_000_000), keygen.splitmix64(14, 20_000)]
        tickets = [srv.submit(k, cfg) for k in reqs]
        outs = [srv.wait(t) for t in tickets]
        srv.reserve(dev, pinned)  # idle again: a no-op
        assert srv.stats()["peak_bytes"] <= 3 * dev
    with phobic.Context(0) as alone:
        for k, (st, got) in zip(reqs, outs):
            assert st == 0
            ref = alone.build(k, cfg)
            assert (got.pilots == ref.pilots).all() and (got.partition_offsets == ref.partition_offsets).all()


def test_concurrent_contexts_with_different_launch_shapes(phobic):
    """Two contexts build from two host threads at once, with different partition counts
    and (lambda, P), so their kernels ask for different amounts of shared memory; every
    build succeeds and equals the same build made alone."""
    import threading

    jobs = [(phobic.MPHFconfig(7.0, 2500), [20_000, 3_000_000, 200_000, 6_000_000]),
            (phobic.MPHFconfig(3.0, 1024), [1_000_000, 50_000, 4_000_000])]
    keys = {n: keygen.splitmix64(900 + n % 97, n) for _, sizes in jobs for n in sizes}
    errors, firsts = [], {}

    def run(j, cfg, sizes):
        try:
            with phobic.Context(0) as c:
                for r in range(40):
                    n = sizes[r % len(sizes)]
                    got = c.build(keys[n], cfg)
                    firsts.setdefault((j, n), got)
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(repr(e))

    threads = [threading.Thread(target=run, args=(j, cfg, sizes)) for j, (cfg, sizes) in enumerate(jobs)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    with phobic.Context(0) as alone:
        for (j, n), got in firsts.items():
            ref = alone.build(keys[n], jobs[j][0])
            assert (got.pilots == ref.pilots).all() and (got.partition_offsets == ref.partition_offsets).all()
