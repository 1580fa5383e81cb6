"""Replay of a build's device stages as one CUDA graph, through the C ABI.

A build whose launches are exactly those of the context's previous build (same sizes,
parameters, search shape and buffers) is captured the second time in a row and replayed
from then on (phobic_tuning::graphs_off = 0).  A replay reads the keys and writes the
results wherever the buffers hold them at that moment, so a replayed build of new keys in
the same buffers must give the oracle's pilots for the new keys (search.comp:105-124), the
oracle's error status, and stage timings like a build launched stage by stage."""
import numpy as np
import pytest

import keygen
import oracle_lib as O

pytestmark = pytest.mark.gpu


def oracle(keys, cfg, kind="u64"):
    return O.build(O.hash_keys(keys, kind), cfg.partitionSize, cfg.bucketCountPerPartition, cfg.getFulcs())


def test_repeated_host_builds_replay_and_match(phobic):
    cfg = phobic.MPHFconfig(7.0, 2500)
    with phobic.Context(0) as ctx:
        replays = []
        for i in range(4):
            keys = keygen.splitmix64(100 + i, 300_000)
            got = ctx.build(keys, cfg)
            want = oracle(keys, cfg)
            assert (got.pilots == want["pilots"]).all() and (got.partition_offsets == want["offsets"]).all()
            replays.append(got.timings["graph_replays"])
        assert replays == [0, 1, 1, 1]


def test_device_keys_rewritten_in_place_between_replays(phobic):
    import torch

    cfg = phobic.MPHFconfig(5.0, 2048)
    n = 1_000_000
    parts, B = cfg.partitions(n), cfg.bucketCountPerPartition
    with phobic.Context(0) as ctx:
        dk = torch.empty(n, dtype=torch.int64, device="cuda")
        dp = torch.empty(parts * B, dtype=torch.int32, device="cuda")
        do = torch.empty(parts + 1, dtype=torch.int32, device="cuda")
        replays = []
        for seed in (1, 2, 3, 4):
            keys = keygen.splitmix64(seed, n)
            dk.copy_(torch.from_numpy(keys.view(np.int64)))
            r = ctx.build(dk, cfg, out=(dp, do))
            want = oracle(keys, cfg)
            assert (dp.cpu().numpy().view(np.uint32) == want["pilots"]).all()
            assert (do.cpu().numpy().view(np.uint32) == want["offsets"]).all()
            assert r.timings["bucket_sizes"] > 0 and r.timings["search"] > 0 and r.timings["kernels"] == 6
            replays.append(r.timings["graph_replays"])
        assert replays == [0, 1, 1, 1]


def test_replayed_build_reports_errors_like_the_oracle(phobic):
    cfg = phobic.MPHFconfig(5.0, 2048)
    good = keygen.splitmix64(7, 50_000)
    dup = good.copy()
    dup[5] = dup[4]
    with phobic.Context(0) as ctx:
        for _ in range(2):
            ctx.build(good, cfg)
        with pytest.raises(phobic.PhobicError) as e:
            ctx.build(dup, cfg)
        assert e.value.status == oracle(dup, cfg)["status"] == phobic.ERR_DUPLICATE_KEY
        got = ctx.build(good, cfg)
        assert (got.pilots == oracle(good, cfg)["pilots"]).all()
        assert got.timings["graph_replays"] == 1


def test_strings_replay_and_match(phobic):
    cfg = phobic.MPHFconfig(6.0, 2048)
    strs = keygen.strings(21, 60_000)
    want = oracle(strs, cfg, "strings")
    with phobic.Context(0) as ctx:
        replays = []
        for _ in range(3):
            got = ctx.build(strs, cfg)
            assert (got.pilots == want["pilots"]).all() and (got.partition_offsets == want["offsets"]).all()
            replays.append(got.timings["graph_replays"])
        assert replays == [0, 1, 1]


def test_changed_launches_are_never_replayed(phobic):
    cfg = phobic.MPHFconfig(6.0, 2048)
    a, b = keygen.splitmix64(11, 200_000), keygen.splitmix64(12, 150_000)
    with phobic.Context(0) as ctx:
        ctx.set_tuning(graphs_off=1)
        assert [ctx.build(a, cfg).timings["graph_replays"] for _ in range(3)] == [0, 0, 0]
        ctx.set_tuning()
        replays = []
        for keys in (a, b, a, b):  # other sizes: other launches every time
            got = ctx.build(keys, cfg)
            assert (got.pilots == oracle(keys, cfg)["pilots"]).all()
            replays.append(got.timings["graph_replays"])
        assert replays == [0, 0, 0, 0]
        assert [ctx.build(a, cfg).timings["graph_replays"] for _ in range(2)] == [0, 1]
        ctx.set_tuning(search_group=4, search_pipeline=1)  # another search shape: captured anew
        got = ctx.build(a, cfg)
        assert got.timings["graph_replays"] == 0
        assert (got.pilots == oracle(a, cfg)["pilots"]).all()
        other = phobic.MPHFconfig(6.0, 2048)
        other.params.max_pilot_counter = 3  # another kernel argument: captured anew
        want = O.build(O.hash_keys(a, "u64"), 2048, other.bucketCountPerPartition, other.getFulcs(), max_k=3)
        for _ in range(2):
            if want["status"] == 0:
                assert (ctx.build(a, other).pilots == want["pilots"]).all()
            else:
                with pytest.raises(phobic.PhobicError) as e:
                    ctx.build(a, other)
                assert e.value.status == want["status"]


def test_batch_builds_replay_and_match(phobic):
    cfg = phobic.MPHFconfig(6.0, 2048)
    sets = [keygen.splitmix64(50 + i, 3000 * (i + 1)) for i in range(6)]
    with phobic.Context(0) as ctx:
        for _ in range(3):
            outs, st = phobic.build_batch(ctx, sets, cfg)
            assert all(s == 0 for s in st)
            for keys, r in zip(sets, outs):
                w = oracle(keys, cfg)
                assert (r.pilots == w["pilots"]).all() and (r.partition_offsets == w["offsets"]).all()


def test_large_builds_launch_stage_by_stage(phobic):
    cfg = phobic.MPHFconfig(6.0, 2048)
    keys = keygen.splitmix64(13, 5_000_000)  # 2,442 partitions
    with phobic.Context(0) as ctx:
        got = [ctx.build(keys, cfg) for _ in range(3)]
        assert [g.timings["graph_replays"] for g in got] == [0, 0, 0]
        assert (got[-1].pilots == oracle(keys, cfg)["pilots"]).all()
