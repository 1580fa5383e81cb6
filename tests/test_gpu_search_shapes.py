"""Launch shapes of the search and the autotuner, through the C ABI.

Every shape of the search (one warp per partition; groups of 2, 4 or 8 warps that each
try their own pilot counter per step; groups that search several small buckets at once
and commit them in order) must give the oracle's pilots bit for bit
(search.comp:105-124: smallest pilot counter, then smallest offset), and the same
error status where the oracle reports one.  The autotuner writes its table and later
builds still match the oracle."""
import numpy as np
import pytest

import keygen
import oracle_lib as O

pytestmark = pytest.mark.gpu

# (warps per partition, bucket pipeline): one warp; k-split groups; bucket pipelines.
SHAPES = [(1, 0), (2, 0), (4, 0), (8, 0), (2, 1), (4, 1), (8, 1)]


def oracle(keys4, cfg, **kw):
    return O.build(keys4, cfg.partitionSize, cfg.bucketCountPerPartition, cfg.getFulcs(), **kw)


@pytest.mark.parametrize("group", SHAPES)
@pytest.mark.parametrize("lam,P,n", [(5.0, 2048, 1_000_000), (7.0, 2500, 300_000), (6.0, 2048, 2049),
                                     (8.0, 8192, 200_000), (2.0, 256, 40_000), (1.5, 777, 100_000),
                                     (7.0, 2500, 1), (5.0, 2048, 0), (3.0, 64, 5000)])
def test_every_search_shape_matches_oracle(phobic, lam, P, n, group):
    group, pipe = group
    cfg = phobic.MPHFconfig(lam, P)
    keys = keygen.splitmix64(700 + n % 1000, n)
    want = oracle(O.hash_keys(keys, "u64"), cfg)
    with phobic.Context(0) as ctx:
        ctx.set_tuning(search_group=group, search_pipeline=pipe)
        if want["status"] != 0:
            with pytest.raises(phobic.PhobicError) as e:
                ctx.build(keys, cfg)
            assert e.value.status == want["status"]
            return
        got = ctx.build(keys, cfg)
        assert (got.partition_offsets == want["offsets"]).all()
        assert (got.pilots == want["pilots"]).all()
        if n:
            assert ctx.verify(keys, cfg, got) == 0


@pytest.mark.parametrize("group", SHAPES)
def test_search_shapes_strings_pairs_and_batches(phobic, group):
    group, pipe = group
    cfg = phobic.MPHFconfig(6.0, 2048)
    strs = keygen.strings(41, 30_000)
    pairs = keygen.splitmix64(42, 2 * 25_000).reshape(25_000, 2)
    sets = [keygen.splitmix64(43 + i, 500 * (i + 1) ** 2) for i in range(10)]
    with phobic.Context(0) as ctx:
        ctx.set_tuning(search_group=group, search_pipeline=pipe)
        got = ctx.build(strs, cfg)
        assert (got.pilots == oracle(O.hash_keys(strs, "strings"), cfg)["pilots"]).all()
        got = ctx.build(pairs, cfg, kind=phobic.KEYS_BYTES16)
        assert (got.pilots == oracle(O.hash_keys(pairs, "pairs"), cfg)["pilots"]).all()
        outs, st = phobic.build_batch(ctx, sets, cfg)
        assert all(s == 0 for s in st)
        for keys, r in zip(sets, outs):
            w = oracle(O.hash_keys(keys, "u64"), cfg)
            assert (r.pilots == w["pilots"]).all() and (r.partition_offsets == w["offsets"]).all()


@pytest.mark.parametrize("group", SHAPES)
def test_search_shapes_report_errors_like_the_oracle(phobic, group):
    group, pipe = group
    cfg = phobic.MPHFconfig(5.0, 2048)
    dup = keygen.splitmix64(1, 3000)
    dup[1] = dup[0]
    limited = keygen.splitmix64(1, 4000)
    with phobic.Context(0) as ctx:
        ctx.set_tuning(search_group=group, search_pipeline=pipe)
        with pytest.raises(phobic.PhobicError) as e:
            ctx.build(dup, cfg)
        assert e.value.status == oracle(O.hash_keys(dup, "u64"), cfg)["status"] == phobic.ERR_DUPLICATE_KEY
        lim = phobic.MPHFconfig(5.0, 2048)
        for cap_k in (1, 2, 3, 5):
            lim.params.max_pilot_counter = cap_k
            want = oracle(O.hash_keys(limited, "u64"), lim, max_k=cap_k)
            if want["status"] == 0:
                got = ctx.build(limited, lim)
                assert (got.pilots == want["pilots"]).all()
            else:
                with pytest.raises(phobic.PhobicError) as e:
                    ctx.build(limited, lim)
                assert e.value.status == want["status"] == phobic.ERR_SEARCH_LIMIT
        good = keygen.splitmix64(2, 3000)
        got = ctx.build(good, cfg)
        assert (got.pilots == oracle(O.hash_keys(good, "u64"), cfg)["pilots"]).all()


def test_autotune_writes_its_table_and_builds_still_match(phobic, tmp_path):
    cfg = phobic.MPHFconfig(5.0, 2048)
    table = tmp_path / "tuning.tsv"
    table.write_text("# device\tpartition_size\tbuckets\tmax_partition_size\tmax_partitions\tsearch_group"
                     "\tsearch_pipeline\n"
                     "Some Other GPU\t2048\t410\t3072\t64\t2\t0\n")
    with phobic.Context(0) as ctx:
        assert ctx.autotune(cfg, str(table)) == 8
        lines = [l.split("\t") for l in table.read_text().splitlines() if l and not l.startswith("#")]
        assert ["Some Other GPU", "2048", "410", "3072", "64", "2", "0"] in [l[:7] for l in lines]
        ours = [l for l in lines if l[0] != "Some Other GPU"]
        assert [int(l[4]) for l in ours] == [16, 64, 256, 512, 768, 1024, 2048, 4096]
        assert all((l[5], l[6]) in (("1", "0"), ("2", "0"), ("4", "0"), ("2", "1"), ("4", "1"), ("8", "1"))
                   and len(l) == 13 for l in ours)
        keys = keygen.splitmix64(9, 1_000_000)
        got = ctx.build(keys, cfg)
        assert (got.pilots == oracle(O.hash_keys(keys, "u64"), cfg)["pilots"]).all()
