"""Parity of the CUDA build path with the oracle, through the C ABI.

Bit-exact comparisons: hashed Keys, bucket sizes, partition offsets and pilots
equal the oracle's on the same keys and parameters; every build is a bijection
under the GPU query and under the oracle's query."""
import hashlib

import numpy as np
import pytest

import keygen
import oracle_lib as O

pytestmark = pytest.mark.gpu


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def oracle_build(keys4, cfg, **kw):
    return O.build(keys4, cfg.partitionSize, cfg.bucketCountPerPartition, cfg.getFulcs(), **kw)


def check_against_oracle(phobic, ctx, keys, kind, lam, P, debug=True):
    cfg = phobic.MPHFconfig(lam, P)
    okind = {phobic.KEYS_U64: "u64", phobic.KEYS_BYTES16: "pairs", phobic.KEYS_STRINGS: "strings"}.get(kind)
    if kind == phobic.KEYS_PREHASHED:
        keys4 = np.ascontiguousarray(keys, np.uint32)
    else:
        keys4 = O.hash_keys(keys, okind)
    want = oracle_build(keys4, cfg, intermediates=True)
    assert want["status"] == 0
    if debug:
        got, gkeys4, gsizes = ctx.debug_build(keys, cfg, kind=kind)
        assert (gkeys4 == keys4).all()
        assert (gsizes == want["bucket_sizes"]).all()
    else:
        got = ctx.build(keys, cfg, kind=kind)
    assert (got.partition_offsets == want["offsets"]).all()
    assert (got.pilots == want["pilots"]).all()
    pos = ctx.query(keys, cfg, got, kind=kind)
    assert (pos == O.query(keys4, want["partitions"], cfg.bucketCountPerPartition, cfg.getFulcs(), want["pilots"],
                           want["offsets"])).all()
    assert O.is_bijection(pos)
    assert ctx.verify(keys, cfg, got, kind=kind) == 0
    return got


def test_kernels_report_sm100(ctx):
    """cudaFuncGetAttributes: the loaded kernels are sm_100 binaries."""
    assert ctx.kernel_arch() == 100


@pytest.mark.parametrize("n", [0, 1, 2, 31, 2047, 2049, 10000, 100_000])
def test_u64_small_sizes(phobic, ctx, small_builds, n):
    keys = keygen.splitmix64(1, n)
    got = check_against_oracle(phobic, ctx, keys, phobic.KEYS_U64, 5.0, 2048)
    if f"n{n}_pilots" in small_builds:
        assert (got.pilots == small_builds[f"n{n}_pilots"]).all()


def test_c1_u64_matches_golden(phobic, ctx, golden):
    rec = golden["builds"]["C1_u64_seed1_n1e6_l5_P2048"]
    keys = keygen.splitmix64(1, 1_000_000)
    got = check_against_oracle(phobic, ctx, keys, phobic.KEYS_U64, 5.0, 2048)
    assert sha(got.pilots) == rec["pilots_sha256"]
    assert sha(got.partition_offsets) == rec["offsets_sha256"]


def test_c2_sample_matches_golden(phobic, ctx, golden):
    rec = golden["builds"]["C2_sample_u64_seed2_n2e6_l7_P2500"]
    keys = keygen.splitmix64(2, 2_000_000)
    got = check_against_oracle(phobic, ctx, keys, phobic.KEYS_U64, 7.0, 2500)
    assert sha(got.pilots) == rec["pilots_sha256"]


def test_c3_strings_match_golden(phobic, ctx, golden):
    rec = golden["builds"]["C3_sample_strings_seed3_n2e4_l6_P2048"]
    d, o = keygen.strings(3, 20000)
    got = check_against_oracle(phobic, ctx, (d, o), phobic.KEYS_STRINGS, 6.0, 2048)
    assert sha(got.pilots) == rec["pilots_sha256"]


def test_strings_every_length_0_to_300(phobic, ctx):
    """One string of every length 0..300 (every XXH3 input path), plus 3000 more of
    lengths 4..299 made distinct by a 4-byte index prefix."""
    rng = np.random.default_rng(8)
    lens = np.concatenate([np.arange(0, 301), rng.integers(4, 300, 3000)])
    offs = np.zeros(len(lens) + 1, np.uint64)
    np.cumsum(lens, out=offs[1:])
    data = rng.integers(0, 256, int(offs[-1]), dtype=np.uint8)
    for i, L in enumerate(lens):
        if L >= 4 and i > 300:
            data[int(offs[i]):int(offs[i]) + 4] = np.frombuffer(np.uint32(i).tobytes(), np.uint8)
    keys4 = O.hash_keys((data, offs), "strings")
    assert len(np.unique(keys4, axis=0)) == len(keys4)
    check_against_oracle(phobic, ctx, (data, offs), phobic.KEYS_STRINGS, 5.0, 512)


def test_pairs_and_prehashed(phobic, ctx):
    pairs = keygen.splitmix64(11, 2 * 50_000).reshape(50_000, 2)
    check_against_oracle(phobic, ctx, pairs, phobic.KEYS_BYTES16, 6.0, 2048)
    k4 = keygen.splitmix64(12, 2 * 50_000).view(np.uint32).reshape(50_000, 4)
    check_against_oracle(phobic, ctx, k4, phobic.KEYS_PREHASHED, 6.0, 2048)


@pytest.mark.parametrize("lam,P,bucketer,ctor", [(4.5, 2500, 0, 0), (7.5, 2048, 0, 0), (3.0, 1024, 1, 1),
                                                 (6.0, 4096, 2, 1), (2.0, 256, 0, 0), (8.0, 8192, 0, 0)])
def test_configs_and_bucketers(phobic, ctx, lam, P, bucketer, ctor):
    keys = keygen.splitmix64(21, 60_000)
    cfg = phobic.MPHFconfig(lam, P, bucketer, bool(ctor))
    keys4 = O.hash_keys(keys, "u64")
    want = oracle_build(keys4, cfg)
    assert want["status"] == 0
    got = ctx.build(keys, cfg)
    assert (got.pilots == want["pilots"]).all() and (got.partition_offsets == want["offsets"]).all()


def test_device_resident_keys_and_result(phobic, ctx):
    torch = pytest.importorskip("torch")
    keys = keygen.splitmix64(2, 300_000)
    cfg = phobic.MPHFconfig(7.0, 2500)
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    parts = cfg.partitions(len(keys))
    dp = torch.zeros(parts * cfg.bucketCountPerPartition, dtype=torch.int32, device="cuda")
    do = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
    got = ctx.build(dk, cfg, out=(dp, do))
    want = oracle_build(O.hash_keys(keys, "u64"), cfg)
    assert (dp.cpu().numpy().view(np.uint32) == want["pilots"]).all()
    assert (do.cpu().numpy().view(np.uint32) == want["offsets"]).all()
    assert ctx.verify(dk, cfg, got) == 0


def test_pinned_and_pageable_host_results_agree(phobic, ctx):
    """Host results go straight to pinned memory and through the worker's pinned stage to
    pageable memory (5.7 MB of pilots: the copy-out is split over host threads)."""
    torch = pytest.importorskip("torch")
    keys = keygen.splitmix64(8, 10_000_000)
    cfg = phobic.MPHFconfig(7.0, 2500)
    parts, B = cfg.partitions(len(keys)), cfg.bucketCountPerPartition
    assert 4 * B * parts > 4 << 20
    pageable = ctx.build(keys, cfg)
    pil = torch.zeros(B * parts, dtype=torch.int32).pin_memory()
    off = torch.zeros(parts + 1, dtype=torch.int32).pin_memory()
    ctx.build(keys, cfg, out=(pil, off))
    assert (pil.numpy().view(np.uint32) == pageable.pilots).all()
    assert (off.numpy().view(np.uint32) == pageable.partition_offsets).all()
    small = keygen.splitmix64(9, 3000)
    a, b = ctx.build(small, cfg), ctx.build(small, cfg)
    assert (a.pilots == b.pilots).all() and (a.partition_offsets == b.partition_offsets).all()


def test_bijection_at_ten_million(phobic, ctx):
    keys = keygen.splitmix64(5, 10_000_000)
    cfg = phobic.MPHFconfig(7.0, 2500)
    got = ctx.build(keys, cfg)
    assert ctx.verify(keys, cfg, got) == 0
    # partition offsets are size-independent facts: last = n, increments = partition sizes
    assert got.partition_offsets[-1] == len(keys) and (np.diff(got.partition_offsets.astype(np.int64)) >= 0).all()


def test_bijection_beyond_two_to_the_31_keys(phobic):
    """One set of 2.3 billion keys (above 2^31, so a signed 32-bit index anywhere on the
    path would overflow): the build is a bijection onto [0, n) under the on-device query,
    and the partition offsets end at n.  About 80 GB of device memory."""
    torch = pytest.importorskip("torch")
    n = 2_300_000_000
    cfg = phobic.MPHFconfig(7.0, 2500)
    parts, B = cfg.partitions(n), cfg.bucketCountPerPartition
    keys = keygen.splitmix64_cuda(2, n)
    with phobic.Context(0) as c:
        pil = torch.zeros(B * parts, dtype=torch.int32, device="cuda")
        off = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
        c.build(keys, cfg, out=(pil, off))
        assert c.verify(keys, cfg, phobic.BuildResult(pil, off, parts, B)) == 0
        last = int(off[-1].item()) & 0xFFFFFFFF
        assert last == n
    del keys, pil, off
    torch.cuda.empty_cache()


def test_repeated_builds_are_identical(phobic, ctx):
    keys = keygen.splitmix64(6, 500_000)
    cfg = phobic.MPHFconfig(7.0, 2500)
    a = ctx.build(keys, cfg)
    b = ctx.build(keys, cfg)
    assert (a.pilots == b.pilots).all()


# ------------------------------------------------------------------ error paths (host-made inputs)

def test_partition_overflow_is_reported(phobic, ctx):
    k4 = O.hash_keys(keygen.splitmix64(1, 4000), "u64")
    k4[:, 0] = 7
    cfg = phobic.MPHFconfig(5.0, 2048)
    want = oracle_build(k4, cfg)
    with pytest.raises(phobic.PhobicError) as e:
        ctx.build(k4, cfg, kind=phobic.KEYS_PREHASHED)
    assert e.value.status == want["status"] == phobic.ERR_PARTITION_OVERFLOW


def test_bucket_overflow_is_reported(phobic, ctx):
    k4 = O.hash_keys(keygen.splitmix64(1, 3000), "u64")
    k4[:300, 1] = 5
    k4[:300, 0] = k4[0, 0]
    cfg = phobic.MPHFconfig(5.0, 2048)
    with pytest.raises(phobic.PhobicError) as e:
        ctx.build(k4, cfg, kind=phobic.KEYS_PREHASHED)
    assert e.value.status == oracle_build(k4, cfg)["status"] == phobic.ERR_BUCKET_OVERFLOW


def test_duplicate_keys_are_reported(phobic, ctx):
    keys = keygen.splitmix64(1, 3000)
    keys[1] = keys[0]
    cfg = phobic.MPHFconfig(5.0, 2048)
    with pytest.raises(phobic.PhobicError) as e:
        ctx.build(keys, cfg)
    assert e.value.status == oracle_build(O.hash_keys(keys, "u64"), cfg)["status"] == phobic.ERR_DUPLICATE_KEY


def test_search_limit_is_reported(phobic, ctx):
    keys = keygen.splitmix64(1, 4000)
    cfg = phobic.MPHFconfig(5.0, 2048)
    cfg.params.max_pilot_counter = 1
    with pytest.raises(phobic.PhobicError) as e:
        ctx.build(keys, cfg)
    want = O.build(O.hash_keys(keys, "u64"), 2048, cfg.bucketCountPerPartition, cfg.getFulcs(), max_k=1)
    assert e.value.status == want["status"] == phobic.ERR_SEARCH_LIMIT


def test_context_survives_errors(phobic, ctx):
    keys = keygen.splitmix64(1, 3000)
    keys[1] = keys[0]
    cfg = phobic.MPHFconfig(5.0, 2048)
    with pytest.raises(phobic.PhobicError):
        ctx.build(keys, cfg)
    good = keygen.splitmix64(1, 3000)
    got = ctx.build(good, cfg)
    assert ctx.verify(good, cfg, got) == 0


@pytest.mark.parametrize("case", range(24))
def test_random_configurations_match_oracle(phobic, ctx, case):
    """A seeded sweep of configurations: lambda in [1.5, 9], partition size 64..6000,
    0..150 000 keys, any bucketer and constructor, u64 or 16-byte keys.  The GPU result
    equals the oracle's bit for bit, or both report the same error (an oversized
    partition or bucket)."""
    rng = np.random.default_rng(1000 + case)
    lam = float(np.round(rng.uniform(1.5, 9.0), 2))
    P = int(rng.choice([64, 100, 256, 777, 1024, 2048, 2500, 3000, 4096, 6000]))
    n = int(rng.integers(0, 150_000)) if case % 4 else int(rng.integers(0, 300))
    bucketer, ctor = int(rng.integers(0, 3)), int(rng.integers(0, 2))
    cfg = phobic.MPHFconfig(lam, P, bucketer, bool(ctor))
    if case % 3 == 2:
        keys = keygen.splitmix64(3000 + case, 2 * n).reshape(n, 2)
        keys4, kind = O.hash_keys(keys, "pairs"), phobic.KEYS_BYTES16
    else:
        keys = keygen.splitmix64(3000 + case, n)
        keys4, kind = O.hash_keys(keys, "u64"), phobic.KEYS_U64
    want = oracle_build(keys4, cfg)
    if want["status"] != 0:
        with pytest.raises(phobic.PhobicError) as e:
            ctx.build(keys, cfg, kind=kind)
        assert e.value.status == want["status"], (lam, P, n, bucketer, ctor)
        return
    got = ctx.build(keys, cfg, kind=kind)
    assert (got.partition_offsets == want["offsets"]).all(), (lam, P, n, bucketer, ctor)
    assert (got.pilots == want["pilots"]).all(), (lam, P, n, bucketer, ctor)


# ------------------------------------------------------------------ 52K-104K partitions: packed 16-bit counters in K1

def chunk_of_plan(n):
    """Keys per CTA of K1's chunked plan for an n-key build (148 chunks of >= 16384 keys)."""
    ctas = min(-(-n // 16384), 148)
    return -(-n // ctas)


def partitioner_for(p, M):
    """The smallest partitioner word that maps to partition p of M (partition = (x * M) >> 32)."""
    return (p * (1 << 32) + M - 1) // M


def random_keys4(seed, n):
    return np.random.default_rng(seed).integers(0, 1 << 32, size=(n, 4), dtype=np.uint64).astype(np.uint32)


@pytest.mark.parametrize("kind", ["u64", "pairs"])
def test_packed_counter_builds_match_oracle(phobic, ctx, kind):
    """60 000 partitions of 200 keys: K1 counts in packed 16-bit shared-memory counters;
    keys, bucket sizes, offsets and pilots equal the oracle's."""
    n = 12_000_000
    if kind == "u64":
        keys, k = keygen.splitmix64(41, n), phobic.KEYS_U64
    else:
        keys, k = keygen.splitmix64(42, 2 * n).reshape(n, 2), phobic.KEYS_BYTES16
    assert 52 * 1024 < phobic.MPHFconfig(5.0, 200).partitions(n) <= 104 * 1024
    check_against_oracle(phobic, ctx, keys, k, 5.0, 200)


def test_packed_counter_strings_match_oracle(phobic, ctx):
    """Strings through the packed 16-bit counters: 12M strings of 11..24 bytes, 60 000
    partitions; pilots and offsets equal the oracle's (the string kernels hash ragged
    rows, a separate instance of K1's counting kernel)."""
    cfg = phobic.MPHFconfig(5.0, 200)
    d, o = keygen.strings(46, 12_000_000, 11, 24)
    assert 52 * 1024 < cfg.partitions(len(o) - 1) <= 104 * 1024
    want = oracle_build(O.hash_keys((d, o), "strings"), cfg)
    assert want["status"] == 0
    got = ctx.build((d, o), cfg)
    assert (got.pilots == want["pilots"]).all() and (got.partition_offsets == want["offsets"]).all()


def test_packed_counter_batch_matches_oracle(phobic, ctx):
    """Eight sets whose 58 000 partitions together take the packed plan."""
    cfg = phobic.MPHFconfig(6.0, 200)
    sets = [keygen.splitmix64(700 + i, 400_000 + 300_000 * i) for i in range(8)]
    assert 52 * 1024 < sum(cfg.partitions(len(s)) for s in sets) <= 104 * 1024
    res, st = phobic.build_batch(ctx, sets, cfg)
    for ks, r, s in zip(sets, res, st):
        w = oracle_build(O.hash_keys(ks, "u64"), cfg)
        assert s == w["status"]
        if s == 0:
            assert (r.pilots == w["pilots"]).all() and (r.partition_offsets == w["offsets"]).all()


def test_packed_counter_wrap_reports_lowest_oversized_partition(phobic, ctx):
    """Two chunks each hold 70 000 keys of one partition, so their 16-bit counters wrap
    (partition 40 000 in a low half, 30 001 in a high half).  The wraps are credited
    exactly: the size check reports partition 30 001, as the oracle does."""
    n, cfg = 12_000_000, phobic.MPHFconfig(5.0, 200)
    M = cfg.partitions(n)
    assert 52 * 1024 < M <= 104 * 1024
    k4 = random_keys4(43, n)
    chunk = chunk_of_plan(n)
    assert chunk > 70_000
    for c, p in ((13, 40_000), (62, 30_001)):
        k4[c * chunk: c * chunk + 70_000, 0] = partitioner_for(p, M)
    want = oracle_build(k4, cfg)
    assert want["status"] == phobic.ERR_PARTITION_OVERFLOW and want["stats"].err_partition == 30_001
    with pytest.raises(phobic.PhobicError) as e:
        ctx.build(k4, cfg, kind=phobic.KEYS_PREHASHED)
    assert e.value.status == phobic.ERR_PARTITION_OVERFLOW
    assert "partition 30001)" in str(e.value)


def test_packed_counter_carry_into_the_next_set(phobic, ctx):
    """Set 0's last partition and set 1's first share one packed word.  70 000 keys of
    the former in one chunk wrap the low half and carry one into the high half; the
    carry is taken back, so set 1, whose first partition holds exactly the largest
    allowed size, builds as the oracle builds it."""
    P = 200
    cfg = phobic.MPHFconfig(5.0, P)
    cap = cfg.params.max_partition_size
    n0, n1 = P * 30_001, P * 30_000
    M0, M1 = cfg.partitions(n0), cfg.partitions(n1)
    assert M0 % 2 == 1 and 52 * 1024 < M0 + M1 <= 104 * 1024
    s0, s1 = random_keys4(44, n0), random_keys4(45, n1)
    chunk = chunk_of_plan(n0 + n1)
    s0[13 * chunk: 13 * chunk + 70_000, 0] = partitioner_for(M0 - 1, M0)
    part1 = (s1[:, 0].astype(np.uint64) * M1) >> 32
    move = np.flatnonzero(part1 != 0)[: cap - int((part1 == 0).sum())]
    s1[move, 0] = 0
    assert int((((s1[:, 0].astype(np.uint64) * M1) >> 32) == 0).sum()) == cap
    w0, w1 = oracle_build(s0, cfg), oracle_build(s1, cfg)
    assert w0["status"] == phobic.ERR_PARTITION_OVERFLOW
    res, st = phobic.build_batch(ctx, [s0, s1], cfg, kind=phobic.KEYS_PREHASHED)
    assert st == [w0["status"], w1["status"]]
    if w1["status"] == 0:
        assert (res[1].pilots == w1["pilots"]).all() and (res[1].partition_offsets == w1["offsets"]).all()


def test_pageable_host_keys_upload_in_chunks(phobic, ctx):
    """Host keys in pageable memory go up through the worker's pinned chunk buffers (80 MB of
    u64 keys: three chunks, both buffers; 11 MB of string bytes); the builds equal the builds
    from device-resident keys and from pinned keys."""
    torch = pytest.importorskip("torch")
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(15, 10_000_000)
    want = ctx.build(torch.from_numpy(keys.view(np.int64)).cuda(), cfg)
    for host in (keys, torch.from_numpy(keys.view(np.int64)).pin_memory()):
        got = ctx.build(host, cfg)
        assert (got.pilots == want.pilots).all() and (got.partition_offsets == want.partition_offsets).all()
    strs = [b"k%07d-" % i + bytes(keygen.splitmix64(i, 1).view(np.uint8)[: i % 29]) for i in range(300_000)]
    offs = np.zeros(len(strs) + 1, np.uint64)
    np.cumsum([len(x) for x in strs], out=offs[1:])
    data = np.frombuffer(b"".join(strs), np.uint8).copy()
    assert len(data) > 4 << 20
    sw = ctx.build((torch.from_numpy(data).cuda(), torch.from_numpy(offs.view(np.int64)).cuda()), cfg)
    sg = ctx.build((data, offs), cfg)
    assert (sg.pilots == sw.pilots).all() and (sg.partition_offsets == sw.partition_offsets).all()
    assert ctx.verify((data, offs), cfg, sg) == 0


def test_query_host_and_device_positions_agree(phobic, ctx):
    """Positions of 10M host keys come back through the pinned chunk buffers (40 MB into a
    numpy array: two chunks); device-resident keys get device positions; both agree and
    form a bijection onto [0, n)."""
    torch = pytest.importorskip("torch")
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(16, 10_000_000)
    built = ctx.build(keys, cfg)
    host = ctx.query(keys, cfg, built)
    dev = ctx.query(torch.from_numpy(keys.view(np.int64)).cuda(), cfg, built)
    assert isinstance(host, np.ndarray) and dev.is_cuda
    assert (dev.cpu().numpy().view(np.uint32) == host).all()
    assert O.is_bijection(host)


def test_device_keys_still_being_written_by_torch(phobic, ctx):
    """Keys that torch is still writing (a copy queued behind 0.1 s of work on torch's
    current stream) are read only after that work: the build, the query and a server
    request equal the builds from settled keys."""
    torch = pytest.importorskip("torch")
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(17, 1_000_000)
    src = torch.from_numpy(keys.view(np.int64)).cuda()
    torch.cuda.synchronize()
    want = ctx.build(keys, cfg)
    spin = 200_000_000  # clock cycles of torch's spin kernel: about 0.1 s

    def late_keys():
        dst = torch.zeros_like(src)
        torch.cuda.synchronize()
        torch.cuda._sleep(spin)
        dst.copy_(src)
        return dst

    got = ctx.build(late_keys(), cfg)
    assert (got.pilots == want.pilots).all() and (got.partition_offsets == want.partition_offsets).all()
    pos = ctx.query(late_keys(), cfg, want)
    assert (pos.cpu().numpy().view(np.uint32) == ctx.query(keys, cfg, want)).all()
    with phobic.Server(0, streams=2, budget_bytes=4 << 30) as srv:
        st, r = srv.wait(srv.submit(late_keys(), cfg))
    assert st == 0 and (r.pilots == want.pilots).all()
