"""Parity at the sizes the workloads are quoted on, through the C ABI.

  * C2: all 10^8 u64 keys of splitmix64(seed 2), lambda 7, P 2500 (40,000 partitions);
  * C3: all 5*10^7 strings (lengths 8..64, printable ASCII, seed 3), lambda 6, P 2048;
  * C4: every one of the 4096 sets of one batched build (2.13*10^9 keys, seed 4),
    lambda 6, P 2048.

Each GPU result is compared element by element with the oracle's build of the same
keys (pilots search.comp:126-175, layout mphf_builder.h:254-261), then with the
SHA-256 digests committed by tests/golden/make_golden.py, whose C2 pilots the
reference's own query accepts as a bijection.  These sizes take the K1 counter plan,
the K3 coarse-bin width and the scan grid of the headline builds, which the smaller
parity cases do not reach.
"""
import hashlib

import numpy as np
import pytest

import keygen
import oracle_lib as O

pytestmark = pytest.mark.gpu


def sha(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _first_diff(a, b) -> str:
    idx = np.nonzero(a != b)[0]
    return f"{idx.size} differ, first at {idx[0] if idx.size else None}"


def test_c2_full_100M_pilots_bit_exact(phobic, ctx, golden):
    torch = pytest.importorskip("torch")
    rec = golden["full_builds"]["C2_u64_seed2_n1e8_l7_P2500"]
    cfg = phobic.MPHFconfig(7.0, 2500)
    keys = keygen.splitmix64(2, 100_000_000)
    parts, B = cfg.partitions(len(keys)), cfg.bucketCountPerPartition
    assert parts == rec["partitions"] == 40_000
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    dp = torch.empty(parts * B, dtype=torch.int32, device="cuda")
    do = torch.empty(parts + 1, dtype=torch.int32, device="cuda")
    got = ctx.build(dk, cfg, out=(dp, do))
    assert ctx.verify(dk, cfg, got) == 0
    pil, off = dp.cpu().numpy().view(np.uint32), do.cpu().numpy().view(np.uint32)
    del dk, dp, do
    want = O.build(O.hash_keys(keys, "u64"), 2500, B, cfg.getFulcs())
    assert want["status"] == 0
    assert np.array_equal(off, want["offsets"]), _first_diff(off, want["offsets"])
    assert np.array_equal(pil, want["pilots"]), _first_diff(pil, want["pilots"])
    assert sha(pil) == rec["pilots_sha256"] and sha(off) == rec["offsets_sha256"]


def test_c3_full_50M_strings_bit_exact(phobic, ctx, golden):
    torch = pytest.importorskip("torch")
    rec = golden["full_builds"]["C3_strings_seed3_n5e7_l6_P2048"]
    cfg = phobic.MPHFconfig(6.0, 2048)
    data, offs = keygen.strings(3, 50_000_000)
    assert sha(data) == rec["bytes_sha256"] and sha(offs) == rec["offsets_input_sha256"]
    n = len(offs) - 1
    parts, B = cfg.partitions(n), cfg.bucketCountPerPartition
    dd = torch.from_numpy(data).cuda()
    doffs = torch.from_numpy(offs.view(np.int64)).cuda()
    ks = phobic.KeySet(phobic.KEYS_STRINGS, n, dd, doffs, True)
    dp = torch.empty(parts * B, dtype=torch.int32, device="cuda")
    do = torch.empty(parts + 1, dtype=torch.int32, device="cuda")
    got = ctx.build(ks, cfg, out=(dp, do))
    assert ctx.verify(ks, cfg, got) == 0
    pil, off = dp.cpu().numpy().view(np.uint32), do.cpu().numpy().view(np.uint32)
    del dd, doffs, dp, do
    want = O.build(O.hash_keys((data, offs), "strings"), 2048, B, cfg.getFulcs())
    assert want["status"] == 0
    assert np.array_equal(off, want["offsets"]), _first_diff(off, want["offsets"])
    assert np.array_equal(pil, want["pilots"]), _first_diff(pil, want["pilots"])
    assert sha(pil) == rec["pilots_sha256"] and sha(off) == rec["offsets_sha256"]


def test_c4_full_batch_every_set_bit_exact(phobic, ctx, golden):
    """One batched build of all 4096 sets; every set equals the oracle's build of that set."""
    torch = pytest.importorskip("torch")
    rec = golden["full_builds"]["C4_batch_u64_seed4_4096sets_l6_P2048"]
    cfg = phobic.MPHFconfig(6.0, 2048)
    B = cfg.bucketCountPerPartition
    sizes = keygen.set_sizes(4, 4096, 1000, 4 << 20)
    total = int(sizes.sum())
    assert total == rec["total_keys"]
    keys = keygen.splitmix64_cuda(4, total)
    starts = np.concatenate([[0], np.cumsum(sizes)])
    parts = [cfg.partitions(int(n)) for n in sizes]
    pstart = np.concatenate([[0], np.cumsum([B * m for m in parts])])
    ostart = np.concatenate([[0], np.cumsum([m + 1 for m in parts])])
    fp = torch.empty(int(pstart[-1]), dtype=torch.int32, device="cuda")
    fo = torch.empty(int(ostart[-1]), dtype=torch.int32, device="cuda")
    sets = [keys[int(starts[i]):int(starts[i + 1])] for i in range(len(sizes))]
    outs = [(fp[int(pstart[i]):int(pstart[i + 1])], fo[int(ostart[i]):int(ostart[i + 1])]) for i in range(len(sizes))]
    _, st = phobic.build_batch(ctx, sets, cfg, outs_in=outs)
    assert all(s == 0 for s in st)
    pil_all, off_all = fp.cpu().numpy().view(np.uint32), fo.cpu().numpy().view(np.uint32)
    del fp, fo, outs
    hp, ho = hashlib.sha256(), hashlib.sha256()
    fulcs = cfg.getFulcs()
    for i, n in enumerate(sizes):
        host_keys = sets[i].cpu().numpy().view(np.uint64)
        want = O.build(O.hash_keys(host_keys, "u64"), 2048, B, fulcs)
        assert want["status"] == 0
        p = pil_all[int(pstart[i]):int(pstart[i + 1])]
        o = off_all[int(ostart[i]):int(ostart[i + 1])]
        assert np.array_equal(o, want["offsets"]), (i, int(n), _first_diff(o, want["offsets"]))
        assert np.array_equal(p, want["pilots"]), (i, int(n), _first_diff(p, want["pilots"]))
        hp.update(p.tobytes())
        ho.update(o.tobytes())
    assert hp.hexdigest() == rec["pilots_concat_sha256"]
    assert ho.hexdigest() == rec["offsets_concat_sha256"]
