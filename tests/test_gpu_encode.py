"""Encoding on the GPU (phobic_encode_gpu) against the host encoders.

The compact-vector encoders (interleaved<compact> and mono<compact> pilots, diff
and direct compact offsets) are written by kernels; their bytes and bits per key
must equal the host encoders' (phobic_encode, which follows the reference's
encoders byte for byte) and the golden SHA-256 of the reference's own encoders."""
import hashlib

import numpy as np
import pytest

import keygen

pytestmark = pytest.mark.gpu

PILOT = ("interleaved_compact", "mono_compact")
OFFSET = ("diff", "direct")


def host_and_gpu(phobic, ctx, built, cfg, pe, oe):
    want, want_bpk = phobic.encode(built, cfg, pe, oe)
    got, got_bpk, size = phobic.encode_gpu(ctx, built, cfg, pe, oe)
    return want, want_bpk, got, got_bpk, size


@pytest.mark.parametrize("n", [0, 1, 2, 31, 2047, 2049, 10_000, 200_000])
@pytest.mark.parametrize("lam,P", [(5.0, 2048), (7.0, 2500)])
def test_gpu_encoding_equals_host_encoding(phobic, ctx, n, lam, P):
    cfg = phobic.MPHFconfig(lam, P)
    built = ctx.build(keygen.splitmix64(31, n), cfg)
    for pe in PILOT:
        for oe in OFFSET:
            want, want_bpk, got, got_bpk, size = host_and_gpu(phobic, ctx, built, cfg, pe, oe)
            assert size == len(want), (pe, oe)
            assert got == want, (pe, oe)
            assert got_bpk == want_bpk, (pe, oe)


def test_gpu_encoding_from_device_result(phobic, ctx):
    torch = pytest.importorskip("torch")
    cfg = phobic.MPHFconfig(7.0, 2500)
    n = 300_000
    keys = keygen.splitmix64(32, n)
    host = ctx.build(keys, cfg)
    parts = cfg.partitions(n)
    pil = torch.zeros(cfg.bucketCountPerPartition * parts, dtype=torch.int32, device="cuda")
    off = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
    dev = ctx.build(torch.from_numpy(keys.view(np.int64)).cuda(), cfg, out=(pil, off))
    for pe in PILOT:
        for oe in OFFSET:
            want, want_bpk = phobic.encode(host, cfg, pe, oe)
            got, got_bpk, _ = phobic.encode_gpu(ctx, dev, cfg, pe, oe)
            assert got == want and got_bpk == want_bpk, (pe, oe)
            # bytes written to device memory
            buf = torch.zeros(len(want), dtype=torch.uint8, device="cuda")
            none, bpk2, size = phobic.encode_gpu(ctx, dev, cfg, pe, oe, out=buf)
            assert none is None and size == len(want) and bpk2 == want_bpk
            assert bytes(buf.cpu().numpy().tobytes()) == want


@pytest.mark.parametrize("case,seed,n,lam,P", [("C1_u64_seed1_n1e6_l5_P2048", 1, 1_000_000, 5.0, 2048),
                                               ("C2_sample_u64_seed2_n2e6_l7_P2500", 2, 2_000_000, 7.0, 2500)])
def test_gpu_encoding_matches_reference_golden(phobic, ctx, golden, case, seed, n, lam, P):
    cfg = phobic.MPHFconfig(lam, P)
    built = ctx.build(keygen.splitmix64(seed, n), cfg)
    want = golden["builds"][case]["encoded"]
    for pe in PILOT:
        for oe in OFFSET:
            got, bpk, size = phobic.encode_gpu(ctx, built, cfg, pe, oe)
            w = want[f"{pe}+{oe}"]
            assert size == w["bytes"], (pe, oe)
            assert hashlib.sha256(got).hexdigest() == w["sha256"], (pe, oe)
            assert abs(bpk - w["bits_per_key"]) < 1e-6


def test_gpu_encoding_rejects_other_encoders(phobic, ctx):
    cfg = phobic.MPHFconfig(7.0, 2500)
    built = ctx.build(keygen.splitmix64(33, 5000), cfg)
    for pe in ("interleaved_dictionary", "interleaved_rice", "mono_dictionary", "dual_rice_compact"):
        with pytest.raises(phobic.PhobicError) as e:
            phobic.encode_gpu(ctx, built, cfg, pe, "diff")
        assert e.value.status == phobic.ERR_INVALID
