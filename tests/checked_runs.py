"""Parity builds on the bounds-checked library (run by test_gpu_checked.py in a
process of its own, with PHOBIC_LIBRARY=checked): every build must match the
oracle bit for bit and no bounds check may fail."""
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "phobic-gpu_b200"))
sys.path.insert(0, str(ROOT / "tests"))

import numpy as np  # noqa: E402

import keygen  # noqa: E402
import oracle_lib as O  # noqa: E402
import phobic  # noqa: E402


def main() -> int:
    assert phobic.LIB_PATH.name == "libphobic_b200_checked.so", phobic.LIB_PATH
    with phobic.Context(0) as ctx:
        compiled, lines = ctx.checks(reset=True)
        assert compiled, "not the checked library"
        cases = [(7.0, 2500, n) for n in (1, 2, 31, 2047, 2049, 10_000, 300_000)]
        cases += [(5.0, 2048, 200_000), (4.5, 2500, 100_000), (3.0, 1024, 60_000), (6.0, 4096, 60_000),
                  (2.0, 256, 40_000), (8.0, 8192, 60_000), (8.0, 8192, 50_000), (3.63, 64, 84_498),
                  (5.95, 100, 68_243), (4.03, 100, 90_128), (1.5, 777, 137_762),
                  (5.0, 200, 12_000_000)]  # 60 000 partitions: packed 16-bit counters in K1
        for lam, P, n in cases:
            cfg = phobic.MPHFconfig(lam, P)
            keys = keygen.splitmix64(90 + n, n)
            want = O.build(O.hash_keys(keys, "u64"), P, cfg.bucketCountPerPartition, cfg.getFulcs())
            if want["status"] != 0:  # e.g. a bucket above 256 keys: the same error status
                try:
                    ctx.build(keys, cfg)
                    raise AssertionError(f"no error for {(lam, P, n)}")
                except phobic.PhobicError as e:
                    assert e.status == want["status"], (lam, P, n, e.status, want["status"])
                continue
            got = ctx.build(keys, cfg)
            assert np.array_equal(got.pilots, want["pilots"]), (lam, P, n)
            assert np.array_equal(got.partition_offsets, want["offsets"]), (lam, P, n)
        strs = [bytes(keygen.splitmix64(7, 1).view(np.uint8)[: i % 8]) * 5 + b"%d" % i for i in range(30_000)]
        offs = np.zeros(len(strs) + 1, np.uint64)
        np.cumsum([len(x) for x in strs], out=offs[1:])
        data = np.frombuffer(b"".join(strs), np.uint8)
        cfg = phobic.MPHFconfig(6.0, 2048)
        got = ctx.build((data, offs), cfg)
        want = O.build(O.hash_keys((data, offs), "strings"), 2048, cfg.bucketCountPerPartition, cfg.getFulcs())
        assert np.array_equal(got.pilots, want["pilots"])
        for group, pipe in ((1, 0), (2, 0), (4, 0), (8, 0), (2, 1), (4, 1), (8, 1)):  # every search shape
            ctx.set_tuning(search_group=group, search_pipeline=pipe)
            for lam, P, n in ((5.0, 2048, 1_000_000), (8.0, 8192, 200_000), (7.5, 4096, 300_000), (3.0, 64, 5000)):
                g_cfg = phobic.MPHFconfig(lam, P)
                keys = keygen.splitmix64(700 + n % 1000, n)
                w = O.build(O.hash_keys(keys, "u64"), P, g_cfg.bucketCountPerPartition, g_cfg.getFulcs())
                if w["status"] != 0:  # the same error status as the oracle
                    try:
                        ctx.build(keys, g_cfg)
                        raise AssertionError(f"no error for {(group, lam, P, n)}")
                    except phobic.PhobicError as e:
                        assert e.status == w["status"], (group, lam, P, n, e.status)
                    continue
                got = ctx.build(keys, g_cfg)
                assert np.array_equal(got.pilots, w["pilots"]), (group, lam, P, n)
        ctx.set_tuning(search_group=0)
        sets = [keygen.splitmix64(200 + i, 1000 * (i + 1)) for i in range(12)]
        res, st = phobic.build_batch(ctx, sets, cfg)
        for ks, r in zip(sets, res):
            w = O.build(O.hash_keys(ks, "u64"), 2048, cfg.bucketCountPerPartition, cfg.getFulcs())
            assert np.array_equal(r.pilots, w["pilots"])
        compiled, lines = ctx.checks(reset=True)
        print("checked builds:", len(cases) + 2, "failed check lines (map, partition, search):", lines)
        if lines != [0, 0, 0]:
            return 1
        # Keys that change between the passes (injected from the host), on the regular and
        # the no-allocation build: the status must say so.  The clamps that keep such a
        # build's stores inside its arrays fire here by design; the first fired check of
        # each kernel file is printed for the record.
        import ctypes as C

        import torch

        cfg = phobic.MPHFconfig(7.0, 2500)
        keys = keygen.splitmix64(62, 500_000)
        dk = torch.from_numpy(keys.view(np.int64)).cuda()
        phobic.debug_change_key(499_999, 0xFFFF_0000_0000_0000)
        try:
            ctx.build(dk, cfg)
            raise AssertionError("keys changed, yet the build succeeded")
        except phobic.PhobicError as e:
            assert e.status == phobic.ERR_KEYS_CHANGED, e.status
        dk.copy_(torch.from_numpy(keys.view(np.int64)))
        parts = cfg.partitions(len(keys))
        dp = torch.zeros(parts * cfg.bucketCountPerPartition, dtype=torch.int32, device="cuda")
        do = torch.zeros(parts + 1, dtype=torch.int32, device="cuda")
        k = phobic.Keys(phobic.KEYS_U64, 1, len(keys), dk.data_ptr(), None)
        r = phobic.Result(1, dp.data_ptr(), do.data_ptr())
        torch.cuda.synchronize()
        phobic.debug_change_key(12_345, 0x5A5A_0000_FFFF_0001)
        st = phobic.lib().phobic_build_noalloc(C.byref(k), C.byref(cfg.params), C.byref(r), None)
        assert st == phobic.ERR_KEYS_CHANGED, st
        _, fired = ctx.checks(reset=True)
        print("keys-changed builds: status ok; first clamp fired (map, partition, search):", fired)
        return 0


if __name__ == "__main__":
    sys.exit(main())
