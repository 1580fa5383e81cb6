"""Sweep of the search's launch shapes (warps per partition) across workload sizes.

    python phobic-gpu_b200/shape_sweep.py [--device 0] [--seeds 11] [--cases C1,C2,...]

For each case (the parameter sets and set sizes of the benchmark workloads) and seed,
builds the same synthetic u64 keys (splitmix64 on the device) with every shape of the
search (one warp per partition "1", k-split groups "2k" and "4k", bucket pipelines "2p",
"4p" and "8p", and "auto", the shape a build gets by default), device-resident keys and
results, and prints one JSON line per case: build and search ms per shape (CUDA events on
the context's stream) and whether each shape's pilots equal the one-warp build's.  Set PHOBIC_TUNING_FILE to a missing path to see the automatic rule instead of
the shipped tuning table.
"""
from __future__ import annotations

import argparse
import json
import statistics
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parent))

SHAPES = [("1", 1, 0), ("2k", 2, 0), ("4k", 4, 0), ("2p", 2, 1), ("4p", 4, 1), ("8p", 8, 1), ("auto", 0, 0)]
CASES = [("C1", 5.0, 2048, 1_000_000), ("C5 median request", 7.0, 2048, 700_000),
         ("C4 small set", 6.0, 2048, 10_000), ("C4 mid set", 6.0, 2048, 100_000),
         ("C4 large set", 6.0, 2048, 4_000_000), ("C5 large request", 7.0, 2048, 20_000_000),
         ("C3-size u64", 6.0, 2048, 50_000_000), ("C2", 7.0, 2500, 100_000_000)]


def main() -> None:
    import torch

    import keygen
    import phobic

    ap = argparse.ArgumentParser()
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--seeds", default="11", help="comma-separated key seeds")
    ap.add_argument("--cases", default="", help="comma-separated case names (default: all)")
    args = ap.parse_args()
    seeds = [int(x) for x in args.seeds.split(",")]
    wanted = {c for c in args.cases.split(",") if c}
    torch.cuda.set_device(args.device)
    ctx = phobic.Context(args.device)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    for (name, lam, P, n), seed in [(c, sd) for c in CASES for sd in seeds]:
        if wanted and name not in wanted:
            continue
        cfg = phobic.MPHFconfig(lam, P)
        keys = keygen.splitmix64_cuda(seed, n)
        parts, B = cfg.partitions(n), cfg.bucketCountPerPartition
        dp = torch.empty(max(parts * B, 1), dtype=torch.int32, device="cuda")
        do = torch.empty(parts + 1, dtype=torch.int32, device="cuda")
        row = {"case": name, "seed": seed, "lambda": lam, "P": P, "n": n, "partitions": parts}
        ref = None
        for label, g, pipe in SHAPES:
            ctx.set_tuning(search_group=g, search_pipeline=pipe)
            steps = 20 if n <= 4_000_000 else 5
            for _ in range(3):
                ctx.build(keys, cfg, out=(dp, do))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            a.record(stream)
            search = []
            for _ in range(steps):
                r = ctx.build(keys, cfg, out=(dp, do))
                search.append(r.timings["search"])
            b.record(stream)
            torch.cuda.synchronize()
            out = dp.clone()
            same = ref is None or bool(torch.equal(out, ref))
            ref = out if ref is None else ref
            row[label] = {"build_ms": a.elapsed_time(b) / steps, "search_ms": statistics.median(search),
                          "equal_1": same}
        ctx.set_tuning(search_group=0)
        print(json.dumps(row), flush=True)
        del keys, dp, do, ref
        torch.cuda.empty_cache()
    ctx.close()


if __name__ == "__main__":
    main()
