"""Benchmark of the PHOBIC MPHF construction path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n KEYS]

One step = one complete construction of the serialized pilot layout (the part of
MPHFbuilder::build that the C ABI replaces: hash, partition, bucket sort, pilot
search) for the headline workload: 100M unique uint64 keys from splitmix64(seed=2),
lambda=7.0, alpha=1.0, partition size 2500.  Synthetic data, generated from a seed.

Our arm prints one JSON line with
  value   Mkeys/s over K steps with keys and results resident in HBM, timed with CUDA
          events on the library's own launching stream (max over ranks);
  e2e     the same metric through phobic_build with pinned HOST keys and HOST result
          arrays: every step copies the keys in and the pilots/offsets out;
  roofline  the search kernel (K4, the dominant one): algorithmic integer operations
          (16 per pilot-hash evaluation, 2 per bitmap probe, counted by the oracle on the
          same keys) per second against the device's measured integer peak, with its
          issue rate and HBM figures beside it;
  batched the 4096-set batched build against 4096 plain sequential builds (every set
          compared with its plain build);
  served  a slice of the Poisson request stream, served with continuous batching and
          one request at a time: p50/p99 latency and Mkeys/s;
  cpu_baseline  the oracle port of the reference's pipeline on this host's cores,
          building the same 100M keys.
The reference arm (--impl reference) times that CPU pipeline on the same 100M keys.
Under torchrun every rank builds its own independent key set (weak scaling, no
collective on the data path); rank 0 prints.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import queue
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "phobic-gpu_b200"))

LAMBDA, PSIZE, SEED = 7.0, 2500, 2
METRIC = "Mkeys/s MPHF build @100M u64 keys; p50/p99 latency, batched vs plain"
CONFIG_NAME = "plain build, 100M unique u64 keys splitmix64(seed=2), lambda=7.0, alpha=1.0, partition 2500"


def workload_name(n: int) -> str:
    return CONFIG_NAME if n == 100_000_000 else CONFIG_NAME.replace("100M", f"{n:,}")
# Algorithmic bytes of the search kernel per key: read its (lower1, lower2) record (8 B)
# and bucket id (2 B), write 4 B of pilot per bucket (1/lambda buckets per key).
K4_BYTES_PER_KEY = 8 + 2 + 4 / LAMBDA


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clock and throttle-reason samples during the timed region."""

    Q = ("clocks.sm,clocks.max.sm,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.rows: list[list[str]] = []
        self.proc = None
        self.thread = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=5)

    def summary(self) -> dict:
        sm = [float(r[0]) for r in self.rows if len(r) >= 7 and r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if len(r) >= 7 and r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 7 for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(sm)}


def dist_setup():
    import ranks

    info = ranks.RankInfo.from_env()
    return info.world, info.rank, info.local


def oracle_pipeline(keys, cores: int):
    """One construction by the oracle port (host hash + all stages + search): (s, stats)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import orc  # the oracle: CPU restatement of the reference's construction

    B, f = orc.config(LAMBDA, PSIZE)
    t0 = time.perf_counter()
    r = orc.build(orc.hash_keys(keys, "u64", threads=cores), PSIZE, B, f, threads=cores)
    dt = time.perf_counter() - t0
    assert r["status"] == 0, r["status"]
    return dt, r["stats"]


def cpu_baseline(n: int, min_seconds: float = 10.0, max_reps: int = 12) -> dict:
    """Oracle port of the reference pipeline on all host threads, on the same n keys as
    the GPU arm (seed 2); also returns the search's work counters of that build."""
    import keygen

    keys = keygen.splitmix64(SEED, n)
    cores = os.cpu_count() or 1
    times, stats = [], None
    t_start = time.perf_counter()
    while len(times) < max_reps and (time.perf_counter() - t_start < min_seconds or len(times) < 2):
        dt, stats = oracle_pipeline(keys, cores)
        times.append(dt)
    best = min(times)
    return {"value": n / best / 1e6, "unit": "Mkeys/s", "cores": cores, "kind": "port",
            "sample": f"the whole workload ({n} keys, same seed, lambda, P), {len(times)} runs, best taken",
            "seconds": sum(times),
            "_stats": {"hash_evals": int(stats.hash_evals), "probe_keys": int(stats.probe_keys),
                       "probe_windows": int(stats.probe_words), "k_retries": int(stats.k_retries)}}


def run_reference(args) -> None:
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    import keygen

    n = args.n
    keys = keygen.splitmix64(SEED, n)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        oracle_pipeline(keys, cores)
    times = [oracle_pipeline(keys, cores)[0] for _ in range(args.steps)]
    ms = 1e3 * sum(times) / len(times)
    value = n / (ms / 1e3) / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mkeys/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32", "data": "synthetic (splitmix64 seed 2)",
        "config": {"workload": workload_name(n), "n_keys": n, "lambda": LAMBDA, "alpha": 1.0,
                   "partition_size": PSIZE,
                   "note": "CPU oracle restatement of the reference pipeline (its Vulkan path cannot run here): "
                           "host XXH128 + every stage + pilot search, each step one whole build of the n keys"},
        "cpu_baseline": {"value": value, "unit": "Mkeys/s", "cores": cores, "kind": "port",
                         "sample": f"the whole workload ({n} keys) per step"},
        "e2e": {"value": value, "unit": "Mkeys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args) -> None:
    import torch

    import keygen
    import phobic

    import ranks

    info = ranks.RankInfo.from_env()
    world, rank, local = info.world, info.rank, info.local
    torch.cuda.set_device(local)
    grp = ranks.Group(info, "nccl", device="cuda")

    n = args.n
    cfg = phobic.MPHFconfig(LAMBDA, PSIZE)
    keys = keygen.splitmix64(ranks.rank_seed(SEED, rank), n)  # every rank: its own independent key set
    ctx = phobic.Context(local)
    parts = cfg.partitions(n)
    B = cfg.bucketCountPerPartition

    # ---- device-resident keys and results
    dk = torch.from_numpy(keys.view(np.int64)).cuda()
    dp = torch.empty(parts * B, dtype=torch.int32, device="cuda")
    do = torch.empty(parts + 1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    clocks = ClockSampler(local).__enter__()
    for _ in range(args.warmup):
        ctx.build(dk, cfg, out=(dp, do))
    torch.cuda.synchronize()
    grp.barrier()
    t_start, t_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    search_ms = []
    torch.cuda.synchronize()
    t_start.record(stream)
    for _ in range(args.steps):
        r = ctx.build(dk, cfg, out=(dp, do))
        search_ms.append(r.timings["search"])
    t_end.record(stream)
    torch.cuda.synchronize()
    dev_ms = t_start.elapsed_time(t_end)
    stage = dict(r.timings)
    dev_ms = grp.max(dev_ms)
    ms_per_step = dev_ms / args.steps
    value = world * n / (ms_per_step / 1e3) / 1e6

    # ---- correctness of what was timed: on-device bijection check
    bad = ctx.verify(dk, cfg, phobic.BuildResult(dp, do, parts, B))

    # ---- end to end through the C ABI with pinned host buffers
    hk = torch.from_numpy(keys.view(np.int64)).pin_memory()
    hp = torch.empty(parts * B, dtype=torch.int32).pin_memory()
    ho = torch.empty(parts + 1, dtype=torch.int32).pin_memory()
    hks = phobic.KeySet(phobic.KEYS_U64, n, hk.data_ptr())
    for _ in range(max(1, args.warmup)):
        ctx.build(hks, cfg, out=(hp.data_ptr(), ho.data_ptr()))
    grp.barrier()
    # (a) one build at a time: each step's copy in, kernels and copy out in sequence
    e2e_wall, e2e_dev = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        r2 = ctx.build(hks, cfg, out=(hp.data_ptr(), ho.data_ptr()))
        e2e_wall.append(time.perf_counter() - t0)
        e2e_dev.append(r2.timings["total"])
    single_ms = grp.max(1e3 * sum(e2e_wall) / len(e2e_wall))
    # (b) the same K steps on two contexts (two streams) from two host threads, as a
    # caller with a stream of key sets runs them: one build's host copies overlap the
    # other's kernels.  Every step still copies its keys in and its result out.
    ctx_b = phobic.Context(local)
    hp_b = torch.empty(parts * B, dtype=torch.int32).pin_memory()
    ho_b = torch.empty(parts + 1, dtype=torch.int32).pin_memory()
    for _ in range(max(1, args.warmup)):
        ctx_b.build(hks, cfg, out=(hp_b.data_ptr(), ho_b.data_ptr()))
    lanes = [(ctx, hp, ho, (args.steps + 1) // 2), (ctx_b, hp_b, ho_b, args.steps // 2)]

    def lane_run(c, p_, o_, k):
        for _ in range(k):
            c.build(hks, cfg, out=(p_.data_ptr(), o_.data_ptr()))

    grp.barrier()
    t0 = time.perf_counter()
    th = [threading.Thread(target=lane_run, args=ln) for ln in lanes]
    for t in th:
        t.start()
    for t in th:
        t.join()
    e2e_ms = grp.max(1e3 * (time.perf_counter() - t0) / args.steps)
    clocks.__exit__(None, None, None)
    same = bool((hp.numpy() == dp.cpu().numpy()).all()) and bool((hp_b.numpy() == dp.cpu().numpy()).all())

    # ---- host encoding of the result (Mphf::setData), C2's encoder: interleaved dictionary + diff compact
    built = phobic.BuildResult(hp.numpy().view(np.uint32), ho.numpy().view(np.uint32), parts, B)
    t0 = time.perf_counter()
    blob, bits_per_key = phobic.encode(built, cfg, "interleaved_dictionary", "diff")
    encode_ms = 1e3 * (time.perf_counter() - t0)
    # ---- the compact-vector encoders: on the host, and on the GPU from the device-resident result
    t0 = time.perf_counter()
    blob_c, bpk_c = phobic.encode(built, cfg, "interleaved_compact", "diff")
    encode_compact_ms = 1e3 * (time.perf_counter() - t0)
    dev_built = phobic.BuildResult(dp, do, parts, B)
    phobic.encode_gpu(ctx, dev_built, cfg, "interleaved_compact", "diff")  # warm-up
    gpu_enc = []
    for _ in range(3):
        t0 = time.perf_counter()
        blob_g, bpk_g, _ = phobic.encode_gpu(ctx, dev_built, cfg, "interleaved_compact", "diff")
        gpu_enc.append(1e3 * (time.perf_counter() - t0))
    encode_gpu_ms = min(gpu_enc)

    if rank != 0:
        ctx_b.close()
        ctx.close()
        grp.close()
        return
    peaks = measured_peaks()
    k4_ms = statistics.mean(search_ms)
    hbm_achieved = K4_BYTES_PER_KEY * n / (k4_ms / 1e3) / 1e9
    traffic = None
    tp = ROOT / "profiles" / "k4_traffic.json"
    if tp.exists():
        tr = json.loads(tp.read_text())
        traffic = tr.get("bytes_per_key", 0) * n if tr.get("bytes_per_key") else None
    # Issue-rate view of K4: warp instructions per launch from the ncu capture of the
    # same kernel (per partition, scaled by partitions) over the K4 event time, against
    # 4 schedulers per SM at the SM clock sampled during the timed region.
    issue = None
    ip = ROOT / "profiles" / "k4_issue.json"
    clk = clocks.summary()
    if ip.exists() and clk.get("sm_mhz"):
        per_part = json.loads(ip.read_text())["warp_instructions_per_partition"]
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        inst = per_part * parts
        ach = inst / (k4_ms / 1e3)
        peak_issue = sms * 4 * clk["sm_mhz"] * 1e6
        issue = {"warp_inst_per_launch": inst, "achieved": ach, "peak": peak_issue, "unit": "warp-inst/s",
                 "frac": ach / peak_issue, "sm_count": sms, "sm_mhz": clk["sm_mhz"],
                 "source": "profiles/k4_issue.json (ncu smsp__inst_executed per partition x partitions)"}
    base = cpu_baseline(n) if not args.no_cpu_baseline else None
    # K4's roofline: algorithmic integer operations of the pilot search (the oracle's counts
    # for these very keys: 16 per pilot-hash evaluation H, 2 per bitmap probe Pr of one key's
    # 64-offset window) over the K4 event time, against this device's integer peak for the
    # hash's instruction mix, measured now by the library (phobic_measure_int_peak).
    counts = base.pop("_stats") if base else None
    if counts is None:
        cp = ROOT / "profiles" / "k4_intops.json"
        counts = json.loads(cp.read_text()) if cp.exists() and n == 100_000_000 else None
    int_peak, int_peak_ms = ctx.int_peak()
    roofline = {"kernel": "k_search (K4)", "bound": "issue", "unit": "int-op/s", "peak": int_peak,
                "peak_source": f"measured: phobic_measure_int_peak, {int_peak_ms:.2f} ms kernel, this run",
                "launch_ms": k4_ms, "traffic": traffic, "issue": issue,
                "hbm": {"achieved": hbm_achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": hbm_achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                        "bytes_per_key": K4_BYTES_PER_KEY}}
    if counts:
        int_ops = 16 * counts["hash_evals"] + 2 * counts["probe_keys"]
        roofline.update({"achieved": int_ops / (k4_ms / 1e3), "frac": int_ops / (k4_ms / 1e3) / int_peak,
                         "int_ops_per_launch": int_ops, "hash_evals": counts["hash_evals"],
                         "probe_keys": counts["probe_keys"], "formula": "16*hash_evals + 2*probe_keys"})
    extra = {}
    if world == 1 and not args.no_extra:
        ctx_b.close()
        extra["batched"] = c4_leg(args)
        extra["served"] = c5_leg(args, args.served_seconds)
    line = {
        "metric": METRIC, "value": value, "unit": "Mkeys/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (splitmix64 seed 2 + rank)",
        "config": {"workload": workload_name(n), "n_keys": n, "lambda": LAMBDA, "alpha": 1.0, "partition_size": PSIZE,
                   "buckets_per_partition": B, "partitions": parts, "parallelism": f"replicas x{world}",
                   "l2": f"inputs larger than L2 ({8 * n / 1e6:,.0f} MB keys per step)" if 8 * n > 126e6
                   else f"inputs smaller than L2 ({8 * n / 1e6:,.0f} MB keys per step)"},
        "stages_ms": {k: round(v, 4) for k, v in stage.items() if k != "kernels"},
        "bijection_bad": bad, "host_result_equals_device": same,
        "gpu_launches": int(stage["kernels"]) * args.steps,
        "e2e": {"value": world * n / (e2e_ms / 1e3) / 1e6, "unit": "Mkeys/s", "h2d_bytes_per_step": 8 * n,
                "d2h_bytes_per_step": 4 * (parts * B + parts + 1), "ms_per_step": e2e_ms,
                "how": "phobic_build with pinned host keys and results, K steps on two contexts from two host "
                       "threads (copies of one build overlap the other's kernels); wall clock",
                "single": {"value": world * n / (single_ms / 1e3) / 1e6, "ms_per_step": single_ms,
                           "device_ms_per_step": statistics.mean(e2e_dev),
                           "how": "one build at a time on one context"}},
        "roofline": roofline,
        **extra,
        "encoding": {"encoder": "interleaved<dictionary> + diff<compact>", "ms": encode_ms,
                     "bits_per_key": bits_per_key, "bytes": len(blob), "host_threads": os.cpu_count(),
                     "e2e_with_encoding_mkeys_s": world * n / ((e2e_ms + encode_ms) / 1e3) / 1e6},
        "encoding_compact": {"encoder": "interleaved<compact> + diff<compact>", "host_ms": encode_compact_ms,
                             "gpu_ms": encode_gpu_ms, "gpu_bytes_equal_host": blob_g == blob_c,
                             "bits_per_key": bpk_g, "bytes": len(blob_g),
                             "note": "gpu_ms: phobic_encode_gpu from the device-resident result, bytes copied to "
                                     "host memory (wall clock, best of 3)"},
        "cpu_baseline": base,
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)
    if not extra:
        ctx_b.close()
    ctx.close()
    grp.close()


# ------------------------------------------------------------------ other workloads

def _plain_device_ms(ctx, keys_dev, cfg, steps, warmup, torch, kind=None):
    """Mean device time of a plain build with device-resident keys and results (CUDA events)."""
    import phobic

    ks = phobic.keyset(keys_dev, kind)
    parts = cfg.partitions(ks.n)
    dp = torch.empty(max(parts * cfg.bucketCountPerPartition, 1), dtype=torch.int32, device="cuda")
    do = torch.empty(parts + 1, dtype=torch.int32, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    for _ in range(warmup):
        r = ctx.build(ks, cfg, out=(dp, do))
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record(stream)
    for _ in range(steps):
        r = ctx.build(ks, cfg, out=(dp, do))
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / steps, r.timings, phobic.BuildResult(dp, do, parts, cfg.bucketCountPerPartition)


def run_plain_workload(args, name, lam, P, make_keys, describe) -> None:
    """C1 / C3: a plain build of one key set (device-resident value, host e2e)."""
    import torch

    import phobic

    cfg = phobic.MPHFconfig(lam, P)
    host_keys, kind = make_keys()
    ctx = phobic.Context(0)
    if kind == phobic.KEYS_STRINGS:
        data, offs = host_keys
        dev = (torch.from_numpy(data).cuda(), torch.from_numpy(offs.view(np.int64)).cuda())
        pinned = (torch.from_numpy(data).pin_memory(), torch.from_numpy(offs.view(np.int64)).pin_memory())
        n = len(offs) - 1
        dev_ks = phobic.KeySet(kind, n, dev[0], dev[1], True)
        host_ks = phobic.KeySet(kind, n, pinned[0].data_ptr(), pinned[1].data_ptr())
        h2d = int(offs[-1]) + 8 * (n + 1)
    else:
        n = len(host_keys)
        dev_ks = phobic.KeySet(kind, n, torch.from_numpy(host_keys.view(np.int64)).cuda(), None, True)
        pinned = torch.from_numpy(host_keys.view(np.int64)).pin_memory()
        host_ks = phobic.KeySet(kind, n, pinned.data_ptr())
        h2d = 8 * n
    ms, stages, built = _plain_device_ms(ctx, dev_ks, cfg, args.steps, args.warmup, torch)
    bad = ctx.verify(dev_ks, cfg, built)
    parts = cfg.partitions(n)
    hp = torch.empty(max(parts * cfg.bucketCountPerPartition, 1), dtype=torch.int32).pin_memory()
    ho = torch.empty(parts + 1, dtype=torch.int32).pin_memory()
    ctx.build(host_ks, cfg, out=(hp.data_ptr(), ho.data_ptr()))
    wall = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ctx.build(host_ks, cfg, out=(hp.data_ptr(), ho.data_ptr()))
        wall.append(time.perf_counter() - t0)
    e2e_ms = 1e3 * statistics.mean(wall)
    print(json.dumps({
        "workload": name, "metric": "Mkeys/s MPHF build", "value": n / ms / 1e3, "unit": "Mkeys/s",
        "ms_per_step": ms, "steps": args.steps, "warmup": args.warmup, "config": describe, "n_keys": n,
        "stages_ms": {k: round(v, 4) for k, v in stages.items() if k != "kernels"}, "bijection_bad": bad,
        "e2e": {"value": n / e2e_ms / 1e3, "unit": "Mkeys/s", "ms_per_step": e2e_ms, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 4 * (parts * cfg.bucketCountPerPartition + parts + 1)},
    }), flush=True)
    ctx.close()


def c4_leg(args) -> dict:
    """Batched build: 4096 u64 key sets, sizes log-uniform in [1K, 4M] (seed 4), lambda 6,
    P 2048, all sets in one batch vs 4096 plain sequential builds on the same GPU.  Every
    set's batched result is compared with its plain build."""
    import torch

    import keygen
    import phobic

    lam, P = 6.0, 2048
    cfg = phobic.MPHFconfig(lam, P)
    B = cfg.bucketCountPerPartition
    sizes = keygen.set_sizes(4, args.c4_sets, 1000, 4 << 20)
    total = int(sizes.sum())
    keys = keygen.splitmix64_cuda(4, total)  # one stream split into the sets: unique keys
    starts = np.concatenate([[0], np.cumsum(sizes)])
    sets = [keys[int(starts[i]):int(starts[i + 1])] for i in range(len(sizes))]
    parts = [cfg.partitions(int(n)) for n in sizes]
    pstart = np.concatenate([[0], np.cumsum([B * m for m in parts])])
    ostart = np.concatenate([[0], np.cumsum([m + 1 for m in parts])])
    flat = {mode: (torch.empty(int(pstart[-1]), dtype=torch.int32, device="cuda"),
                   torch.empty(int(ostart[-1]), dtype=torch.int32, device="cuda")) for mode in ("batched", "plain")}

    def outs(mode):
        fp, fo = flat[mode]
        return [(fp[int(pstart[i]):int(pstart[i + 1])], fo[int(ostart[i]):int(ostart[i + 1])]) for i in range(len(sets))]

    ctx = phobic.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    ob, op = outs("batched"), outs("plain")
    fp, fo = flat["batched"]
    phobic.build_batch_flat(ctx, keys, sizes, cfg, fp, fo)  # warm-up: grows the arena
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, _, st, timings = phobic.build_batch_flat(ctx, keys, sizes, cfg, fp, fo)
    batch_wall = time.perf_counter() - t0
    batch_dev = timings["total"]
    assert (st == 0).all(), st
    for k, o in zip(sets[:8], op[:8]):  # warm-up of the plain path
        ctx.build(k, cfg, out=o)
    lat = []
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    a.record(stream)
    for k, o in zip(sets, op):
        t1 = time.perf_counter()
        ctx.build(k, cfg, out=o)
        lat.append(1e3 * (time.perf_counter() - t1))
    b.record(stream)
    torch.cuda.synchronize()
    seq_wall = time.perf_counter() - t0
    seq_dev = a.elapsed_time(b)
    same = bool(torch.equal(flat["batched"][0], flat["plain"][0])) and bool(torch.equal(flat["batched"][1],
                                                                                       flat["plain"][1]))
    bad = sum(ctx.verify(sets[i], cfg, phobic.BuildResult(ob[i][0], ob[i][1], parts[i], B))
              for i in range(0, len(sets), max(1, len(sets) // 64)))
    ctx.close()
    del keys, sets, flat, ob, op
    torch.cuda.empty_cache()
    return {
        "workload": "batched build, 4096 u64 key sets log-uniform in [1e3, 4*2^20] (seed 4), lambda 6, P 2048",
        "sets": len(sizes), "total_keys": total,
        "mkeys_per_s": total / batch_wall / 1e6, "wall_ms": 1e3 * batch_wall, "device_ms": batch_dev,
        "kernel_launches": timings["kernels"],
        "plain": {"mkeys_per_s": total / seq_wall / 1e6, "wall_ms": 1e3 * seq_wall, "device_ms": seq_dev,
                  "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                  "kernel_launches": 6 * len(sizes), "how": "4096 phobic_build calls in sequence, one context"},
        "speedup_vs_plain": seq_wall / batch_wall,
        "all_sets_equal_plain": same, "bijection_bad_sample_of_64": bad,
        "how": "one phobic_build_batch call through phobic.build_batch_flat (wall clock; device_ms from its "
               "events), keys and results on the device",
    }


def c5_leg(args, seconds: float) -> dict:
    """Served stream: Poisson arrivals at 200 req/s, sizes log-uniform in [1e4, 5e7], 70 % u64 /
    30 % strings (seed 5), lambda 7, P 2048, device budget 120 GB; continuous batching on
    several streams vs plain one-at-a-time builds (one stream, no batching) of the same stream."""
    import torch

    import keygen
    import phobic

    lam, P = 7.0, 2048
    cfg = phobic.MPHFconfig(lam, P)
    times, sizes, kinds = keygen.request_stream(5, 200.0, seconds, 1e4, args.c5_max, 0.3)
    rng = np.random.default_rng(55)
    u64_pool = keygen.splitmix64_cuda(5, int(sizes.max()))
    n_str = int(sizes[kinds == "strings"].max()) if (kinds == "strings").any() else 1
    sdata, soffs = keygen.strings_cuda(5, n_str)
    reqs = []
    for t, n, k in zip(times, sizes, kinds):
        n = int(n)
        if k == "u64":
            a = int(rng.integers(0, len(u64_pool) - n + 1))
            reqs.append((t, phobic.KeySet(phobic.KEYS_U64, n, u64_pool[a:a + n], None, True)))
        else:
            a = int(rng.integers(0, n_str - n + 1))
            reqs.append((t, phobic.KeySet(phobic.KEYS_STRINGS, n, sdata, soffs[a:a + n + 1], True)))
    total = int(sizes.sum())
    # Both modes size their streams up front for the largest request of the stream, so that
    # no arena grows (a free and a reallocation that waits for the device) while serving.
    largest = [max((ks for (_, ks), k in zip(reqs, kinds) if k == kk), key=lambda ks: ks.n)
               for kk in ("u64", "strings") if (kinds == kk).any()]
    need = [phobic.Server.bytes_for(ks, cfg) for ks in largest]
    reserve = (max(d for d, _ in need), max(p for _, p in need))

    def replay(streams, max_batch):
        outs, statuses = [], []
        with phobic.Server(0, streams=streams, budget_bytes=120 << 30, max_batch_sets=max_batch) as srv:
            srv.reserve(*reserve)
            tickets = queue.Queue()

            def consume():  # results are hashed and dropped as they complete
                for _ in reqs:
                    st, r = srv.wait(tickets.get())
                    statuses.append(st)
                    outs.append(hashlib.sha1(np.ascontiguousarray(r.pilots).tobytes()).hexdigest() if st == 0 else None)

            waiter = threading.Thread(target=consume)
            waiter.start()
            t0 = time.perf_counter()
            for t, ks in reqs:
                delay = t - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                tickets.put(srv.submit(ks, cfg))
            waiter.join()
            wall = time.perf_counter() - t0
            stats = srv.stats()
        failed = {int(k): int(v) for k, v in zip(*np.unique([x for x in statuses if x], return_counts=True))}
        return outs, wall, stats, failed

    served, s_wall, s_stats, s_failed = replay(4, 0)
    plain, p_wall, p_stats, p_failed = replay(1, 1)
    same = served == plain and not s_failed and not p_failed
    del u64_pool, sdata, soffs, reqs
    torch.cuda.empty_cache()

    def summary(wall, st, failed):
        return {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "max_ms": st["max_ms"],
                "mkeys_per_s": total / (st["busy_ms"] / 1e3) / 1e6, "busy_s": st["busy_ms"] / 1e3, "wall_s": wall,
                "peak_device_bytes": st["peak_bytes"], "max_batch_requests": st["max_batch_requests"],
                "max_batches_in_flight": st["max_batches_in_flight"],
                "max_device_overlap": st["max_device_overlap"], "failed_by_status": failed}

    return {
        "workload": f"served build stream, Poisson 200 req/s for {seconds:g} s (seed 5), sizes log-uniform "
                    f"[1e4, {args.c5_max:.0e}], 70 % u64 / 30 % 8-64-byte strings, lambda 7, P 2048, 120 GB budget",
        "requests": len(times), "total_keys": total,
        "string_requests": int((kinds == "strings").sum()),
        **summary(s_wall, s_stats, s_failed),
        "how": "4 streams, continuous batching (phobic_server); results copied to host memory; mkeys_per_s over "
               "the time with a request in flight",
        "plain": {**summary(p_wall, p_stats, p_failed), "how": "1 stream, one request per build"},
        "results_identical": same,
        "reserved_per_stream": {"device_bytes": reserve[0], "pinned_bytes": reserve[1]},
    }


def run_c4(args) -> None:
    print(json.dumps(c4_leg(args)), flush=True)


def run_c5(args) -> None:
    r = c5_leg(args, args.c5_seconds)
    print(json.dumps(r), flush=True)
    if r["failed_by_status"] or r["plain"]["failed_by_status"]:
        sys.exit(1)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=100_000_000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extra", action="store_true", help="skip the batched and served legs of the headline line")
    ap.add_argument("--served-seconds", type=float, default=20.0, help="slice of the request stream in the line")
    ap.add_argument("--workload", choices=["c1", "c2", "c3", "c4", "c5"], default="c2")
    ap.add_argument("--c4-sets", type=int, default=4096)
    ap.add_argument("--c5-seconds", type=float, default=60.0)
    ap.add_argument("--c5-max", type=float, default=5e7)
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "c2":
        run_ours(args)
    elif args.workload == "c1":
        import keygen
        import phobic
        run_plain_workload(args, "C1", 5.0, 2048, lambda: (keygen.splitmix64(1, 1_000_000), phobic.KEYS_U64),
                           "1M u64 splitmix64(seed=1), lambda 5, P 2048")
    elif args.workload == "c3":
        import keygen
        import phobic
        run_plain_workload(args, "C3", 6.0, 2048, lambda: (keygen.strings(3, args.n if args.n != 100_000_000 else 50_000_000),
                                                           phobic.KEYS_STRINGS),
                           "50M strings, length U[8,64], printable ASCII, seed 3, lambda 6, P 2048")
    elif args.workload == "c4":
        run_c4(args)
    else:
        run_c5(args)


if __name__ == "__main__":
    main()
