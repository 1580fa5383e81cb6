"""Multi-rank logic on CPU: two gloo ranks as separate processes (no GPU).

Covers what bench.py and a sharded build rely on: the max over ranks of a
timing, barriers, distinct per-rank key sets, disjoint covering shards, and a
rank that raises is reported by its peers' short process-group timeout instead of
hanging them."""
import os
import socket
import subprocess
import sys
import textwrap
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "phobic-gpu_b200"


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(body: str, world: int = 2, timeout: float = 120) -> list[subprocess.CompletedProcess]:
    port = free_port()
    code = textwrap.dedent(f"""
        import sys
        sys.path.insert(0, {str(PKG)!r})
        import ranks
        info = ranks.RankInfo.from_env()
    """) + textwrap.dedent(body)
    procs = []
    for r in range(world):
        env = dict(os.environ, WORLD_SIZE=str(world), RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port), CUDA_VISIBLE_DEVICES="")
        procs.append(subprocess.Popen([sys.executable, "-c", code], env=env, stdout=subprocess.PIPE,
                                      stderr=subprocess.PIPE, text=True))
    out = []
    for p in procs:
        try:
            so, se = p.communicate(timeout=timeout)
        except subprocess.TimeoutExpired:
            p.kill()
            so, se = p.communicate()
        out.append(subprocess.CompletedProcess(p.args, p.returncode, so, se))
    return out


def test_max_and_sum_over_two_gloo_ranks():
    res = run_ranks("""
        g = ranks.Group(info, "gloo", timeout_s=30)
        g.barrier()
        print("max", g.max(10.0 + 5 * info.rank), "sum", g.sum(1 + info.rank))
        g.close()
    """)
    for r in res:
        assert r.returncode == 0, r.stderr
        assert "max 15.0 sum 3.0" in r.stdout


def test_ranks_build_distinct_key_sets():
    res = run_ranks("""
        import numpy as np, keygen
        g = ranks.Group(info, "gloo", timeout_s=30)
        k = keygen.splitmix64(ranks.rank_seed(2, info.rank), 1000)
        # the two ranks' sets share no key
        other = keygen.splitmix64(ranks.rank_seed(2, 1 - info.rank), 1000)
        print("overlap", len(np.intersect1d(k, other)), "first", int(k[0]))
        g.close()
    """)
    firsts = set()
    for r in res:
        assert r.returncode == 0, r.stderr
        assert "overlap 0" in r.stdout
        firsts.add(r.stdout.split("first")[1].strip())
    assert len(firsts) == 2


def test_a_failing_rank_ends_its_peer_with_an_error():
    """Rank 1 raises before the barrier; rank 0's barrier ends by the group timeout."""
    res = run_ranks("""
        g = ranks.Group(info, "gloo", timeout_s=5)
        if info.rank == 1:
            raise SystemExit(3)
        try:
            g.barrier()
            print("barrier passed")
        except Exception as e:
            print("peer failure detected:", type(e).__name__)
    """, timeout=90)
    assert res[1].returncode == 3
    assert "peer failure detected" in res[0].stdout or res[0].returncode != 0


def test_shard_ranges_are_disjoint_and_cover():
    sys.path.insert(0, str(PKG))
    import ranks

    for n in (0, 1, 7, 1000, 10**8 + 3):
        for world in (1, 2, 3, 8):
            spans = [ranks.shard_range(n, world, r) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert max(h - l for l, h in spans) - min(h - l for l, h in spans) <= 1
    with pytest.raises(ValueError):
        ranks.shard_range(10, 2, 2)


def test_reference_arm_under_two_ranks_prints_once():
    """bench.py --impl reference: rank 0 times the CPU port and prints one line; rank 1 exits 0."""
    port = free_port()
    outs = []
    for r in range(2):
        env = dict(os.environ, WORLD_SIZE="2", RANK=str(r), LOCAL_RANK=str(r), MASTER_ADDR="127.0.0.1",
                   MASTER_PORT=str(port))
        outs.append(subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2",
                                    "--steps", "1", "--warmup", "0", "--n", "20000"], env=env,
                                   capture_output=True, text=True, timeout=300))
    assert all(o.returncode == 0 for o in outs), [o.stderr for o in outs]
    assert outs[1].stdout.strip() == ""
    import json

    line = json.loads(outs[0].stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["e2e"]["h2d_bytes_per_step"] == 0
