"""The C ABI library without a GPU: it loads, exports every symbol that
include/phobic_b200.h declares, and its host-side arithmetic (MPHFconfig)
matches the reference's tables.  No compute call is made here."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "phobic_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"PHOBIC_API[^;(]*?\b(phobic_\w+)\s*\(", text, flags=re.S)))


def test_header_declares_the_abi():
    syms = declared_symbols()
    assert "phobic_build" in syms and "phobic_server_submit" in syms and len(syms) >= 20


def test_library_exports_every_declared_symbol(phobic):
    out = subprocess.run(["nm", "-D", "--defined-only", str(phobic.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r" T (phobic_\w+)", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    lib = phobic.lib()
    for s in declared_symbols():
        assert getattr(lib, s) is not None


def test_build_recipe_targets_sm100a():
    """The recipe compiles every kernel for sm_100a only (the GPU test
    test_kernels_report_sm100 reads the same fact back through the runtime)."""
    import importlib.util

    spec = importlib.util.spec_from_file_location("phobic_build_recipe", ROOT / "phobic-gpu_b200" / "build.py")
    recipe = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(recipe)
    assert recipe.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert recipe.NVCC_FLAGS[:2] == recipe.ARCH


def test_config_matches_reference_tables(phobic, golden, golden_fulcrums):
    for name, meta in golden["fulcrums"].items():
        cfg = phobic.MPHFconfig(meta["lambda"], meta["P"], meta["bucketer"], bool(meta["bucketer_ctor"]))
        assert cfg.bucketCountPerPartition == meta["buckets"], name
        assert (cfg.getFulcs() == golden_fulcrums[name]).all(), name
        assert cfg.partitionMaxSize() == meta["partition_max_size"]
        assert cfg.params.max_partition_size == 32 * (meta["partition_max_size"] // 32)


def test_config_rejects_bad_arguments(phobic):
    p = phobic.Params()
    lib = phobic.lib()
    assert lib.phobic_config(0.0, 2048, 0, 0, C.byref(p)) == phobic.ERR_INVALID
    assert lib.phobic_config(5.0, 0, 0, 0, C.byref(p)) == phobic.ERR_INVALID
    assert lib.phobic_config(5.0, 2048, 7, 0, C.byref(p)) == phobic.ERR_INVALID
    assert lib.phobic_config(1e-9, 2048, 0, 0, C.byref(p)) == phobic.ERR_INVALID  # buckets > 65535


def test_partitions_formula(phobic):
    lib = phobic.lib()
    for n, P, want in [(0, 2048, 0), (1, 2048, 1), (2048, 2048, 1), (2049, 2048, 2), (100_000_000, 2500, 40000)]:
        assert lib.phobic_partitions(n, P) == want


def test_status_strings(phobic):
    lib = phobic.lib()
    for s in range(14):
        assert lib.phobic_status_string(s) and lib.phobic_status_string(s) != b"unknown status"
    assert lib.phobic_status_string(phobic.ERR_KEYS_CHANGED) == b"keys changed during the build"
    assert lib.phobic_status_string(999) == b"unknown status"


def test_null_context_is_rejected(phobic):
    lib = phobic.lib()
    cfg = phobic.MPHFconfig(5.0, 2048)
    k = phobic.Keys(phobic.KEYS_U64, 0, 0, None, None)
    r = phobic.Result(0, None, None)
    assert lib.phobic_build(None, C.byref(k), C.byref(cfg.params), C.byref(r), None) == phobic.ERR_INVALID


def test_bytes_needed_formula(phobic):
    cfg = phobic.MPHFconfig(7.0, 2500)
    lib = phobic.lib()
    k = phobic.Keys(phobic.KEYS_U64, 1, 100_000_000, None, None)
    need = lib.phobic_build_bytes_needed(C.byref(k), C.byref(cfg.params))
    # device-resident u64 keys: lowers 8 + bucket ids 2 + partition records 16 bytes per key, plus the
    # (partition, chunk) count matrix and its prefix, pilots and offsets
    assert 26e8 < need < 28e8


def test_context_without_device_fails_loudly(phobic):
    try:
        import torch

        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(phobic.PhobicError) as e:
        phobic.Context(0)
    assert e.value.status == phobic.ERR_NO_DEVICE


def test_shipped_tuning_table_is_well_formed(phobic):
    """phobic-gpu_b200/tuning.tsv (written by phobic_autotune on a B200): tab-separated lines
    of device, P, B, partition capacity, size class, search shape (warps, bucket pipeline)
    and the measured build times of the six timed shapes; for every parameter set the
    classes ascend and the chosen shape is the fastest measured one."""
    shapes = [(1, 0), (2, 0), (4, 0), (2, 1), (4, 1), (8, 1)]
    table = ROOT / "phobic-gpu_b200" / "tuning.tsv"
    rows = [l.split("\t") for l in table.read_text().splitlines() if l and not l.startswith("#")]
    assert rows
    groups = {}
    for r in rows:
        assert len(r) == 7 + len(shapes), r
        dev, P, B, cap, cls, group, pipe = r[0], *map(int, r[1:7])
        ms = [float(x) for x in r[7:]]
        assert (group, pipe) in shapes
        assert ms[shapes.index((group, pipe))] == min(ms), r
        cfg = None
        for lam in (4.5, 5.0, 6.0, 7.0, 7.5):
            c = phobic.MPHFconfig(lam, P)
            if c.bucketCountPerPartition == B:
                cfg = c
        assert cfg is not None and cfg.params.max_partition_size == cap, r
        groups.setdefault((dev, P, B, cap), []).append(cls)
    for key, classes in groups.items():
        assert classes == sorted(classes) and len(set(classes)) == len(classes), key
