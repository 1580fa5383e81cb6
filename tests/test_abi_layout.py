"""The ctypes mirrors in phobic.py have the layout of the C ABI's structs.

A small C program, compiled with gcc against include/phobic_b200.h, prints the size and the
offset of every field of each struct the binding passes by pointer; the ctypes classes must
agree field by field, so a field added to the header (timings, tuning, server stats) cannot
leave the Python binding reading the wrong bytes.  No GPU and no library load is needed."""
import ctypes as C
import shutil
import subprocess

import pytest

from conftest import PKG, ROOT

# C struct -> (ctypes class name in phobic.py, C field names in order; arrays by name)
STRUCTS = {
    "phobic_params": ("Params", ["partition_size", "buckets", "max_partition_size", "max_pilot_counter", "fulcrums"]),
    "phobic_keys": ("Keys", ["kind", "on_device", "n", "data", "offsets"]),
    "phobic_result": ("Result", ["on_device", "pilots", "partition_offsets"]),
    "phobic_timings": ("Timings", ["input_transfer", "bucket_sizes", "partition_offsets", "key_redistribution",
                                   "search", "result_transfer", "total", "kernels", "graph_replays"]),
    "phobic_tuning": ("Tuning", ["search_group", "search_pipeline", "graphs_off", "reserved"]),
    "phobic_server_config": ("ServerConfig", ["device", "streams", "queue_capacity", "max_batch_sets",
                                              "budget_bytes"]),
    "phobic_server_stats": ("ServerStats", ["completed", "failed", "keys", "p50_ms", "p99_ms", "max_ms", "busy_ms",
                                            "peak_bytes", "max_batch_requests", "max_batches_in_flight",
                                            "max_device_overlap", "pad"]),
}


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    if shutil.which("gcc") is None:
        pytest.skip("gcc not found")
    d = tmp_path_factory.mktemp("abi")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "phobic_b200.h"', "int main(void) {"]
    for struct, (_, fields) in STRUCTS.items():
        lines.append(f'    printf("{struct} sizeof %zu\\n", sizeof({struct}));')
        for f in fields:
            lines.append(f'    printf("{struct} {f} %zu\\n", offsetof({struct}, {f}));')
    lines += ["    return 0;", "}"]
    src = d / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = d / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    table = {}
    for line in out.splitlines():
        struct, field, value = line.split()
        table[(struct, field)] = int(value)
    return table


def _binding():
    import sys

    sys.path.insert(0, str(PKG))
    import phobic

    return phobic


@pytest.mark.parametrize("struct", sorted(STRUCTS))
def test_ctypes_mirror_matches_the_header(c_layout, struct):
    phobic = _binding()
    cls_name, fields = STRUCTS[struct]
    cls = getattr(phobic, cls_name)
    assert [name for name, _ in cls._fields_] == fields, f"{cls_name} fields differ from {struct}"
    assert C.sizeof(cls) == c_layout[(struct, "sizeof")], f"sizeof({struct})"
    for f in fields:
        assert getattr(cls, f).offset == c_layout[(struct, f)], f"offsetof({struct}, {f})"
