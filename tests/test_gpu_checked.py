"""The bounds-checked build of the library (every shared- and global-memory index on
the kernels' paths checked; a failed check is recorded, never a fault): parity
builds of several sizes, configurations, key kinds and a batch run on it in a
separate process, and no check may fail."""
import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
pytestmark = pytest.mark.gpu


def test_checked_library_parity_and_no_failed_check():
    lib = ROOT / "phobic-gpu_b200" / "lib" / "libphobic_b200_checked.so"
    if not lib.exists():
        sys.path.insert(0, str(ROOT / "phobic-gpu_b200"))
        import build

        build.build(checked=True)
    env = dict(os.environ, PHOBIC_LIBRARY="checked")
    out = subprocess.run([sys.executable, str(ROOT / "tests" / "checked_runs.py")], env=env, capture_output=True,
                         text=True, timeout=900)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "failed check lines (map, partition, search): [0, 0, 0]" in out.stdout


def test_normal_library_reports_no_checks(phobic, ctx):
    compiled, lines = ctx.checks()
    assert not compiled and lines == [0, 0, 0]
