"""Build recipe for libphobic_b200.so (CUDA kernels for sm_100a + the C ABI).

Run as ``python phobic-gpu_b200/build.py`` or through ``__graft_entry__.build()``.
Objects go to ``phobic-gpu_b200/_build/``, the library to ``phobic-gpu_b200/lib/``;
both stay in the source tree so that the built library travels with it.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
OBJ = PKG / "_build"
LIB = PKG / "lib" / "libphobic_b200.so"
# The bounds-checked variant (-DPHOBIC_CHECKED): kernels check their indexes and
# record the first failing check instead of making the access.
OBJ_CHECKED = PKG / "_build_checked"
LIB_CHECKED = PKG / "lib" / "libphobic_b200_checked.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
    "-Xcompiler", "-fPIC,-O3,-ffp-contract=off,-fvisibility=hidden,-fopenmp",
    "-Xptxas", "-O3",
    f"-I{ROOT / 'include'}", f"-I{CSRC}", f"-I{PKG / 'cpp'}",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return [*CSRC.glob("*.cuh"), *CSRC.glob("*.hpp"), *(PKG / "cpp").rglob("*.hpp"), *(ROOT / "include").glob("*.h")]


def _stale(obj: Path, src: Path, newest_header: float) -> bool:
    return not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, newest_header)


def _compile(src: Path, extra: list[str], objdir: Path = OBJ) -> Path:
    obj = objdir / (src.stem + ".o")
    cmd = [nvcc(), *NVCC_FLAGS, *extra, "-c", str(src), "-o", str(obj)]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{res.stderr}")
    if extra and res.stderr:
        print(res.stderr, end="")
    return obj


def build(verbose: bool = False, force: bool = False, ptxas_verbose: bool = False, checked: bool = False) -> Path:
    objdir, lib = (OBJ_CHECKED, LIB_CHECKED) if checked else (OBJ, LIB)
    objdir.mkdir(exist_ok=True)
    lib.parent.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cpp"))
    newest = max((h.stat().st_mtime for h in _headers()), default=0.0)
    todo = [s for s in sources if force or _stale(objdir / (s.stem + ".o"), s, newest)]
    extra = (["-Xptxas", "-v"] if ptxas_verbose else []) + (["-DPHOBIC_CHECKED"] if checked else [])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for obj in ex.map(lambda s: _compile(s, extra, objdir), todo):
            if verbose:
                print("compiled", obj.name)
    objs = [objdir / (s.stem + ".o") for s in sources]
    if todo or not lib.exists() or lib.stat().st_mtime < max(o.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lpthread", "-lgomp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
        if verbose:
            print("linked", lib)
    return lib


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_verbose="--ptxas" in sys.argv,
          checked="--checked" in sys.argv)
