import json
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "phobic-gpu_b200"
GOLDEN = ROOT / "tests" / "golden"
sys.path.insert(0, str(PKG))
sys.path.insert(0, str(ROOT / "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels through the C ABI")


@pytest.fixture(scope="session")
def golden():
    return json.loads((GOLDEN / "golden.json").read_text())


@pytest.fixture(scope="session")
def golden_fulcrums():
    return dict(np.load(GOLDEN / "fulcrums.npz"))


@pytest.fixture(scope="session")
def small_builds():
    return dict(np.load(GOLDEN / "small_builds.npz"))


@pytest.fixture(scope="session")
def phobic():
    """The product binding; the library is built from source when missing."""
    lib = PKG / "lib" / "libphobic_b200.so"
    if not lib.exists():
        subprocess.run([sys.executable, str(PKG / "build.py")], check=True)
    import phobic as ph

    return ph


@pytest.fixture(scope="session")
def ctx(phobic):
    c = phobic.Context(0)
    yield c
    c.close()
