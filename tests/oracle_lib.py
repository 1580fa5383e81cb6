"""The oracle's ctypes wrapper (oracle/orc.py), re-exported for the tests."""
import sys
from pathlib import Path

sys.path.insert(0, str(Path(__file__).resolve().parents[1] / "oracle"))

from orc import *  # noqa: E402,F401,F403
