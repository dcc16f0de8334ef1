import os
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
PKG = ROOT / "nim-conv22-shared_b200"
for p in (str(PKG), str(ROOT / "oracle"), str(ROOT)):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def _built():
    return ((PKG / "lib" / "libnim_host.so").exists() and (ROOT / "oracle" / "_build" / "libnim_oracle.so").exists())


@pytest.fixture(scope="session", autouse=True)
def _build_libs():
    """Build the host library and the oracle when they are missing (CPU
    only; the CUDA library is built by __graft_entry__.build())."""
    if not _built():
        env = dict(os.environ)
        env.pop("CXX", None)
        env.pop("CC", None)
        subprocess.run(["make", "-C", str(PKG), "host"], check=True, env=env)
        subprocess.run(["make", "-C", str(ROOT / "oracle")], check=True, env=env)
    yield
