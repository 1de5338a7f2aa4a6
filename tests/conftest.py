import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "info-centric_ge_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (PKG, os.path.join(ROOT, "tests"), GOLDEN):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    gpu = os.path.join(PKG, "felog_b200", "libfelog_gpu.so")
    tools = os.path.join(PKG, "felog_b200", "libfelog_tools.so")
    if not (os.path.exists(gpu) and os.path.exists(tools)):
        subprocess.check_call(["make", "-s", "-C", PKG])
    orc = os.path.join(ROOT, "oracle", "_build", "liboracle.so")
    if not os.path.exists(orc):
        subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "port"])


_ensure_built()


def load_golden(name):
    return dict(np.load(os.path.join(GOLDEN, name)))


@pytest.fixture
def golden():
    return load_golden


def walk_draws(fx, r):
    """Injected draw streams of round r of a walk fixture (p as exact doubles)."""
    p = fx[f"r{r}_p"].astype(np.float64) / 2147483647.0
    return (fx[f"r{r}_idx_off"], fx[f"r{r}_idx"], fx[f"r{r}_p_off"], p)
