"""Shared test set-up: import paths, build of the native libraries, the `gpu` marker."""
from __future__ import annotations

import os
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "cell-fluid-structure-analysis_b200"
ORACLE = ROOT / "oracle"
for p in (PKG, ORACLE, ROOT):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")
    for d in (PKG, ORACLE):
        lib = d / "lib"
        if not lib.exists() or not any(lib.glob("*.so")):
            subprocess.run(["make", "-s", "-C", str(d)], check=True)


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def cf():
    import cfsa_b200

    return cfsa_b200


@pytest.fixture(scope="session")
def po():
    import pyoracle

    return pyoracle


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
