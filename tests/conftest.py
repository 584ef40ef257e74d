"""Shared test set-up.

Markers: ``gpu`` -- needs a CUDA device (run on a B200); everything else runs
on the CPU.  The product binding (ehd-convection-3d_b200/ehd.py) and the
oracle (oracle/oracle.py) are loaded by path.
"""
import importlib.util
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "ehd-convection-3d_b200"
GOLDEN = ROOT / "tests" / "golden"

sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(GOLDEN))


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


ehd = _load("ehd", PKG / "ehd.py")
fno = _load("ehd_fno_binding", PKG / "fno.py")
import oracle as O  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def golden(name):
    return np.load(GOLDEN / f"{name}.npz")


def golden_params(g):
    return json.loads(str(g["params"]))


def relerr(a, b):
    """max |a - b| / max |b|: the per-field max-norm relative error."""
    s = np.abs(b).max()
    return float(np.abs(a - b).max() / (s if s > 0 else 1.0))


@pytest.fixture(scope="session")
def oracle_mod():
    return O


@pytest.fixture(scope="session")
def ehd_mod():
    return ehd
