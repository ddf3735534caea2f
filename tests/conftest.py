"""Shared test setup.

The engine package lives in the directory ``galaxy-collision-simulation_b200`` (not an
importable identifier); it is loaded here once under the module name ``gx`` so tests can
``import gx``.  GPU tests carry ``@pytest.mark.gpu``; everything else runs on a CPU-only host.
"""
import importlib.util
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "galaxy-collision-simulation_b200"
GOLDEN = Path(__file__).resolve().parent / "golden"

if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def _load_gx():
    if "gx" in sys.modules:
        return sys.modules["gx"]
    spec = importlib.util.spec_from_file_location("gx", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["gx"] = mod
    spec.loader.exec_module(mod)
    return mod


_load_gx()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    def load(name):
        return dict(np.load(GOLDEN / name, allow_pickle=False))
    return load


def rel_err(a, b):
    """Per-row relative error |a - b| / max(|b|, 1e-12) of (n, 3) arrays (the reference KAT's
    metric, cpp/tests/smoke_tests.cpp:107-115)."""
    a = np.asarray(a)
    b = np.asarray(b)
    return np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-12)
