"""Shared fixtures.  GPU tests carry ``@pytest.mark.gpu``; everything else runs on CPU."""

from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def pkg(name: str = ""):
    return importlib.import_module("2d_nozzle_b200" + (f".{name}" if name else ""))


def golden(name: str):
    return np.load(os.path.join(GOLDEN, name))


def rel(a, b) -> float:
    """The reference tests' normwise metric: max |a - b| / max |b|."""
    a, b = np.asarray(a), np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def tiny_ops(kind: str, p: int):
    g = golden(f"tiny_{kind}_p{p}.npz")
    topo, _, _ = pkg("mesh").channel_topology(kind, refine=0)
    return pkg("operators").build_operators(topo, g["node_coords"], p), g


TINY = [("tri", 0), ("tri", 1), ("tri", 2), ("tri", 3), ("quad", 1), ("quad", 2), ("quad", 3)]


@pytest.fixture(scope="session")
def cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    pkg("build").build()
    return torch
