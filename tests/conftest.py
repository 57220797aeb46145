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


def roundoff_spread(run, U0, seeds=(1, 2), eps=2e-16):
    """Per-element spread of ``run(U0)`` under relative input perturbations of size ``eps``.

    ``run`` maps an (E, NP, 4) state to the state after some steps (the CPU
    oracle).  Elements where the reference algorithm itself amplifies round-off
    (a limiter decision within round-off of its bound) show a large spread.
    """
    base = run(np.array(U0, copy=True))
    spread = np.zeros(base.shape[0])
    for seed in seeds:
        noise = np.random.default_rng(seed).standard_normal(np.shape(U0))
        V = run(np.asarray(U0) * (1.0 + eps * noise))
        spread = np.maximum(spread, np.abs(V - base).reshape(base.shape[0], -1).max(axis=1))
    return base, spread


def assert_step_agrees(got, ref, spread, tol=1e-12, cap=0.01, mask=None):
    """``got`` within ``tol`` of ``ref`` (normwise) except on round-off-sensitive elements.

    Elements whose ``spread`` (see roundoff_spread) exceeds 1e-13 of the scale
    are reported, limited to a fraction ``cap`` of the elements, and held to 100
    times their spread instead.
    """
    got, ref = np.asarray(got), np.asarray(ref)
    mask = np.ones(ref.shape[0], bool) if mask is None else mask
    scale = np.abs(ref[mask]).max()
    sens = mask & (spread > 1e-13 * scale)
    dev = np.abs(got - ref).reshape(ref.shape[0], -1).max(axis=1)
    if sens.any():
        print(f"{int(sens.sum())} of {int(mask.sum())} elements round-off-sensitive in the reference algorithm "
              f"(spread up to {spread[mask].max() / scale:.1e}, deviation there {dev[sens].max() / scale:.1e})")
    assert sens.sum() <= cap * mask.sum()
    assert dev[mask & ~sens].max() / scale < tol, dev[mask & ~sens].max() / scale
    assert np.all(dev[sens] <= 100.0 * spread[sens] + tol * scale)


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
