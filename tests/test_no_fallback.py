"""The product path has no CPU fallback: without the built library, or without a CUDA device, every
entry point raises instead of computing anything on the host."""

from __future__ import annotations

import os
import subprocess
import sys

import pytest

from conftest import pkg

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_a_missing_library_raises():
    code = (
        "import importlib, sys\n"
        "capi = importlib.import_module('2d_nozzle_b200.capi')\n"
        "try:\n"
        "    capi.load()\n"
        "except capi.NativeError as e:\n"
        "    print('raised:', e)\n"
        "    sys.exit(0)\n"
        "sys.exit(3)\n"
    )
    env = dict(os.environ, NZB_LIBRARY=os.path.join(ROOT, "no", "such", "libnozzle_b200.so"))
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "no CPU fallback" in r.stdout


@pytest.mark.parametrize("order,q", [(1, 1), (4, 1), (2, 2)])
def test_backends_refuse_a_host_device(order, q):
    """Specialised and generic backends alike refuse to run anywhere but on a CUDA device."""
    cfg, nz = pkg("config"), pkg("nozzle")
    cs = nz.build_case(element="tri", order=order, refine=0, geometry_order=q, area_ratio=2.2,
                       flow=cfg.FlowConditions(back_pressure_ratio=0.15), options=cfg.SolverOptions())
    with pytest.raises(pkg("capi").NativeError):
        pkg("backend").B200Backend(cs.operators, cs.flow, cs.options, device="cpu")
