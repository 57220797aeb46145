"""The C restatement of the reference's compiled CPU step (oracle/cpu_step.c), which bench.py times as the
CPU baseline, against the NumPy oracle: rates and three fused steps on every tiny mesh and flux.  The
reference pins its compiled path against its NumPy path to 1e-10 (tests/test_backends.py); this holds
the port to the same bound."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TINY, pkg, rel, tiny_ops
from oracle import cpu_port
from oracle import dg_oracle as orc


@pytest.mark.parametrize("kind,p", [c for c in TINY if c[1] > 0])
@pytest.mark.parametrize("flux", ["roe", "hllc", "ausmup"])
def test_cpu_port_matches_the_oracle(kind, p, flux):
    cfg = pkg("config")
    ops, g = tiny_ops(kind, p)
    flow = cfg.FlowConditions(flux=flux, backflow=True)
    opts = cfg.SolverOptions(cfl=0.5, scheme="ssprk3")
    st = cpu_port.CpuStepper(ops, flow, opts)
    F, wave = st.rate(g["U"])
    F_ref, wave_ref = orc.rate(g["U"], ops, flow)
    assert rel(F, F_ref) < 1e-12 and rel(wave, wave_ref) < 1e-12
    V, res = st.run(g["U"], 3)
    V_ref, res_ref = orc.Stepper(ops, flow, opts).run(np.array(g["U"]), 3)
    assert rel(V, V_ref) < 1e-10
    assert abs(res - res_ref) <= 1e-10 * abs(res_ref)


def test_cpu_port_threads_give_the_same_answer():
    cfg = pkg("config")
    ops, g = tiny_ops("tri", 2)
    flow, opts = cfg.FlowConditions(flux="hllc"), cfg.SolverOptions(cfl=0.5)
    st = cpu_port.CpuStepper(ops, flow, opts)
    cpu_port.set_threads(1)
    a, ra = st.run(g["U"], 2)
    cpu_port.set_threads(4)
    b, rb = st.run(g["U"], 2)
    cpu_port.set_threads(1)
    assert rel(a, b) < 1e-13 and abs(ra - rb) <= 1e-13 * abs(ra)
