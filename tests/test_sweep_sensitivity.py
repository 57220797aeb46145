"""How a non-converging sweep point's outcome turns on round-off, on the reference's own compiled step.

Point 152 of the sampled 256-point sweep (AR 1.70, p_b 0.238, p = 2 quadrilaterals, refine 2) does
not converge in the reference: it stalls at a scaled residual of 1.4e3 after 3851 iterations
(tests/golden/sweep_reference.json).  Marched on the C restatement of the reference's Numba step
(oracle/cpu_step.c) from the host's initial state it does the same; from that state perturbed by
3e-15 (relative) it diverges after 1901 iterations instead.  The sweep test therefore lets such
points differ in kind.  About 25 s on 8 cores.
"""

from __future__ import annotations

import json

import numpy as np

from conftest import GOLDEN, pkg
from oracle import cpu_port


class _Port:
    """The C port behind the few attributes the march reads."""

    def __init__(self, inst):
        self.ops, self.flow, self.opts = inst.ops, inst.flow, inst.opts
        self.st = cpu_port.CpuStepper(inst.ops, inst.flow, inst.opts)
        self.scheme = self.st.scheme
        self.n_mean_repaired = 0

    def run(self, U, n, scheme):
        return self.st.run(U, n, scheme)

    def limiter_activity(self):
        return 0.0


def test_point_152_outcome_turns_on_round_off():
    ref = {r["point"]: r for r in json.load(open(f"{GOLDEN}/sweep_reference.json"))["rows"]}[152]
    sw, march = pkg("sweep"), pkg("march")
    inst = sw.build_instances([sw.sample_points(256, 0)[152]], max_iterations=20000, lean=False)[0][0]
    cpu_port.set_threads(8)
    try:
        a = march.solve(_Port(inst), np.asarray(inst.U0), length=inst.length)
        noise = np.random.default_rng(1).standard_normal(inst.U0.shape)
        b = march.solve(_Port(inst), np.asarray(inst.U0) * (1.0 + 3e-15 * noise), length=inst.length)
    finally:
        cpu_port.set_threads(1)
    assert not a.converged and a.iterations == ref["iterations"] and "stalled" in a.message
    assert not b.converged and "diverg" in b.message and b.iterations != a.iterations
