"""March bookkeeping and failure detection on the host, with scripted backends (no GPU).

Failures are made on the host: a backend whose residual goes non-finite, grows
past the divergence factor, or parks -- exactly what the march must turn into a
message instead of an exception.
"""

from __future__ import annotations

import math

import numpy as np

from conftest import golden, pkg, rel


class Scripted:
    """A backend whose ``run`` returns residuals from a script, one per call."""

    def __init__(self, residuals, opts):
        self.residuals = list(residuals)
        self.opts = opts
        self.scheme = "ssprk3"
        self.calls = []

    def run(self, U, n, scheme):
        self.calls.append(n)
        return U, self.residuals.pop(0)


def opts(**kw):
    return pkg("config").SolverOptions(tolerance=1e-10, **kw)


def test_converges_at_the_first_check_below_tolerance():
    m = pkg("march")
    bk = Scripted([1.0, 0.5, 1e-11], opts())
    U, its, res, res0, conv, msg, _, _ = m.march(np.zeros(1), bk, bk.opts, 1.0)
    assert conv and its == 1 + 50 + 50 and bk.calls == [1, 50, 50] and msg == ""


def test_non_finite_residual_is_reported_not_raised():
    m = pkg("march")
    bk = Scripted([1.0, 0.5, float("nan")], opts())
    *_, conv, msg, _, _ = m.march(np.zeros(1), bk, bk.opts, 1.0)
    assert not conv and "non-finite" in msg


def test_divergence_factor():
    m = pkg("march")
    bk = Scripted([1.0, 2.0, 2e4], opts())
    *_, conv, msg, _, _ = m.march(np.zeros(1), bk, bk.opts, 1.0)
    assert not conv and "divergence" in msg


def test_stall_window():
    m = pkg("march")
    bk = Scripted([1.0] + [0.5] * 100, opts(stall_window=5))
    U, its, *_ , conv, msg, _, _ = m.march(np.zeros(1), bk, bk.opts, 1.0)
    assert not conv and "stalled" in msg and its == 1 + 5 * 50


def test_max_iterations_caps_the_last_chunk():
    m = pkg("march")
    bk = Scripted([1.0] + [0.9 ** k for k in range(1, 10)], opts(max_iterations=120, stall_window=40))
    U, its, *_ , conv, msg, _, _ = m.march(np.zeros(1), bk, bk.opts, 1.0)
    assert its == 120 and bk.calls == [1, 50, 50, 19] and "max_iterations" in msg


def test_initial_non_finite():
    m = pkg("march")
    bk = Scripted([math.inf], opts())
    *_, conv, msg, _, _ = m.march(np.zeros(1), bk, bk.opts, 1.0)
    assert not conv and "initial" in msg


def test_observables_of_the_reference_solution():
    """Thrust, mass flow and exit Mach of the reference's converged config-1 state."""
    g = golden("config1.npz")
    topo, _, _ = pkg("mesh").channel_topology("tri", refine=1)
    ops = pkg("operators").build_operators(topo, g["node_coords"], 1)
    perf = pkg("observables").performance(g["U_final"], ops, pkg("config").FlowConditions())
    assert rel(perf["thrust"], g["thrust"]) < 1e-13
    assert rel(perf["mass_flow_in"], g["mass_flow_in"]) < 1e-13
    assert rel(perf["exit_mach"], g["exit_mach"]) < 1e-13
