"""Config 1 end to end: smooth AR 2.5, p=1 triangles, refine 1, Roe, cfl 0.5, to 1e-10."""

from __future__ import annotations

import pytest

from conftest import golden, pkg, rel

pytestmark = pytest.mark.gpu


def test_plain_steady_solve_matches_the_reference(cuda):
    g = golden("config1.npz")
    cfg = pkg("config")
    topo, _, _ = pkg("mesh").channel_topology("tri", refine=1)
    ops = pkg("operators").build_operators(topo, g["node_coords"], 1)
    flow = cfg.FlowConditions(flux="roe", back_pressure_ratio=0.15)
    opts = cfg.SolverOptions(cfl=0.5, tolerance=1e-10, limiter="positivity", scheme="ssprk3", print_interval=0)
    bk = pkg("backend").B200Backend(ops, flow, opts)
    res = pkg("march").solve(bk, g["U0"], length=float(g["length"]))
    assert res.converged, res.message
    assert res.iterations == int(g["iterations"])
    perf = pkg("observables").performance(res.U, ops, flow)
    assert rel(perf["thrust"], g["thrust"]) < 1e-10
    assert rel(perf["mass_flow_in"], g["mass_flow_in"]) < 1e-10
    assert rel(perf["exit_mach"], g["exit_mach"]) < 1e-10
    assert rel(res.U, g["U_final"]) < 1e-9
    assert res.mean_repairs == 0
