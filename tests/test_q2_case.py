"""Curved (Q = 2) nozzle cases on the host: the case build, the initial state and the parity
observables against the reference's own config-1 solve on quadratic triangles (tests/golden/
config1_q2.npz, made by make_golden.py from the reference's build_case and solve_nozzle)."""

from __future__ import annotations

import numpy as np

from conftest import golden, pkg, rel


def case(lean=False):
    cfg, nz = pkg("config"), pkg("nozzle")
    flow = cfg.FlowConditions(flux="roe", back_pressure_ratio=0.15)
    opts = cfg.SolverOptions(cfl=0.5, tolerance=1e-10, limiter="positivity", scheme="ssprk3", print_interval=0)
    return nz.build_case(contour="smooth", area_ratio=2.5, element="tri", order=1, refine=0, geometry_order=2,
                         flow=flow, options=opts, lean=lean)


def test_curved_case_is_the_references():
    g = golden("config1_q2.npz")
    cs = case()
    assert cs.topology.geometry_order == 2
    assert np.array_equal(np.asarray(cs.topology.elem_nodes), g["elem_nodes"])
    assert np.array_equal(np.asarray(cs.node_coords), g["node_coords"])
    assert rel(cs.initial_state(), g["U0"]) < 1e-13
    assert pkg("generic").needs_generic(cs.operators)


def test_curved_case_observables_are_the_references():
    g = golden("config1_q2.npz")
    cs = case()
    perf = pkg("observables").performance(g["U_final"], cs.operators, cs.flow)
    for k in ("thrust", "mass_flow_in", "exit_mach"):
        assert rel(perf[k], g[k]) < 1e-12, k


def test_geometry_order_is_checked():
    import pytest

    with pytest.raises(ValueError, match="geometry_order"):
        pkg("nozzle").build_case(geometry_order=0)
