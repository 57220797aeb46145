"""Observables (src/post/postprocess.py:193-263) against the reference's own performance().

``observables.npz`` holds every field of the reference's ``Performance`` for the
tiny cases' states and for the reference's converged config-1 state; the host
sums and the metrics formed from them must reproduce each one.
"""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TINY, golden, pkg, rel, tiny_ops

FIELDS = ("thrust", "thrust_wall", "thrust_imbalance", "thrust_coefficient", "mass_flow_in", "mass_flow_out",
          "mass_imbalance", "entropy_error", "exit_mach_area_averaged", "exit_pressure_ratio",
          "exit_temperature_ratio", "specific_thrust", "specific_thrust_ratio", "discharge_coefficient",
          "ideal_thrust", "thrust_efficiency")
# relative tolerance per field: the imbalances are differences of nearly equal
# numbers, so their own relative error is that of the terms over the difference
TOL = {"thrust_imbalance": 1e-9, "mass_imbalance": 1e-9}


def check(perf, g, prefix):
    for f in FIELDS:
        assert rel(perf[f], g[f"{prefix}_{f}"]) < TOL.get(f, 1e-12), (prefix, f, perf[f], float(g[f"{prefix}_{f}"]))


@pytest.mark.parametrize("kind,p", TINY)
def test_tiny_states_match_the_reference(kind, p):
    ops, gt = tiny_ops(kind, p)
    geom = pkg("nozzle").Geometry()
    perf = pkg("observables").performance(gt["U"], ops, pkg("config").FlowConditions(), geom)
    check(perf, golden("observables.npz"), f"{kind}{p}")


def test_converged_config1_matches_the_reference():
    g = golden("config1.npz")
    topo, _, _ = pkg("mesh").channel_topology("tri", refine=1)
    ops = pkg("operators").build_operators(topo, g["node_coords"], 1)
    geom = pkg("nozzle").Geometry(area_ratio=2.5)
    perf = pkg("observables").performance(g["U_final"], ops, pkg("config").FlowConditions(), geom)
    check(perf, golden("observables.npz"), "config1")


def test_segments_cover_each_instance():
    """Boundary-edge lists and element ranges of instances laid out one after another."""
    obs = pkg("observables")
    ops_a, _ = tiny_ops("tri", 1)
    ops_b, _ = tiny_ops("quad", 2)
    k_a = ops_a.n_interior + ops_a.n_boundary
    b, bs, es = obs.segments([(ops_a, 0, 0), (ops_b, ops_a.n_elem, k_a)])
    mesh = pkg("mesh")
    for i, (ops, k0) in enumerate(((ops_a, 0), (ops_b, k_a))):
        mine = b[bs[i]:bs[i + 1]] - k0
        tags = np.asarray(ops.topology.edges.bedge_tag)[mine - ops.n_interior]
        assert set(tags.tolist()) == {mesh.INFLOW, mesh.OUTFLOW, mesh.WALL}
        assert len(mine) == int(np.sum(np.isin(np.asarray(ops.topology.edges.bedge_tag),
                                               [mesh.INFLOW, mesh.OUTFLOW, mesh.WALL])))
    assert list(es) == [0, ops_a.n_elem, ops_a.n_elem + ops_b.n_elem]
