"""Orders above 3 and curved (Q = 2) elements on the host: the operator build and the oracle against the
reference's fixtures (tests/golden/tiny_{kind}_p{p}_q{q}.npz, made by make_golden.py's generic_cases)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, pkg, rel
from oracle import dg_oracle as orc

CASES = [("tri", 4, 1), ("tri", 5, 1), ("quad", 4, 1), ("tri", 2, 2), ("tri", 3, 2), ("quad", 2, 2)]


def generic_ops(kind, p, q):
    g = golden(f"tiny_{kind}_p{p}_q{q}.npz")
    topo, _, _ = pkg("mesh").channel_topology(kind, refine=0, geometry_order=q)
    return pkg("operators").build_operators(topo, g["node_coords"], p), g


@pytest.mark.parametrize("kind,p,q", CASES)
def test_host_operators_are_the_references(kind, p, q):
    ops, g = generic_ops(kind, p, q)
    assert np.array_equal(np.asarray(ops.topology.elem_nodes), g["elem_nodes"])
    for name in ("inv_mass", "edge_normal", "edge_jac", "edge_length", "elem_area", "mean_weights"):
        assert np.array_equal(np.asarray(getattr(ops, name)), g[name]), name
    assert pkg("generic").needs_generic(ops)


@pytest.mark.parametrize("kind,p,q", CASES)
def test_oracle_matches_the_reference(kind, p, q):
    ops, g = generic_ops(kind, p, q)
    cfg = pkg("config")
    for flux in ("roe", "hllc", "ausmup"):
        R, wave = orc.residual(g["U"], ops, cfg.FlowConditions(flux=flux))
        assert rel(R, g[f"R_{flux}"]) < 1e-13 and rel(wave, g[f"wave_{flux}"]) < 1e-13
    L, _, _ = orc.positivity(g["U_bad"], ops, cfg.FlowConditions())
    assert rel(L, g["limited_bad"]) < 1e-13
    V, res = orc.Stepper(ops, cfg.FlowConditions(), cfg.SolverOptions(scheme="ssprk3")).run(g["U"].copy(), 3)
    assert rel(V, g["run3_ssprk3"]) < 1e-12 and abs(res - g["run3_ssprk3_res"]) <= 1e-12 * g["run3_ssprk3_res"]


@pytest.mark.parametrize("kind,p,q", CASES)
def test_oracle_superbee_matches_the_reference_on_generic_meshes(kind, p, q):
    """The oracle's Superbee (then positivity) and three SSP-RK3 steps with it against the reference's own
    superbee_limiter, apply_limiter and NumPy backend on the generic meshes (tiny_*_superbee.npz: the
    fixture state with per-node jumps, TVB constant 0.5).  The device's generic Superbee is checked
    against this oracle on the same states."""
    ops, _ = generic_ops(kind, p, q)
    f = golden(f"tiny_{kind}_p{p}_q{q}_superbee.npz")
    cfg = pkg("config")
    sb, changed = orc.superbee(f["U"], ops, 0.5)
    assert changed.sum() > 0
    assert rel(sb, f["superbee"]) < 1e-13
    assert rel(orc.positivity(sb, ops, cfg.FlowConditions())[0], f["superbee_positivity"]) < 1e-13
    W, res = orc.Stepper(ops, cfg.FlowConditions(), cfg.SolverOptions(scheme="ssprk3", limiter="superbee",
                                                                      tvb_constant=0.5)).run(f["U"].copy(), 3)
    assert rel(W, f["run3_ssprk3"]) < 1e-12
    assert abs(res - f["run3_ssprk3_res"]) <= 1e-12 * f["run3_ssprk3_res"]
