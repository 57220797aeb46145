"""The CPU oracle against outputs of the reference solver itself (tests/golden)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TINY, golden, pkg, rel, tiny_ops
from oracle import dg_oracle as orc

FLUXES = ("roe", "hllc", "ausmup")


@pytest.mark.parametrize("kind,p", TINY)
@pytest.mark.parametrize("flux", FLUXES)
def test_residual_and_rate(kind, p, flux):
    ops, g = tiny_ops(kind, p)
    flow = pkg("config").FlowConditions(flux=flux)
    R, wave = orc.residual(g["U"], ops, flow)
    assert rel(R, g[f"R_{flux}"]) < 1e-13
    assert rel(wave, g[f"wave_{flux}"]) < 1e-13
    assert rel(orc.rate(g["U"], ops, flow)[0], g[f"rate_{flux}"]) < 1e-13


@pytest.mark.parametrize("kind,p", TINY)
def test_backflow_outflow(kind, p):
    ops, g = tiny_ops(kind, p)
    R, _ = orc.residual(g["U"], ops, pkg("config").FlowConditions(backflow=True))
    assert rel(R, g["R_roe_backflow"]) < 1e-13


@pytest.mark.parametrize("kind,p", TINY)
def test_limiter_restores_the_reference_state(kind, p):
    ops, g = tiny_ops(kind, p)
    out, bad, rep = orc.positivity(g["U_bad"], ops, pkg("config").FlowConditions())
    assert rel(out, g["limited_bad"]) < 1e-13
    if p > 0:
        assert set(np.flatnonzero(rep)) == {11}


@pytest.mark.parametrize("kind,p", TINY)
@pytest.mark.parametrize("scheme", ["euler", "ssprk3"])
def test_three_steps(kind, p, scheme):
    ops, g = tiny_ops(kind, p)
    cfg = pkg("config")
    st = orc.Stepper(ops, cfg.FlowConditions(), cfg.SolverOptions(scheme=scheme))
    V, res = st.run(g["U"].copy(), 3)
    assert rel(V, g[f"run3_{scheme}"]) < 1e-12
    assert abs(res - g[f"run3_{scheme}_res"]) <= 1e-12 * abs(g[f"run3_{scheme}_res"])


@pytest.mark.parametrize("flux", FLUXES)
def test_microbench_distribution_step_and_limited_sets(flux):
    """Config-2 state distribution at 400 cubic triangles: heavy limiting."""
    g = golden("rect_tri_p3.npz")
    topo, _, _ = pkg("mesh").channel_topology("tri", nx=20, nr=10)
    ops = pkg("operators").build_operators(topo, g["node_coords"], 3)
    cfg = pkg("config")
    flow = cfg.FlowConditions(flux=flux)
    R, wave = orc.residual(g["U"], ops, flow)
    assert rel(R, g[f"R_{flux}"]) < 1e-13 and rel(wave, g[f"wave_{flux}"]) < 1e-13
    st = orc.Stepper(ops, flow, cfg.SolverOptions(cfl=0.5))
    V, res = st.run(g["U"].copy(), 1)
    assert rel(V, g[f"step_{flux}"]) < 1e-12
    assert np.array_equal(np.stack(st.stage_masks), g[f"step_{flux}_limited"])


@pytest.mark.parametrize("kind,p", [("tri", 1), ("tri", 2), ("tri", 3), ("quad", 1), ("quad", 2), ("quad", 3)])
def test_oracle_superbee_matches_the_reference(kind, p):
    """The Superbee TVB slope limiter, with and without the threshold, then positivity; and 3 SSP-RK3 steps."""
    ops, _ = tiny_ops(kind, p)
    g = golden(f"superbee_{kind}_p{p}.npz")
    cfg = pkg("config")
    flow = cfg.FlowConditions()
    out, _ = orc.superbee(g["U"], ops, 50.0)
    assert rel(out, g["superbee"]) < 1e-13
    out0, changed0 = orc.superbee(g["U"], ops, 0.0)
    assert rel(out0, g["superbee_tvb0"]) < 1e-13 and changed0.any()
    assert rel(orc.positivity(out, ops, flow)[0], g["superbee_positivity"]) < 1e-13
    st = orc.Stepper(ops, flow, cfg.SolverOptions(limiter="superbee", scheme="ssprk3"))
    V, res = st.run(g["U"].copy(), 3)
    assert rel(V, g["run3_ssprk3"]) < 1e-12 and abs(res - g["run3_ssprk3_res"]) <= 1e-12 * abs(g["run3_ssprk3_res"])
