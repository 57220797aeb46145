"""Orders above 3 and curved (Q = 2) elements on the device (csrc/generic.cuh, GenericB200Backend) against
the reference's fixtures: residual, rate and wave per flux and with backflow, the limiter, three SSP-RK3
steps; twenty steps against the oracle; the generic kernels on a p = 3 straight mesh against the
specialised ones."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, pkg, rel, tiny_ops
from oracle import dg_oracle as orc
from test_oracle_generic import CASES, generic_ops

pytestmark = pytest.mark.gpu


def backend(ops, flux="roe", **opt):
    cfg = pkg("config")
    flow = cfg.FlowConditions(flux=flux, **{k: v for k, v in opt.items() if k == "backflow"})
    opts = cfg.SolverOptions(scheme="ssprk3", **{k: v for k, v in opt.items() if k != "backflow"})
    return pkg("backend").B200Backend(ops, flow, opts)


@pytest.mark.parametrize("kind,p,q", CASES)
def test_generic_kernels_match_the_reference(cuda, kind, p, q):
    ops, g = generic_ops(kind, p, q)
    for flux in ("roe", "hllc", "ausmup"):
        bk = backend(ops, flux)
        assert type(bk).__name__ == "GenericB200Backend"
        R, wave = bk.residual(g["U"])
        F, _ = bk.rate(g["U"])
        assert rel(R, g[f"R_{flux}"]) < 1e-12 and rel(wave, g[f"wave_{flux}"]) < 1e-12
        assert rel(F, g[f"rate_{flux}"]) < 1e-12
        assert rel(bk.inverse_mass(R), -g[f"rate_{flux}"]) < 1e-12
    bb = backend(ops, "roe", backflow=True)
    assert rel(bb.residual(g["U"])[0], g["R_roe_backflow"]) < 1e-12
    bk = backend(ops)
    assert rel(bk.limit(g["U_bad"]), g["limited_bad"]) < 1e-12
    assert bk.n_limited > 0
    V, res = bk.run(g["U"], 3, "ssprk3")
    assert rel(V, g["run3_ssprk3"]) < 1e-11
    assert abs(res - g["run3_ssprk3_res"]) <= 1e-11 * g["run3_ssprk3_res"]


@pytest.mark.parametrize("kind,p,q", [("tri", 5, 1), ("quad", 2, 2)])
def test_generic_march_follows_the_oracle(cuda, kind, p, q):
    ops, g = generic_ops(kind, p, q)
    cfg = pkg("config")
    bk = backend(ops, "hllc", cfl=0.5)
    V, res = bk.run(g["U"], 20, "ssprk3")
    W, res_ref = orc.Stepper(ops, cfg.FlowConditions(flux="hllc"), cfg.SolverOptions(scheme="ssprk3", cfl=0.5)).run(
        g["U"].copy(), 20)
    assert rel(V, W) < 1e-10 and abs(res - res_ref) <= 1e-10 * res_ref


def test_generic_kernels_agree_with_the_specialised_ones(cuda):
    """On a straight p = 3 mesh, the generic path (forced) against the specialised kernels."""
    ops, g = tiny_ops("tri", 3)
    cfg = pkg("config")
    flow, opts = cfg.FlowConditions(flux="hllc"), cfg.SolverOptions(scheme="ssprk3")
    gen = pkg("generic").GenericB200Backend(ops, flow, opts)
    spec = pkg("backend").B200Backend(ops, flow, opts)
    for U in (g["U"], g["U_bad"]):
        assert rel(gen.residual(U)[0], spec.residual(U)[0]) < 1e-12
        assert rel(gen.limit(U), spec.limit(U)) < 1e-12
    assert rel(gen.run(g["U"], 3, "ssprk3")[0], spec.run(g["U"], 3, "ssprk3")[0]) < 1e-11


@pytest.mark.parametrize("kind,p,q", CASES)
def test_device_built_operators_match_the_host_build(cuda, kind, p, q):
    """nzb_gen_geometry against the host build (the reference's operators, bit for bit): every
    coordinate-dependent array at 1e-13, then the residual, rate, limiter and three steps on the
    device-built mesh against the reference's fixtures."""
    ops, g = generic_ops(kind, p, q)
    cfg = pkg("config")
    gen = pkg("generic")
    flow, opts = cfg.FlowConditions(flux="hllc"), cfg.SolverOptions(scheme="ssprk3")
    bk = gen.GenericB200Backend(ops, flow, opts, device_metrics=True)
    assert bk.device_built
    for name in ("grad_x", "grad_y", "grad_x_m", "grad_y_m", "face_basis_m", "inv_mass", "elem_area", "mean_weights",
                 "edge_normal", "edge_jac", "edge_length"):
        assert rel(bk._arr[name].cpu().numpy(), np.asarray(getattr(ops, name))) < 1e-13, name
    R, wave = bk.residual(g["U"])
    assert rel(R, g["R_hllc"]) < 1e-12 and rel(wave, g["wave_hllc"]) < 1e-12
    assert rel(bk.rate(g["U"])[0], g["rate_hllc"]) < 1e-12
    assert rel(bk.inverse_mass(R), -g["rate_hllc"]) < 1e-12
    assert rel(bk.limit(g["U_bad"]), g["limited_bad"]) < 1e-12
    rk = gen.GenericB200Backend(ops, cfg.FlowConditions(flux="roe"), opts, device_metrics=True)
    V, res = rk.run(g["U"], 3, "ssprk3")
    assert rel(V, g["run3_ssprk3"]) < 1e-11
    assert abs(res - g["run3_ssprk3_res"]) <= 1e-11 * g["run3_ssprk3_res"]


@pytest.mark.parametrize("kind,p,q", [("tri", 3, 2), ("quad", 4, 1)])
def test_lean_operators_build_on_the_device(cuda, kind, p, q):
    """Operators built without the per-element arrays (lean) take the device build automatically."""
    _, g = generic_ops(kind, p, q)
    topo, _, _ = pkg("mesh").channel_topology(kind, refine=0, geometry_order=q)
    lean = pkg("operators").build_operators(topo, g["node_coords"], p, lean=True)
    assert lean.grad_x is None
    cfg = pkg("config")
    bk = pkg("backend").B200Backend(lean, cfg.FlowConditions(flux="ausmup"), cfg.SolverOptions(scheme="ssprk3"))
    assert type(bk).__name__ == "GenericB200Backend" and bk.device_built
    R, wave = bk.residual(g["U"])
    assert rel(R, g["R_ausmup"]) < 1e-12 and rel(wave, g["wave_ausmup"]) < 1e-12


def test_device_build_refuses_an_inverted_element(cuda):
    """A quadrature point with a non-positive Jacobian is refused, as the reference's build refuses it."""
    ops, g = generic_ops("tri", 2, 2)
    X = np.array(g["node_coords"], float)
    en = np.asarray(ops.topology.elem_nodes)
    a, b = en[0, 1], en[0, 2]
    X[[a, b]] = X[[b, a]]  # swap two vertices of element 0: its orientation flips
    import dataclasses

    bad = dataclasses.replace(ops, node_coords=X)
    cfg = pkg("config")
    with pytest.raises(ValueError, match="non-positive Jacobian"):
        pkg("generic").GenericB200Backend(bad, cfg.FlowConditions(), cfg.SolverOptions(), device_metrics=True)


@pytest.mark.parametrize("kind,p,q", CASES)
def test_generic_superbee_follows_the_oracle(cuda, kind, p, q):
    """The Superbee slope limiter then the positivity limiter on the generic path against the oracle's
    restatement (pinned on the reference's own Superbee fixtures), on a state with per-node jumps and a
    small TVB constant so that most elements are limited; then three SSP-RK3 steps."""
    ops, g = generic_ops(kind, p, q)
    cfg = pkg("config")
    flow = cfg.FlowConditions(flux="hllc")
    opts = cfg.SolverOptions(scheme="ssprk3", limiter="superbee", tvb_constant=0.5)
    rng = np.random.default_rng(7)
    U = np.array(g["U"], float)
    U *= 1.0 + 0.3 * rng.uniform(-1.0, 1.0, size=U.shape[:2])[..., None]
    bk = pkg("generic").GenericB200Backend(ops, flow, opts)
    want, changed = orc.superbee(U, ops, 0.5)
    assert changed.sum() > 0
    want = orc.positivity(want, ops, flow)[0]
    assert rel(bk.limit(U), want) < 1e-12
    assert bk.n_limited >= changed.sum()
    V, res = bk.run(U, 3, "ssprk3")
    W, res_ref = orc.Stepper(ops, flow, opts).run(U.copy(), 3)
    assert rel(V, W) < 1e-11 and abs(res - res_ref) <= 1e-11 * res_ref


@pytest.mark.parametrize("device_metrics", [False, True])
def test_curved_nozzle_solve_matches_the_reference(cuda, device_metrics):
    """Config 1 on curved (Q = 2) triangles end to end on the generic path: the reference's own
    solve converges in the same number of iterations to the same thrust, mass flow and exit Mach
    (1e-10), with the operators uploaded from the host or built on the device."""
    from test_q2_case import case

    g = golden("config1_q2.npz")
    full = case()
    cs = case(lean=device_metrics)
    bk = pkg("backend").B200Backend(cs.operators, cs.flow, cs.options, device_metrics=device_metrics)
    assert type(bk).__name__ == "GenericB200Backend" and bk.device_built == device_metrics
    U0 = g["U0"]
    if device_metrics:  # the lean case starts from the device-projected initial state
        U0 = bk.initial_state(cs.geometry)
        assert rel(U0, g["U0"]) < 1e-13
    res = pkg("march").solve(bk, U0, length=cs.geometry.length)
    assert res.converged, res.message
    assert res.iterations == int(g["iterations"])
    perf = pkg("observables").performance(res.U, full.operators, full.flow)
    for k in ("thrust", "mass_flow_in", "exit_mach"):
        assert rel(perf[k], g[k]) < 1e-10, k
    assert rel(res.U, g["U_final"]) < 1e-9


@pytest.mark.parametrize("element,order,q,contour", [("tri", 4, 1, "bell"), ("quad", 4, 1, "conical"),
                                                     ("tri", 2, 2, "bezier"), ("quad", 2, 2, "smooth"),
                                                     ("tri", 3, 2, "bezier8")])
def test_generic_device_initial_state_matches_the_host(cuda, element, order, q, contour):
    """nzb_gen_initial_state against the host projection (the reference's algorithm) on nozzle meshes of
    higher order and curved elements.  The Bezier families evaluate the wall slope by a difference of
    step 1e-6 L, which magnifies the host libm's last-bit differences in pow (as for the specialised
    kernel): 1e-10 there, 1e-13 otherwise."""
    cfg, nz = pkg("config"), pkg("nozzle")
    flow = cfg.FlowConditions(flux="hllc", back_pressure_ratio=0.15)
    cs = nz.build_case(element=element, order=order, refine=0, geometry_order=q, contour=contour, area_ratio=2.2,
                       flow=flow, options=cfg.SolverOptions())
    want = cs.initial_state()
    for device_metrics in (False, True):
        bk = pkg("generic").GenericB200Backend(cs.operators, cs.flow, cs.options, device_metrics=device_metrics)
        got = bk.initial_state(cs.geometry)
        assert rel(got, want) < (1e-10 if contour.startswith("bezier") else 1e-13), device_metrics
        dev = bk.initial_state(cs.geometry, host=False)
        assert rel(dev.cpu().numpy(), got) == 0.0


@pytest.mark.parametrize("kind,p,q", CASES)
def test_generic_device_observables_match_the_host(cuda, kind, p, q):
    """nzb_gen_observables against the host integrals (the reference's performance() restated) on every
    generic fixture mesh, with its operators uploaded or built on the device."""
    ops, g = generic_ops(kind, p, q)
    cfg = pkg("config")
    flow, opts = cfg.FlowConditions(flux="hllc"), cfg.SolverOptions()
    want = pkg("observables").performance(g["U"], ops, flow)
    for device_metrics in (False, True):
        bk = pkg("generic").GenericB200Backend(ops, flow, opts, device_metrics=device_metrics)
        got = bk.performance(g["U"])
        for k, v in want.items():
            assert abs(got[k] - v) <= 1e-11 * max(abs(v), 1e-2), (k, got[k], v)


def test_curved_nozzle_observables_are_the_references(cuda):
    """The device observables of the reference's converged curved-triangle solve against its own
    performance() (1e-12), with the geometry's throat-normalised coefficients."""
    from test_q2_case import case

    g = golden("config1_q2.npz")
    cs = case(lean=True)
    bk = pkg("backend").B200Backend(cs.operators, cs.flow, cs.options)
    perf = bk.performance(g["U_final"], cs.geometry)
    for k in ("thrust", "mass_flow_in", "exit_mach"):
        assert rel(perf[k], g[k]) < 1e-12, k
    assert "thrust_coefficient" in perf and np.isfinite(perf["thrust_coefficient"])
