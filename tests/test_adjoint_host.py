"""The adjoint's CPU pieces: the complex-step oracle, the design-variable contour and the case set-up."""

from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from conftest import pkg, rel, tiny_ops
from oracle import dg_oracle as orc

FLUXES = ("roe", "hllc", "ausmup")


def flow_for(flux, **kw):
    return pkg("config").FlowConditions(flux=flux, **kw)


@pytest.mark.parametrize("kind,p", [("tri", 1), ("tri", 3), ("quad", 2)])
def test_operators_at_reproduces_the_operators(kind, p):
    ops, g = tiny_ops(kind, p)
    flow = flow_for("hllc")
    R0, w0 = orc.residual(g["U"], ops, flow)
    R1, w1 = orc.residual(g["U"], orc.operators_at(ops, np.asarray(ops.node_coords)), flow)
    assert rel(R1, R0) < 1e-13 and rel(w1, w0) < 1e-13
    o = orc.operators_at(ops, np.asarray(ops.node_coords))
    assert rel(o.inv_mass, ops.inv_mass) < 1e-12


@pytest.mark.parametrize("flux", FLUXES)
@pytest.mark.parametrize("kind,p", [("tri", 2), ("quad", 1)])
def test_complex_step_jvp_matches_central_differences(kind, p, flux):
    ops, g = tiny_ops(kind, p)
    flow = flow_for(flux, back_pressure_ratio=0.9)
    U = g["U"]
    V = np.random.default_rng(1).standard_normal(U.shape) * np.abs(U).mean(axis=(0, 1))
    Rc = orc.residual(U.astype(complex) + 1j * orc.H_CS * V, ops, flow)[0]
    jvp = Rc.imag / orc.H_CS
    h = 1e-6
    fd = (orc.residual(U + h * V, ops, flow)[0] - orc.residual(U - h * V, ops, flow)[0]) / (2 * h)
    assert rel(jvp, fd) < 1e-5
    assert rel(Rc.real, orc.residual(U, ops, flow)[0]) < 1e-14


def test_coordinate_and_back_pressure_vjp_match_central_differences():
    ops, g = tiny_ops("tri", 1)
    flow = flow_for("roe", back_pressure_ratio=0.9)
    U = g["U"]
    lam = np.random.default_rng(2).standard_normal(U.shape)
    gX = orc.coord_vjp(U, lam, ops, flow)
    X = np.asarray(ops.node_coords, float)
    rng = np.random.default_rng(3)
    for a in rng.choice(X.shape[0], 6, replace=False):
        for d in range(2):
            h = 1e-6
            Xp, Xm = X.copy(), X.copy()
            Xp[a, d] += h
            Xm[a, d] -= h
            fp = np.sum(lam * orc.residual(U, orc.operators_at(ops, Xp), flow)[0])
            fm = np.sum(lam * orc.residual(U, orc.operators_at(ops, Xm), flow)[0])
            fd = (fp - fm) / (2 * h)
            assert abs(gX[a, d] - fd) <= 1e-6 * max(1.0, abs(fd))
    h = 1e-6
    fp = np.sum(lam * orc.residual(U, ops, dataclasses.replace(flow, back_pressure_ratio=0.9 + h))[0])
    fm = np.sum(lam * orc.residual(U, ops, dataclasses.replace(flow, back_pressure_ratio=0.9 - h))[0])
    gp = orc.back_pressure_vjp(U, lam, ops, flow)
    assert abs(gp - (fp - fm) / (2 * h)) <= 1e-6 * max(1.0, abs(gp))


def test_adjoint_march_reaches_the_linear_solve():
    """Many RK4 steps of the oracle march converge to the solution of J^T lam = seed."""
    ops, g = tiny_ops("tri", 1)
    flow = flow_for("roe")
    U = g["U"]
    J = orc.state_jacobian(U, ops, flow)
    seed = np.zeros_like(U)
    seed[:5] = 1.0
    lam = orc.adjoint_march(U, seed, ops, flow, 0.5, 3, J=J)
    assert np.all(np.isfinite(lam)) and np.abs(lam).max() > 0.0


@pytest.mark.parametrize("contour", ["bell", "smooth", "conical", "moc", "bezier", "bezier8"])
def test_wall_from_design_variables_matches_the_contour(contour):
    nz = pkg("nozzle")
    kw = {"offsets": tuple(0.01 * np.sin(np.arange(8)))} if contour == "bezier8" else {}
    geom = nz.Geometry(contour=contour, area_ratio=2.5, **kw)
    x = np.linspace(0.0, 1.0, 401)
    assert np.array_equal(nz.wall_from_params(x, nz.design_params(geom), contour), nz.wall_half_height(x, geom))
    g2 = nz.geometry_with(geom, {"area_ratio": 3.0, "theta_exit": 0.1})
    assert g2.area_ratio == 3.0 and abs(g2.theta_exit_deg - np.degrees(0.1)) < 1e-12


def test_differentiable_case_routes_keywords_and_freezes_the_grid():
    ad = pkg("adjoint")
    dc = ad.differentiable_case(contour="smooth", order=1, refine=0, back_pressure_ratio=0.15, tolerance=1e-11,
                                flux="ausmup")
    assert dc.flow.flux == "ausmup" and dc.options.tolerance == 1e-11 and dc.flow.back_pressure == 0.15
    base = pkg("nozzle").build_case(contour="smooth", order=1, refine=0)
    assert np.array_equal(dc.node_coords({}), base.node_coords)
    X2 = dc.node_coords({"area_ratio": 3.0})
    assert X2.shape == base.node_coords.shape and np.array_equal(X2[:, 0], base.node_coords[:, 0])
    with pytest.raises(ValueError):
        dc.params_for(["nope"])
    assert set(ad.OBJECTIVES) == {"thrust", "thrust_coefficient", "exit_mach", "mass_flow", "exit_pressure"}


@pytest.mark.parametrize("contour", ["smooth", "bell", "bezier8"])
def test_node_coordinate_derivatives_match_central_differences(contour):
    """torch's derivative of X(a) against central differences of the NumPy contour."""
    import torch

    ad, nz = pkg("adjoint"), pkg("nozzle")
    kw = {"offsets": tuple(0.01 * np.cos(np.arange(8)))} if contour == "bezier8" else {}
    dc = ad.differentiable_case(contour=contour, order=1, refine=0, device="cpu", **kw)
    names = ["area_ratio", "throat_x", "throat_half_height", "inlet_half_height", "theta_exit", "length"]
    names += ["offset_2"] if contour == "bezier8" else ["theta_initial"]
    base = dc.default_params()
    w = np.random.default_rng(0).standard_normal(dc.node_coords({}).shape)
    for k in names:
        P = {kk: torch.tensor(float(v), dtype=torch.float64, requires_grad=(kk == k)) for kk, v in base.items()}
        X = dc.node_coords(P, xp=torch)
        (g,) = torch.autograd.grad((X * torch.as_tensor(w)).sum(), [P[k]])
        h = 1e-6 * max(1.0, abs(base[k]))
        up, dn = dict(base), dict(base)
        up[k] += h
        dn[k] -= h
        fd = np.sum(w * (dc.node_coords(up) - dc.node_coords(dn))) / (2 * h)
        assert abs(float(g) - fd) <= 1e-6 * max(1.0, abs(fd)), (k, float(g), fd)
