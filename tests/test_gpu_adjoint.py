"""The CUDA adjoint against the complex-step oracle, and gradients against published values.

Transposed products: each entry of (dR/dU)^T lam is lam . (column of dR/dU),
the column taken by a complex step through the oracle residual; coordinate and
back-pressure products against complex steps through the oracle's operator
rebuild.  Tolerance: the normwise metric max|a-b|/max|b| at 1e-11 (both sides
are exact to round-off; the summation orders differ).
"""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import TINY, pkg, rel, tiny_ops
from oracle import dg_oracle as orc

pytestmark = pytest.mark.gpu
FLUXES = ("roe", "hllc", "ausmup")
TOL = 1e-11


def flow_for(flux, pb=0.9):
    return pkg("config").FlowConditions(flux=flux, back_pressure_ratio=pb)


@pytest.fixture(params=["t1", "split4"])
def vjp_variant(request, monkeypatch):
    """The adjoint state kernel with one thread per element and with four."""
    monkeypatch.setenv("NZB_VJP_VARIANT", request.param)
    return request.param


def model_for(ops, flow, general=False):
    ad = pkg("adjoint")
    m = ad.AdjointModel(ops, flow, pkg("config").SolverOptions(cfl=0.5))
    if general:
        m.mesh = pkg("layout").DeviceMesh(ops, m.device, force_general=True)
        pkg("autotune").choose_variant(m.mesh)
    return m


def soa(m, A):
    import torch

    return pkg("adjoint").to_soa(torch.as_tensor(np.asarray(A, float), device=m.device))


def aos(m, a):
    return pkg("adjoint").from_soa(a, m.E, m.NP).cpu().numpy()


@pytest.mark.parametrize("kind,p", TINY)
@pytest.mark.parametrize("flux", FLUXES)
def test_state_vjp_matches_complex_steps(cuda, kind, p, flux, vjp_variant):
    ops, g = tiny_ops(kind, p)
    flow = flow_for(flux)
    U = g["U"]
    rng = np.random.default_rng(7)
    lam = rng.standard_normal(U.shape)
    cols = rng.choice(U.size, min(48, U.size), replace=False)
    ref = np.empty(len(cols))
    for n, k in enumerate(cols):
        Uc = U.astype(complex).ravel()
        Uc[k] += 1j * orc.H_CS
        ref[n] = np.sum(lam * orc.residual(Uc.reshape(U.shape), ops, flow)[0].imag) / orc.H_CS
    V = rng.standard_normal(U.shape)
    JV = orc.residual(U.astype(complex) + 1j * orc.H_CS * V, ops, flow)[0].imag / orc.H_CS
    for general in ((False, True) if kind == "tri" else (True,)):
        m = model_for(ops, flow, general)
        v = aos(m, m.vjp_state(soa(m, U), soa(m, lam))).ravel()
        assert rel(v[cols], ref) < TOL
        # the transpose identity lam . (J V) = (J^T lam) . V over every entry
        assert abs(np.sum(lam * JV) - np.sum(v * V.ravel())) <= TOL * np.sum(np.abs(lam * JV))


@pytest.mark.parametrize("kind,p,flux", [("tri", 1, "roe"), ("tri", 2, "hllc"), ("tri", 3, "ausmup"),
                                         ("quad", 1, "hllc"), ("quad", 2, "roe"), ("quad", 3, "ausmup")])
def test_coordinate_and_back_pressure_vjp_match_complex_steps(cuda, kind, p, flux):
    ops, g = tiny_ops(kind, p)
    flow = flow_for(flux)
    U = g["U"]
    lam = np.random.default_rng(11).standard_normal(U.shape)
    ref = orc.coord_vjp(U, lam, ops, flow)
    ref_pb = orc.back_pressure_vjp(U, lam, ops, flow)
    m = model_for(ops, flow)
    gX, gpb = m.vjp_coords(soa(m, U), soa(m, lam))
    assert rel(gX.cpu().numpy(), ref) < TOL
    assert abs(gpb - ref_pb) <= TOL * max(abs(ref_pb), np.abs(ref).max())


@pytest.mark.parametrize("kind,p,flux", [("tri", 2, "hllc"), ("quad", 1, "roe")])
def test_rate_and_rk4_march_match_the_oracle(cuda, kind, p, flux, vjp_variant):
    ad = pkg("adjoint")
    ops, g = tiny_ops(kind, p)
    flow = flow_for(flux)
    U = g["U"]
    rng = np.random.default_rng(5)
    seed = rng.standard_normal(U.shape)
    lam = rng.standard_normal(U.shape)
    J = orc.state_jacobian(U, ops, flow)
    m = model_for(ops, flow)
    r = aos(m, m.adjoint_rate(soa(m, U), soa(m, lam), soa(m, seed)))
    assert rel(r, -orc.inverse_mass(orc.state_vjp(U, lam, ops, flow, J) - seed, ops)) < TOL
    am = ad.AdjointMarch(m, soa(m, U), soa(m, seed), 0.5)
    lam_dev, rel_res, its, ok = am.solve(tolerance=0.0, max_iterations=6, check_interval=3)
    assert its == 6 and not ok
    ref = orc.adjoint_march(U, seed, ops, flow, 0.5, 6, J=J)
    assert rel(aos(m, lam_dev), ref) < 1e-10
    d_ref = orc.state_vjp(U, ref, ops, flow, J) - seed
    assert abs(rel_res - np.sqrt(np.mean(d_ref**2)) / np.sqrt(np.mean(seed**2))) < 1e-9


@pytest.mark.parametrize("kind,p", [c for c in TINY if c[1] > 0])
@pytest.mark.parametrize("flux", FLUXES)
def test_vjp_split_agrees_with_one_thread(cuda, kind, p, flux, monkeypatch):
    """Four threads per element against one in the adjoint state kernel: the product, the rate, the defect
    norm and six RK4 steps of the march, on every tiny mesh, flux and geometry layout, to round-off."""
    ad = pkg("adjoint")
    ops, g = tiny_ops(kind, p)
    flow = flow_for(flux)
    U = g["U"]
    rng = np.random.default_rng(3)
    lam, seed = rng.standard_normal(U.shape), rng.standard_normal(U.shape)
    for general in ((False, True) if kind == "tri" else (True,)):
        out = {}
        for name in ("t1", "split4"):
            monkeypatch.setenv("NZB_VJP_VARIANT", name)
            m = model_for(ops, flow, general)
            assert m.mesh.vjp_split == (4 if name == "split4" else 1)
            v = aos(m, m.vjp_state(soa(m, U), soa(m, lam)))
            r = aos(m, m.adjoint_rate(soa(m, U), soa(m, lam), soa(m, seed)))
            d = m.defect_rms(soa(m, U), soa(m, lam), soa(m, seed))
            am = ad.AdjointMarch(m, soa(m, U), soa(m, seed), 0.5)
            lam6, rr, its, _ = am.solve(tolerance=0.0, max_iterations=6, check_interval=3)
            out[name] = (v, r, d, aos(m, lam6), rr)
        a, b = out["t1"], out["split4"]
        assert rel(b[0], a[0]) < 1e-13 and rel(b[1], a[1]) < 1e-13 and rel(b[3], a[3]) < 1e-12
        assert abs(b[2] - a[2]) <= 1e-13 * a[2] and abs(b[4] - a[4]) <= 1e-12 * a[4]


def test_residual_function_backward_is_the_kernels(cuda):
    import torch

    ad = pkg("adjoint")
    ops, g = tiny_ops("quad", 2)
    flow = flow_for("hllc")
    m = model_for(ops, flow)
    U = soa(m, g["U"]).requires_grad_(True)
    X = m.X0.clone().requires_grad_(True)
    pb = torch.tensor(0.9, dtype=torch.float64, device=m.device, requires_grad=True)
    w = soa(m, np.random.default_rng(3).standard_normal(g["U"].shape))
    R = ad.ResidualFunction(m, U, X, pb)
    assert rel(aos(m, R.detach()), orc.residual(g["U"], ops, flow)[0]) < 1e-12
    (w * R).sum().backward()
    assert torch.equal(U.grad, m.vjp_state(U.detach(), w))
    lam = aos(m, w)
    assert rel(X.grad.cpu().numpy(), orc.coord_vjp(g["U"], lam, ops, flow)) < TOL
    ref_pb = orc.back_pressure_vjp(g["U"], lam, ops, flow)
    assert abs(float(pb.grad) - ref_pb) <= TOL * max(abs(ref_pb), 1.0)


def test_published_gradients(cuda):
    """Smooth contour, p = 1, refine 0, back pressure 0.15, tolerance 1e-11 (docs/validation/gradients.md:13-28)."""
    ad = pkg("adjoint")
    dc = ad.differentiable_case(contour="smooth", order=1, refine=0, back_pressure_ratio=0.15, tolerance=1e-11)
    names = ("area_ratio", "throat_x", "theta_exit", "inlet_half_height", "back_pressure", "length")
    value, grad, fwd = dc.value_and_gradient("thrust", names=names)
    assert fwd.converged
    assert abs(value - 0.0458513361) < 1e-10
    published = {"area_ratio": 9.772082e-03, "throat_x": -1.490300e-02, "theta_exit": 7.602688e-03,
                 "inlet_half_height": -1.524949e+00, "back_pressure": 0.0, "length": 1.353855e-2}
    for k, v in published.items():
        assert abs(grad[k] - v) <= 1e-6 * abs(v) + 1e-12, (k, grad[k], v)


def bezier8_members(n, sigma=0.02, seed=0):
    """Eight radial wall offsets per member, Gaussian with sigma (a fraction of the throat half-height)."""
    rng = np.random.default_rng(seed)
    return [{f"offset_{k}": float(v) for k, v in enumerate(rng.normal(0.0, sigma, 8))} for _ in range(n)]


def test_batched_gradients_match_one_at_a_time(cuda):
    ad = pkg("adjoint")
    dc = ad.differentiable_case(contour="smooth", order=1, refine=0, back_pressure_ratio=0.15, tolerance=1e-11)
    members = [{"area_ratio": a, "throat_x": 0.1388} for a in (2.3, 2.5, 2.7)]
    out = ad.BatchGradient(dc, members, "thrust").run()
    for m, r in zip(members, out):
        assert r.forward_status == "converged" and r.adjoint_converged
        value, grad, fwd = dc.value_and_gradient("thrust", m, names=tuple(m))
        assert fwd.iterations == r.forward_iterations
        assert abs(r.value - value) <= 1e-12 * abs(value)
        for k in m:
            assert abs(r.grad[k] - grad[k]) <= 1e-7 * max(abs(grad[k]), 1e-8), (k, r.grad[k], grad[k])


def test_overlapped_batch_gradients_equal_the_phased_ones(cuda):
    """Members whose forward solves converge early start their adjoint marches while the others' forward
    solves go on (overlap=True); every value, gradient and iteration count is the same, bit for bit, as
    with every forward solve finished first.  The members' forward solves converge at different
    iterations."""
    ad = pkg("adjoint")
    dc = ad.differentiable_case(contour="smooth", order=1, refine=0, back_pressure_ratio=0.15, tolerance=1e-11,
                                max_iterations=9000)
    members = [{"area_ratio": a, "throat_x": 0.1388} for a in (1.6, 2.0, 2.5, 3.2, 3.9)]
    a = ad.BatchGradient(dc, members, "thrust", variants="single").run(overlap=True)
    b = ad.BatchGradient(dc, members, "thrust", variants="single").run(overlap=False)
    # the batch context (tail switch to the single-solve variants) agrees to round-off
    c = ad.BatchGradient(dc, members, "thrust").run(overlap=True)
    for ra, rc in zip(a, c):
        assert ra.forward_iterations == rc.forward_iterations and ra.adjoint_converged == rc.adjoint_converged
        if ra.grad is not None:
            for k in ra.grad:
                assert abs(rc.grad[k] - ra.grad[k]) <= 1e-9 * max(abs(ra.grad[k]), 1e-8)
    assert len({r.forward_iterations for r in a}) > 1
    for ra, rb in zip(a, b):
        assert (ra.forward_status, ra.forward_iterations, ra.adjoint_converged, ra.adjoint_iterations) == \
               (rb.forward_status, rb.forward_iterations, rb.adjoint_converged, rb.adjoint_iterations)
        assert ra.value == rb.value or (ra.value != ra.value and rb.value != rb.value)
        assert ra.grad == rb.grad


def test_bezier8_shape_gradient_matches_the_reference_fd(cuda):
    """Config 4: eight-offset wall, AR 2.5, p = 2 triangles, refine 2, AUSM+-up.

    The adjoint gradient of thrust w.r.t. all eight offsets against central
    differences (h = 1e-6) of the reference's own forward solver
    (tests/golden/config4_fd.json, made by make_golden.py with the eight-offset
    wall patched into the reference in the generating process only; its forward
    solves converged to a scaled residual of 1e-12).  Both the forward
    tolerance and the differences' own noise (a converged thrust to ~1e-13
    over 2h) limit the agreement to about 1e-5 of the largest component.
    """
    import json

    from conftest import GOLDEN

    ad = pkg("adjoint")
    with open(os.path.join(GOLDEN, "config4_fd.json")) as fh:
        ref = json.load(fh)
    c = ref["case"]
    dc = ad.differentiable_case(contour="bezier8", area_ratio=c["area_ratio"], order=c["order"], refine=c["refine"],
                                flux=c["flux"], back_pressure_ratio=c["back_pressure_ratio"], tolerance=1e-12,
                                offsets=tuple(ref["offsets"]))
    names = tuple(f"offset_{k}" for k in range(8))
    value, grad, fwd = dc.value_and_gradient("thrust", names=names, adjoint_tolerance=1e-10)
    assert fwd.converged
    assert abs(value - ref["thrust"]) <= 1e-9 * abs(ref["thrust"])
    fd = np.asarray(ref["gradient"])
    adj = np.array([grad[k] for k in names])
    scale = np.abs(fd).max()
    assert np.abs(adj - fd).max() <= 2e-5 * scale, (adj, fd)
