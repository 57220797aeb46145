"""Batched march against the one-at-a-time march, instance by instance (same kernels, same bookkeeping)."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import pkg, rel

pytestmark = pytest.mark.gpu


def cases(tol=1e-8, max_it=6000, cfl=None):
    nz, cfg = pkg("nozzle"), pkg("config")
    opts = cfg.SolverOptions(tolerance=tol, max_iterations=max_it, limiter="positivity", print_interval=0, cfl=cfl)
    spec = [  # element, order, refine, area ratio, back pressure, contour
        ("tri", 1, 0, 2.5, 0.15, "smooth"),
        ("quad", 1, 0, 3.0, 0.995, "bell"),
        ("tri", 2, 0, 1.8, 0.30, "conical"),
        ("tri", 1, 1, 2.2, 0.10, "bell"),
        ("quad", 2, 0, 2.5, 0.15, "bell"),
    ]
    out = []
    for el, p, r, ar, pb, contour in spec:
        flow = cfg.FlowConditions(flux="hllc", back_pressure_ratio=pb)
        cs = nz.build_case(element=el, order=p, refine=r, area_ratio=ar, contour=contour, flow=flow, options=opts)
        out.append(pkg("batch").Instance(cs.operators, flow, opts, cs.initial_state(), cs.geometry.length, cs.geometry))
    return out


def plain(inst):
    bk = pkg("backend").B200Backend(inst.ops, inst.flow, inst.opts)
    return pkg("march").solve(bk, inst.U0, length=inst.length)


def test_batch_matches_one_at_a_time(cuda):
    insts = cases()
    solver = pkg("batch").BatchSolver(insts, variants="single")
    solver.run()
    got = solver.results()
    for inst, b in zip(insts, got):
        p = plain(inst)
        status = "converged" if p.converged else b.status
        assert b.status == status, (b.status, p.message)
        assert b.iterations == p.iterations
        if np.isfinite(p.residual):
            assert abs(b.residual - p.residual) <= 1e-10 * abs(p.residual)
            assert rel(b.U, p.U) < 1e-12
        else:
            assert not np.isfinite(b.residual)


def test_batch_matches_the_reference_outcomes(cuda):
    """Status, iteration count and parity observables against the reference's own solves."""
    import json

    from conftest import GOLDEN

    ref = json.load(open(f"{GOLDEN}/batch_cases.json"))
    insts = cases()
    solver = pkg("batch").BatchSolver(insts)
    solver.run()
    for inst, b, r in zip(insts, solver.results(), ref):
        assert b.iterations == r["iterations"], (r["case"], b.status, r["message"])
        assert b.converged == r["converged"]
        if r["converged"]:
            perf = pkg("observables").performance(b.U, inst.ops, inst.flow)
            for key in ("thrust", "mass_flow_in", "exit_mach"):
                assert abs(perf[key] - r[key]) <= 1e-9 * abs(r[key]), key
        else:
            # a blow-up: the reference's residual is huge or non-finite, as is ours
            assert b.status in ("diverged", "non-finite")


def test_retired_instances_are_frozen(cuda):
    """A failing instance retires without disturbing the others.

    The failure is injected on the host: one instance starts from a state with
    a NaN coefficient, so its first residual is non-finite.
    """
    good = cases()
    insts = [good[0], good[2]]
    bad = cases()[0]
    U0 = bad.U0.copy()
    U0[5, 0, 3] = np.nan
    bad.U0 = U0
    solver = pkg("batch").BatchSolver([insts[0], bad, insts[1]], variants="single")
    solver.run()
    got = solver.results()
    assert got[1].status == "non-finite" and got[1].iterations == 1
    for k, inst in ((0, insts[0]), (2, insts[1])):
        p = plain(inst)
        assert got[k].iterations == p.iterations and rel(got[k].U, p.U) < 1e-12


def test_sampled_sweep_points_and_refusals(cuda):
    sw = pkg("sweep")
    pts = sw.sample_points(64, seed=0)
    nz = pkg("nozzle")
    refused = [k for k, p in enumerate(pts)
               if not nz.is_shock_free(nz.realised_area_ratio(nz.Geometry(area_ratio=p.area_ratio)), p.back_pressure_ratio)]
    assert 0.3 < len(refused) / len(pts) < 0.8
    assert {p.order for p in pts} == {1, 2, 3} and {p.refine for p in pts} == {1, 2, 3}
