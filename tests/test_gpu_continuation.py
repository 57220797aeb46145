"""p-continuation on the device against the reference's solve_nozzle(p_continuation=True)."""

from __future__ import annotations

import json

import pytest

from conftest import GOLDEN, pkg, rel

pytestmark = pytest.mark.gpu


def reference_cases():
    nz, cfg = pkg("nozzle"), pkg("config")
    out = []
    for row in json.load(open(f"{GOLDEN}/continuation_cases.json")):
        el, p, r, ar, pb, contour, flux = row["case"]
        opts = cfg.SolverOptions(tolerance=1e-8, max_iterations=30000, p_continuation=True, print_interval=0)
        flow = cfg.FlowConditions(flux=flux, back_pressure_ratio=pb)
        out.append((nz.build_case(element=el, order=p, refine=r, area_ratio=ar, contour=contour, flow=flow,
                                  options=opts), row))
    return out


def check(res, cs, row):
    assert res.converged == row["converged"], res.message
    assert res.iterations == row["iterations"]
    assert res.orders == list(range(cs.operators.ref.order + 1))
    perf = pkg("observables").performance(res.U, cs.operators, cs.flow)
    for key in ("thrust", "mass_flow_in", "exit_mach"):
        assert rel(perf[key], row[key]) < 1e-9, key


def test_single_solves_match_the_reference(cuda):
    for cs, row in reference_cases():
        check(pkg("continuation").solve_case(cs), cs, row)


def test_batched_continuation_matches_the_reference(cuda):
    cases = reference_cases()
    got = pkg("continuation").solve_batch([cs for cs, _ in cases])
    for (cs, row), res in zip(cases, got):
        check(res, cs, row)


def test_warm_start_runs_the_target_order_only(cuda):
    cs, row = reference_cases()[0]
    first = pkg("continuation").solve_case(cs)
    again = pkg("continuation").solve_case(cs, U0=first.U)
    assert again.orders == [cs.operators.ref.order] and again.converged
    assert again.iterations < 200
