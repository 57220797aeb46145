"""The Superbee TVB slope limiter (then positivity) on the device, against the reference's fixtures."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, pkg, rel, tiny_ops
from oracle import dg_oracle as orc

pytestmark = pytest.mark.gpu
CASES = [("tri", 1), ("tri", 2), ("tri", 3), ("quad", 1), ("quad", 2), ("quad", 3)]


def backend(ops, **opt):
    cfg = pkg("config")
    return pkg("backend").B200Backend(ops, cfg.FlowConditions(), cfg.SolverOptions(limiter="superbee", **opt))


@pytest.mark.parametrize("kind,p", CASES)
def test_superbee_limit_matches_the_reference(cuda, kind, p):
    ops, _ = tiny_ops(kind, p)
    g = golden(f"superbee_{kind}_p{p}.npz")
    bk = backend(ops)
    out = bk.limit(g["U"])
    assert rel(out, g["superbee_positivity"]) < 1e-12
    ref, _ = orc.superbee(g["U"], ops, 50.0)
    assert rel(out, orc.positivity(ref, ops, pkg("config").FlowConditions())[0]) < 1e-12


@pytest.mark.parametrize("kind,p", CASES)
def test_superbee_ssprk3_steps_match_the_reference(cuda, kind, p):
    ops, _ = tiny_ops(kind, p)
    g = golden(f"superbee_{kind}_p{p}.npz")
    bk = backend(ops, scheme="ssprk3")
    V, res = bk.run(g["U"], 3, "ssprk3")
    assert rel(V, g["run3_ssprk3"]) < 1e-11
    assert abs(res - g["run3_ssprk3_res"]) <= 1e-11 * abs(g["run3_ssprk3_res"])


def _superbee_cases(max_it):
    nz, cfg = pkg("nozzle"), pkg("config")
    opts = cfg.SolverOptions(tolerance=1e-8, max_iterations=max_it, limiter="superbee", print_interval=0)
    spec = [("tri", 1, 0, 2.5, 0.15), ("tri", 2, 0, 1.8, 0.30), ("tri", 3, 0, 2.2, 0.10),
            ("quad", 1, 0, 3.0, 0.20), ("quad", 2, 0, 2.5, 0.15), ("tri", 1, 1, 2.0, 0.12)]
    out = []
    for el, p, r, ar, pb in spec:
        flow = cfg.FlowConditions(flux="hllc", back_pressure_ratio=pb)
        cs = nz.build_case(element=el, order=p, refine=r, area_ratio=ar, contour="bell", flow=flow, options=opts)
        out.append(pkg("batch").Instance(cs.operators, flow, opts, cs.initial_state(), cs.geometry.length, cs.geometry))
    return out


def test_superbee_batch_matches_one_at_a_time(cuda):
    """Each instance of a batch is limited against its own domain (its own maximum of the cell
    averages and area shares): the batch reproduces every one-at-a-time march, status, iteration
    count and state.  A NaN planted on the host in one instance's initial state retires it at the
    first check without disturbing the others (its elements stay out of the maxima and the passes)."""
    insts = _superbee_cases(600)
    bad = _superbee_cases(600)[0]
    U0 = bad.U0.copy()
    U0[3, 1, 0] = np.nan
    bad.U0 = U0
    solver = pkg("batch").BatchSolver(insts + [bad], variants="single")
    solver.run()
    got = solver.results()
    assert got[-1].status == "non-finite" and got[-1].iterations == 1
    for inst, b in zip(insts, got):
        bk = pkg("backend").B200Backend(inst.ops, inst.flow, inst.opts)
        p = pkg("march").solve(bk, inst.U0, length=inst.length)
        assert b.iterations == p.iterations
        assert b.status == ("converged" if p.converged else b.status)
        assert rel(b.U, p.U) < 1e-12
        assert bk.n_limited > 0
