"""p-continuation host logic: change_order against the reference's projections, the stage plan."""

from __future__ import annotations

import pytest

from conftest import golden, pkg, rel


@pytest.mark.parametrize("kind", ["tri", "quad"])
def test_change_order_matches_the_reference(kind):
    g = golden("change_order.npz")
    nz, co = pkg("nozzle"), pkg("continuation")
    cases = {q: nz.build_case(contour="smooth", element=kind, order=q, refine=0) for q in (0, 1, 2, 3)}
    for a in (0, 1, 2, 3):
        U = g[f"{kind}_U{a}"]
        assert rel(cases[a].initial_state(), U) < 1e-12
        for b in (0, 1, 2, 3):
            if a != b:
                out = co.change_order(U, cases[a].operators, cases[b].operators)
                assert rel(out, g[f"{kind}_{a}to{b}"]) < 1e-12, (a, b)


def test_raising_the_order_is_exact():
    nz, co = pkg("nozzle"), pkg("continuation")
    lo = nz.build_case(contour="smooth", element="tri", order=1, refine=0)
    hi = nz.build_case(contour="smooth", element="tri", order=3, refine=0)
    U1 = lo.initial_state()
    back = co.change_order(co.change_order(U1, lo.operators, hi.operators), hi.operators, lo.operators)
    assert rel(back, U1) < 1e-13


def test_stage_plan():
    cfg, co = pkg("config"), pkg("continuation")
    on = cfg.SolverOptions(p_continuation=True, tolerance=1e-10)
    assert co.stage_orders(3, on, warm=False) == [0, 1, 2, 3]
    assert co.stage_orders(3, on, warm=True) == [3]
    assert co.stage_orders(2, cfg.SolverOptions(), warm=False) == [2]
    assert co.stage_options(on, 1, 3).tolerance == 1e-4
    assert co.stage_options(on, 3, 3).tolerance == 1e-10
    assert co.stage_options(on.replace(tolerance=1e-3), 0, 3).tolerance == 1e-3


def test_mesh_mismatch_raises():
    nz, co = pkg("nozzle"), pkg("continuation")
    a = nz.build_case(contour="smooth", element="tri", order=1, refine=0)
    b = nz.build_case(contour="smooth", element="tri", order=2, refine=1)
    with pytest.raises(ValueError, match="same mesh"):
        co.change_order(a.initial_state(), a.operators, b.operators)


class _FakeBatch:
    """Stands in for BatchSolver on the host: records each batch, 'converges' every instance at once."""

    made: list = []

    def __init__(self, instances, device=None):
        self.instances = instances
        _FakeBatch.made.append([(i.ops.ref.order, i.flow.flux, i.opts.tolerance) for i in instances])

    def run(self):
        return 1

    def results(self, with_state=True):
        from types import SimpleNamespace

        return [SimpleNamespace(U=i.U0, converged=True, iterations=10 * (i.ops.ref.order + 1), residual=0.0,
                                status="converged") for i in self.instances]


def test_batched_stages_group_by_flux_and_sum_iterations(monkeypatch):
    nz, cfg, co = pkg("nozzle"), pkg("config"), pkg("continuation")
    monkeypatch.setattr(pkg("batch"), "BatchSolver", _FakeBatch)
    _FakeBatch.made = []
    on = cfg.SolverOptions(p_continuation=True, tolerance=1e-9)
    cases = [nz.build_case(element="tri", order=2, refine=0, contour="smooth", options=on,
                           flow=cfg.FlowConditions(flux=f)) for f in ("roe", "hllc")]
    cases.append(nz.build_case(element="quad", order=1, refine=0, contour="smooth", options=on,
                               flow=cfg.FlowConditions(flux="hllc")))
    warm = [None, None, cases[2].initial_state()]  # the third starts warm: its target order only
    got = co.solve_batch(cases, warm_starts=warm)
    assert [r.orders for r in got] == [[0, 1, 2], [0, 1, 2], [1]]
    assert [r.iterations for r in got] == [10 + 20 + 30, 10 + 20 + 30, 20]
    # stage 0: roe alone, then hllc (tri p0) with the warm quad (target order, its own tolerance)
    assert _FakeBatch.made[0] == [(0, "roe", 1e-4)]
    assert _FakeBatch.made[1] == [(0, "hllc", 1e-4), (1, "hllc", 1e-9)]
    assert _FakeBatch.made[-1] == [(2, "hllc", 1e-9)]
    assert all(r.converged for r in got) and got[0].operators.ref.order == 2
