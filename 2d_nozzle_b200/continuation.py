"""p-continuation and warm starts: one solve, or a batch of them, climbing the orders.

Restates the order loop of ``solve_nozzle`` (src/api.py:358-397) and
``change_order`` (src/timestepping/initialize.py:121-147):

* with ``options.p_continuation`` and no warm start, a solve at order p runs
  the orders 0, 1, ..., p on the same mesh, each from the previous one's state
  re-projected onto the next order's basis, and every order below the target
  only to ``max(tolerance, 1e-4)`` (the transient);
* otherwise only the target order runs, from ``U0`` when given (a warm start,
  e.g. the neighbouring point of a sweep or a line search) or from the
  quasi-1D initial state;
* the reported iterations are the sum over the orders; the state, residual and
  convergence are the last order's.

Every march runs on the device (``B200Backend`` through ``march.solve`` for one
solve, ``BatchSolver`` for many, one bucket per (kind, order) at each stage).
The projection between orders is the host's, once per stage, as in the
reference.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import refelem as re
from .nozzle import project, quasi1d_initial
from .operators import build_operators


def change_order(U, ops_from, ops_to) -> np.ndarray:
    """Re-project ``U (E, NP_from, 4)`` from ``ops_from``'s order onto ``ops_to``'s, same mesh.

    The source solution is evaluated at the target's volume quadrature points
    and L2-projected there; raising the order is exact.
    """
    if ops_from.n_elem != ops_to.n_elem:
        raise ValueError(f"change_order needs the same mesh: {ops_from.n_elem} vs {ops_to.n_elem} elements")
    phi_src, _, _ = re.basis(ops_from.ref.kind, ops_from.ref.order, ops_to.ref.points_vol)
    values = np.einsum("iq,eis->eqs", phi_src, np.asarray(U, float))
    return project(values, ops_to)


def stage_orders(target: int, opts, warm: bool) -> list[int]:
    """The orders a solve marches through (src/api.py:358)."""
    return list(range(target + 1)) if (opts.p_continuation and not warm) else [target]


def stage_options(opts, order: int, target: int):
    """Orders below the target only remove the transient (src/api.py:375-377)."""
    return opts if order == target else opts.replace(tolerance=max(opts.tolerance, 1e-4))


@dataclass
class ContinuationResult:
    U: np.ndarray
    converged: bool
    iterations: int  # summed over the orders
    residual: float
    status: str
    message: str = ""
    orders: list = field(default_factory=list)
    stage_iterations: list = field(default_factory=list)
    operators: object = None


def _stage_operators(cs, order: int, target: int):
    return cs.operators if order == target else build_operators(cs.topology, cs.node_coords, order)


def solve_case(cs, *, U0=None, device=None) -> ContinuationResult:
    """Steady solve of a case built by ``nozzle.build_case`` (its options decide the continuation)."""
    from .backend import B200Backend
    from .march import solve

    opts = cs.options
    target = cs.operators.ref.order
    orders = stage_orders(target, opts, U0 is not None)
    U = None if U0 is None else np.asarray(U0, float)
    prev = None
    its = []
    res = None
    for order in orders:
        ops = _stage_operators(cs, order, target)
        if U is None:
            U = quasi1d_initial(ops, cs.flow, cs.geometry)
        elif prev is not None:
            U = change_order(U, prev, ops)
        bk = B200Backend(ops, cs.flow, stage_options(opts, order, target), device=device)
        res = solve(bk, U, length=cs.geometry.length)
        U, prev = res.U, ops
        its.append(res.iterations)
    status = "converged" if res.converged else (res.message or "not converged")
    return ContinuationResult(res.U, res.converged, int(sum(its)), float(res.residual), status, res.message,
                              orders, its, prev)


def _batch_key(inst):
    f, o = inst.flow, inst.opts
    return (f.gamma, f.flux, f.entropy_fix, f.hllc_low_mach, f.backflow, f.total_pressure, f.total_temperature,
            f.Rgas, f.inflow_angle, o.replace(tolerance=0.0))


def solve_batch(cases, *, warm_starts=None, device=None) -> list[ContinuationResult]:
    """Steady solves of many cases, one batched march per continuation stage.

    At stage k every case whose own order list has a k-th entry marches at that
    order (below its target: to the transient tolerance), in one ``BatchSolver``
    per group of cases that share the gas, the flux and the march options (any
    batch's condition; back pressure and tolerance may differ); between stages
    each state is re-projected onto its next order.
    """
    from .batch import BatchSolver, Instance

    n = len(cases)
    warm = warm_starts if warm_starts is not None else [None] * n
    targets = [cs.operators.ref.order for cs in cases]
    orders = [stage_orders(t, cs.options, w is not None) for t, cs, w in zip(targets, cases, warm)]
    U = [None if w is None else np.asarray(w, float) for w in warm]
    prev = [None] * n
    its = [[] for _ in range(n)]
    last = [None] * n
    for k in range(max(len(o) for o in orders)):
        active = [i for i in range(n) if k < len(orders[i])]
        insts, ops_at = [], {}
        for i in active:
            cs, order = cases[i], orders[i][k]
            ops = _stage_operators(cs, order, targets[i])
            if U[i] is None:
                U[i] = quasi1d_initial(ops, cs.flow, cs.geometry)
            elif prev[i] is not None:
                U[i] = change_order(U[i], prev[i], ops)
            ops_at[i] = ops
            insts.append(Instance(ops, cs.flow, stage_options(cs.options, order, targets[i]), U[i],
                                  float(cs.geometry.length), cs.geometry))
        # one batch per group of cases a batch can hold together: the same gas, flux and march
        # options (back pressure and tolerance may differ per instance)
        groups: dict = {}
        for i, inst in zip(active, insts):
            groups.setdefault(_batch_key(inst), []).append((i, inst))
        for members in groups.values():
            solver = BatchSolver([inst for _, inst in members], device=device)
            solver.run()
            for (i, _), r in zip(members, solver.results(with_state=True)):
                U[i], prev[i] = r.U, ops_at[i]
                its[i].append(r.iterations)
                last[i] = r
            del solver
    return [ContinuationResult(U[i], last[i].converged, int(sum(its[i])), float(last[i].residual), last[i].status,
                               "", orders[i], its[i], prev[i]) for i in range(n)]
