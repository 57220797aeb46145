"""Many gradient-based shape optimisations at once, their evaluations batched on the device.

Restates examples/04_optimise.py:32-64 -- maximise an objective (thrust) over
named design variables with L-BFGS-B (``scipy.optimize.minimize``,
``jac=True``, box bounds), every evaluation one forward solve plus one adjoint
solve -- for several optimisations together: several starting points of one
case, as a multi-start search does.

Each optimisation runs scipy's L-BFGS-B unchanged in a host thread of its own.
Its objective hands the design point to the batcher and waits; whenever every
running optimisation is waiting, the batcher evaluates all pending points in
one go -- for the adjoint case one :class:`~.adjoint.BatchGradient` (one
batched forward march, one batched adjoint march, one coordinate-VJP launch)
-- and hands each its value and gradient.  The optimisations never see each
other: each follows exactly the iterates it would follow alone, and an
evaluation's result does not depend on what else shares its batch.
"""

from __future__ import annotations

import threading
from dataclasses import dataclass, field

import numpy as np


@dataclass
class OptimisationResult:
    x: np.ndarray
    value: float  # the objective at x (maximised when the run maximises)
    success: bool
    message: str
    nit: int
    nfev: int
    history: list = field(default_factory=list)  # (x, value) of every evaluation, in order


def minimize_batch(evaluate, starts, bounds, *, maximise=False, maxiter=25, ftol=1e-10, batch_sizes=None):
    """L-BFGS-B from every start, the evaluations of each round batched.

    ``evaluate(xs)`` takes a list of points and returns a list of ``(value,
    gradient)``.  ``batch_sizes`` (a list), if given, records the size of every
    batch evaluated.  An exception from ``evaluate`` ends every optimisation
    and is raised to the caller.
    """
    from scipy.optimize import minimize

    n = len(starts)
    sign = -1.0 if maximise else 1.0
    cond = threading.Condition()
    pending: dict[int, np.ndarray] = {}
    answers: dict[int, tuple] = {}
    live = set(range(n))
    runs = [None] * n
    errors = [None] * n
    history = [[] for _ in range(n)]
    failure: list[BaseException] = []

    def objective(i, x):
        with cond:
            if failure:
                raise RuntimeError("a batched evaluation failed") from failure[0]
            pending[i] = np.array(x, dtype=float)
            cond.notify_all()
            cond.wait_for(lambda: i in answers or bool(failure))
            if i not in answers:
                raise RuntimeError("a batched evaluation failed") from failure[0]
            value, grad = answers.pop(i)
        history[i].append((np.array(x, dtype=float), float(value)))
        return sign * float(value), sign * np.asarray(grad, dtype=float)

    def worker(i):
        try:
            runs[i] = minimize(lambda x: objective(i, x), np.asarray(starts[i], dtype=float), jac=True,
                               method="L-BFGS-B", bounds=bounds, options={"maxiter": maxiter, "ftol": ftol})
        except BaseException as exc:  # reported to the caller below
            errors[i] = exc
        finally:
            with cond:
                live.discard(i)
                cond.notify_all()

    threads = [threading.Thread(target=worker, args=(i,), daemon=True) for i in range(n)]
    for t in threads:
        t.start()
    while True:
        with cond:
            cond.wait_for(lambda: len(pending) == len(live))
            if not live:
                break
            batch = sorted(pending.items())
            pending.clear()
        if batch_sizes is not None:
            batch_sizes.append(len(batch))
        try:
            got = evaluate([x for _, x in batch])
        except BaseException as exc:
            # every waiting optimisation raises in its own thread and ends
            with cond:
                failure.append(exc)
                cond.notify_all()
            for t in threads:
                t.join()
            raise
        with cond:
            for (i, _), vg in zip(batch, got):
                answers[i] = vg
            cond.notify_all()
    for t in threads:
        t.join()
    for e in errors:
        if e is not None:
            raise e
    return [OptimisationResult(np.asarray(r.x), sign * float(r.fun), bool(r.success), str(r.message), int(r.nit),
                               int(r.nfev), history[i]) for i, r in enumerate(runs)]


def optimise_case(case, starts, names, bounds, *, objective="thrust", maximise=True, maxiter=25, ftol=1e-10,
                  adjoint_tolerance=1e-8, batch_sizes=None, variants="batch"):
    """Shape optimisations of a :class:`~.adjoint.DifferentiableCase` from several starting points.

    ``starts``: points (one value per name in ``names``); each evaluation is the
    objective and its adjoint gradient with respect to ``names``.  A member
    whose forward solve fails evaluates to NaN, which L-BFGS-B reports as a
    failed run (its result's ``success`` is false or its value not finite).
    """
    from .adjoint import BatchGradient

    names = tuple(names)

    def evaluate(xs):
        members = [dict(zip(names, map(float, x))) for x in xs]
        res = BatchGradient(case, members, objective, names, variants=variants).run(adjoint_tolerance=adjoint_tolerance)
        out = []
        for r in res:
            if r.grad is None:
                out.append((float("nan"), np.full(len(names), np.nan)))
            else:
                out.append((float(r.value), np.array([r.grad[k] for k in names])))
        return out

    return minimize_batch(evaluate, starts, bounds, maximise=maximise, maxiter=maxiter, ftol=ftol,
                          batch_sizes=batch_sizes)
