"""The batched L-BFGS-B driver on a known objective (no GPU): lockstep batches, unchanged iterates."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.optimize import minimize

from conftest import pkg

CENTRE = np.array([0.7, -0.2, 1.5])
BOUNDS = [(-2.0, 2.0), (-2.0, 2.0), (-2.0, 1.0)]


def coupled_bowl(x):
    d = x - CENTRE
    return float(d @ d + 0.5 * d[0] ** 2 * d[1] ** 2), 2.0 * d + np.array([d[0] * d[1] ** 2, d[0] ** 2 * d[1], 0.0])


def test_every_start_follows_its_own_run():
    opt = pkg("optimise")
    starts = [np.zeros(3), np.array([1.9, 1.9, -1.9]), np.array([-1.0, 0.5, 0.2]), np.array([0.7, -0.2, 0.0])]
    sizes, calls = [], []

    def evaluate(xs):
        calls.append(len(xs))
        return [coupled_bowl(x) for x in xs]

    got = opt.minimize_batch(evaluate, starts, BOUNDS, maxiter=50, ftol=1e-14, batch_sizes=sizes)
    assert sizes == calls and sizes[0] == len(starts) and sum(sizes) == sum(r.nfev for r in got)
    assert sorted(sizes, reverse=True) == sizes  # optimisations only ever leave the batch
    for x0, r in zip(starts, got):
        alone = minimize(coupled_bowl, x0, jac=True, method="L-BFGS-B", bounds=BOUNDS,
                         options={"maxiter": 50, "ftol": 1e-14})
        assert np.array_equal(r.x, alone.x) and r.nfev == alone.nfev and r.nit == alone.nit
        assert r.success
        assert np.allclose(r.x, [0.7, -0.2, 1.0], atol=1e-6)  # x2 held at its upper bound
        assert len(r.history) == r.nfev


def test_maximise_reports_the_objective_itself():
    opt = pkg("optimise")
    got = opt.minimize_batch(lambda xs: [(-(x @ x), -2.0 * x) for x in xs], [np.array([0.5, -0.5])],
                             [(-1.0, 1.0), (-1.0, 1.0)], maximise=True)
    assert got[0].value == pytest.approx(0.0, abs=1e-12) and np.allclose(got[0].x, 0.0, atol=1e-6)


def test_a_failed_evaluation_ends_every_run():
    opt = pkg("optimise")
    n = [0]

    def evaluate(xs):
        n[0] += 1
        if n[0] == 3:
            raise FloatingPointError("planted")
        return [coupled_bowl(x) for x in xs]

    with pytest.raises(FloatingPointError, match="planted"):
        opt.minimize_batch(evaluate, [np.zeros(3), np.ones(3)], BOUNDS)


def test_optimise_case_batches_members_and_maps_failures(monkeypatch):
    """optimise_case turns each round into one BatchGradient; a failed member evaluates to NaN."""
    from types import SimpleNamespace

    ad, opt = pkg("adjoint"), pkg("optimise")
    seen = []

    class FakeBatch:
        def __init__(self, case, members, objective, names, variants="batch"):
            self.members, self.names = members, names
            seen.append(len(members))

        def run(self, adjoint_tolerance=1e-8):
            out = []
            for m in self.members:
                x = np.array([m[k] for k in self.names])
                if x[0] > 1.9:  # a member whose forward solve fails
                    out.append(SimpleNamespace(value=float("nan"), grad=None))
                else:
                    out.append(SimpleNamespace(value=float(-(x - 0.5) @ (x - 0.5)),
                                               grad={k: float(-2.0 * (v - 0.5)) for k, v in zip(self.names, x)}))
            return out

    monkeypatch.setattr(ad, "BatchGradient", FakeBatch)
    got = opt.optimise_case(None, [np.array([0.0, 1.0]), np.array([1.95, 0.0])], ("a", "b"),
                            [(-2.0, 2.0), (-2.0, 2.0)], maxiter=20)
    assert seen[0] == 2 and sum(seen) == len(got[0].history) + len(got[1].history)
    assert np.allclose(got[0].x, [0.5, 0.5], atol=1e-5) and got[0].value == pytest.approx(0.0, abs=1e-9)
    assert not np.isfinite(got[1].history[0][1]) and not (got[1].success and np.isfinite(got[1].value))
