"""Batched multi-start L-BFGS-B on the reference's optimisation example (examples/04_optimise.py:32-64)."""

from __future__ import annotations

import numpy as np
import pytest
from scipy.optimize import minimize

from conftest import pkg

pytestmark = pytest.mark.gpu

NAMES = ("area_ratio", "bezier_w1", "bezier_w2")
BOUNDS = [(1.8, 4.5), (0.05, 0.95), (0.30, 0.99)]


def test_batched_runs_follow_the_one_at_a_time_runs(cuda):
    dc = pkg("adjoint").differentiable_case(contour="bezier", order=1, refine=0, back_pressure_ratio=0.15,
                                            tolerance=1e-10)
    x0 = np.array([dc.default_params()[n] for n in NAMES])
    starts = [x0, np.array([2.2, 0.4, 0.8])]
    sizes = []
    got = pkg("optimise").optimise_case(dc, starts, NAMES, BOUNDS, maxiter=3, batch_sizes=sizes,
                                          variants="single")
    assert sizes[0] == 2
    for x_start, r in zip(starts, got):

        def objective(x):
            value, grad, _ = dc.value_and_gradient("thrust", dict(zip(NAMES, x)), names=NAMES)
            return -value, -np.array([grad[n] for n in NAMES])

        alone = minimize(objective, x_start, jac=True, method="L-BFGS-B", bounds=BOUNDS,
                         options={"maxiter": 3, "ftol": 1e-10})
        assert r.nfev == alone.nfev
        assert np.allclose(r.x, alone.x, rtol=1e-9, atol=0.0)
        assert r.value == pytest.approx(-alone.fun, rel=1e-10)
        assert r.value > r.history[0][1]  # thrust went up
