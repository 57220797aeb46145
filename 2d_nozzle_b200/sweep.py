"""Design sweeps: sample operating points, refuse the shocked band, solve as a batch.

The sampled sweep is BASELINE's batched design sweep: area ratio uniform in
[1.5, 4.0], back-pressure ratio uniform in [0.1, 0.9], order uniform over
{1, 2, 3}, refinement uniform over {1, 2, 3}, triangles and quadrilaterals
50/50, HLLC with the positivity limiter, tolerance 1e-10.  A point whose back
pressure stands a normal shock in the diverging section is refused and
recorded, as the reference's sweep does (src/sweep.py:233-265, src/api.py:
320-334); every other point is built on the host (:mod:`.nozzle`) and all of
them are marched together by :class:`~.batch.BatchSolver`.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .batch import BatchSolver, Instance
from .config import FlowConditions, SolverOptions
from .nozzle import ShockInNozzle, build_case


@dataclass
class Point:
    area_ratio: float
    back_pressure_ratio: float
    order: int
    refine: int
    element: str


def sample_points(n=256, seed=0) -> list[Point]:
    rng = np.random.default_rng(seed)
    ar = rng.uniform(1.5, 4.0, n)
    pb = rng.uniform(0.1, 0.9, n)
    order = rng.integers(1, 4, n)
    refine = rng.integers(1, 4, n)
    quad = rng.random(n) < 0.5
    return [Point(float(a), float(b), int(p), int(r), "quad" if q else "tri")
            for a, b, p, r, q in zip(ar, pb, order, refine, quad)]


def build_instances(points, *, flux="hllc", tolerance=1e-10, max_iterations=200_000, contour="bell"):
    """``(instances, index, refused)``: cases of the shock-free points, their point index, refused indices."""
    opts = SolverOptions(tolerance=tolerance, max_iterations=max_iterations, limiter="positivity", print_interval=0)
    instances, index, refused = [], [], []
    for k, pt in enumerate(points):
        flow = FlowConditions(flux=flux, back_pressure_ratio=pt.back_pressure_ratio)
        try:
            cs = build_case(element=pt.element, order=pt.order, refine=pt.refine, area_ratio=pt.area_ratio,
                            contour=contour, flow=flow, options=opts)
        except ShockInNozzle:
            refused.append(k)
            continue
        instances.append(Instance(cs.operators, flow, opts, cs.initial_state(), cs.geometry.length, cs.geometry))
        index.append(k)
    return instances, index, refused


def run_sweep(points, device=None, **kw):
    instances, index, refused = build_instances(points, **kw)
    solver = BatchSolver(instances, device=device)
    solver.run()
    return solver, index, refused
