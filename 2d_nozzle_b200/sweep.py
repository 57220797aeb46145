"""Design sweeps: sample operating points, refuse the shocked band, solve as a batch.

The sampled sweep of the benchmark: area ratio uniform in
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


def build_instances(points, *, flux="hllc", tolerance=1e-10, max_iterations=200_000, contour="bell", lean=True):
    """``(instances, index, refused)``: cases of the shock-free points, their point index, refused indices.

    ``lean`` (the default) builds only what the host must -- topology, node coordinates, the quasi-1D
    solution -- and leaves the metric terms and the projected initial state to the device
    (``BatchSolver`` runs ``nzb_geometry`` and ``nzb_initial_state``); ``lean=False`` builds the
    reference's full operators and initial state on the host, as its ``build_case`` does."""
    opts = SolverOptions(tolerance=tolerance, max_iterations=max_iterations, limiter="positivity", print_interval=0)
    instances, index, refused = [], [], []
    for k, pt in enumerate(points):
        flow = FlowConditions(flux=flux, back_pressure_ratio=pt.back_pressure_ratio)
        try:
            cs = build_case(element=pt.element, order=pt.order, refine=pt.refine, area_ratio=pt.area_ratio,
                            contour=contour, flow=flow, options=opts, lean=lean)
        except ShockInNozzle:
            refused.append(k)
            continue
        U0 = None if lean else cs.initial_state()
        instances.append(Instance(cs.operators, flow, opts, U0, cs.geometry.length, cs.geometry))
        index.append(k)
    return instances, index, refused


PARAMETERS = ("area_ratio", "back_pressure_ratio", "order", "refine")
METRICS = ("thrust", "thrust_wall", "thrust_imbalance", "thrust_coefficient", "mass_flow_in", "mass_flow_out",
           "mass_imbalance", "entropy_error", "exit_mach", "exit_pressure_ratio", "exit_temperature_ratio",
           "specific_thrust", "specific_thrust_ratio", "discharge_coefficient", "ideal_thrust", "thrust_efficiency")


@dataclass
class SweepResult:
    """Tabulated outcomes of a sweep, indexed like the reference's (src/sweep.py:68-140).

    ``result["thrust"]`` (a metric, NaN where a point did not converge) or
    ``result["area_ratio"]`` (a swept parameter) give arrays aligned with
    ``points``; ``status`` is each point's march outcome ("refused" for a point
    in the shocked band), ``iterations`` its step count.
    """

    points: list
    values: dict
    converged: np.ndarray
    status: list
    iterations: np.ndarray
    messages: list
    solver: object = None

    def __getitem__(self, key: str) -> np.ndarray:
        if key in self.values:
            return self.values[key]
        if key in PARAMETERS:
            return np.asarray([getattr(p, key) for p in self.points])
        raise KeyError(f"{key!r} is neither a swept parameter {PARAMETERS} nor a metric; metrics are {tuple(self.values)}")

    @property
    def n_points(self) -> int:
        return len(self.points)

    @property
    def all_converged(self) -> bool:
        return bool(np.all(self.converged))

    def failures(self) -> list:
        """The points that did not converge, with the reason."""
        return [(p, m) for p, m, ok in zip(self.points, self.messages, self.converged) if not ok]

    def table(self, metrics=("thrust_coefficient", "exit_mach", "entropy_error")) -> str:
        cols = list(PARAMETERS) + list(metrics) + ["ok"]
        head = "  ".join(f"{c:>18s}" for c in cols)
        lines = [head, "-" * len(head)]
        for i, pt in enumerate(self.points):
            row = [f"{float(getattr(pt, p)):18.6g}" for p in PARAMETERS]
            row += [f"{self.values[m][i]:18.6g}" for m in metrics]
            row.append(f"{'yes' if self.converged[i] else 'NO':>18s}")
            lines.append("  ".join(row))
        return "\n".join(lines)

    def to_csv(self, path: str) -> None:
        cols = list(PARAMETERS) + ["element"] + list(self.values) + ["converged", "status", "iterations"]
        with open(path, "w", encoding="utf-8") as fh:
            fh.write(",".join(cols) + "\n")
            for i, pt in enumerate(self.points):
                row = [repr(getattr(pt, p)) for p in PARAMETERS] + [pt.element]
                row += [repr(float(self.values[m][i])) for m in self.values]
                row += [str(bool(self.converged[i])), self.status[i], str(int(self.iterations[i]))]
                fh.write(",".join(row) + "\n")


def run_sweep(points, device=None, **kw) -> SweepResult:
    """Every point of ``points`` marched in one batch; metrics of the converged points from the device."""
    instances, index, refused = build_instances(points, **kw)
    n = len(points)
    values = {m: np.full(n, np.nan) for m in METRICS}
    converged = np.zeros(n, bool)
    status = ["refused"] * n
    iterations = np.zeros(n, np.int64)
    messages = ["back pressure stands a normal shock inside the nozzle"] * n
    solver = None
    if instances:
        solver = BatchSolver(instances, device=device)
        solver.run()
        perf = solver.observables()
        for k, r, pf in zip(index, solver.results(with_state=False), perf):
            converged[k], status[k], iterations[k] = r.converged, r.status, r.iterations
            messages[k] = "" if r.converged else r.status
            if r.converged:
                for m in METRICS:
                    values[m][k] = pf.get(m, np.nan)
    return SweepResult(list(points), values, converged, status, iterations, messages, solver)
