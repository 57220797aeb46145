"""The pseudo-time march to steady state, driving any backend through ``run``.

Restates ``march`` (src/timestepping/march.py:125-230) so a steady solve can run
where the reference is not installed; where it is, the reference's own
``solve_nozzle(..., backend=...)`` drives :class:`~.backend.B200Backend`
through exactly the same calls.  The bookkeeping must match the reference's to
reproduce its iteration counts:

* one step alone first, for the initial residual;
* chunks of ``check_interval`` steps, each a single ``backend.run`` call;
* stop on a non-finite residual, on ``res <= tolerance * rho_t a_t / L``, on
  growth past ``divergence_factor * res0``, on a stall (the best/worst ratio of
  the last ``stall_window`` checks above ``stall_ratio``), or at
  ``max_iterations``;
* a converged state with a non-positive density or pressure at a probe point
  is reported as not converged (src/timestepping/march.py:271-279).
"""

from __future__ import annotations

import math
import time
from dataclasses import dataclass, field

import numpy as np

from .config import residual_scale


@dataclass
class MarchResult:
    U: np.ndarray
    converged: bool
    iterations: int
    residual: float
    residual_initial: float
    residual_scale: float
    message: str = ""
    history_iterations: list = field(default_factory=list)
    history_residual: list = field(default_factory=list)
    wall_time: float = 0.0
    min_density: float = float("nan")
    min_pressure: float = float("nan")
    limiter_activity: float = float("nan")
    mean_repairs: int = 0

    @property
    def residual_scaled(self) -> float:
        return self.residual / self.residual_scale


def march(U, backend, opts, scale: float):
    """Advance to steady state; returns ``(U, its, res, res0, converged, message, hist_it, hist_res)``."""
    chunk = min(max(1, opts.check_interval), opts.max_iterations)
    hist_it, hist_res = [], []
    U, res0 = backend.run(U, 1, backend.scheme)
    done = 1
    hist_it.append(done)
    hist_res.append(float(res0))
    if not math.isfinite(res0):
        return U, done, res0, res0, False, "initial residual is not finite", hist_it, hist_res
    if res0 <= opts.tolerance * scale:
        return U, done, res0, res0, True, "", hist_it, hist_res
    res = res0
    window: list[float] = []
    message = ""
    converged = False
    while done < opts.max_iterations:
        n = min(chunk, opts.max_iterations - done)
        U, res = backend.run(U, n, backend.scheme)
        done += n
        hist_it.append(done)
        hist_res.append(float(res))
        if not math.isfinite(res):
            message = f"residual became non-finite after {done} iterations"
            break
        if res <= opts.tolerance * scale:
            converged = True
            break
        if res > opts.divergence_factor * res0:
            message = f"residual grew by {res / res0:.1e}x after {done} iterations (divergence)"
            break
        window.append(res)
        if len(window) > opts.stall_window:
            window.pop(0)
        if len(window) == opts.stall_window:
            best, worst = min(window), max(window)
            if worst > 0.0 and best / worst > opts.stall_ratio:
                message = f"the residual has stalled at {res / scale:.3e} (scaled)"
                break
    if not converged and not message:
        message = f"hit max_iterations={opts.max_iterations} at scaled residual {res / scale:.2e}"
    return U, done, float(res), float(res0), converged, message, hist_it, hist_res


def probe_minima(U, ops, gamma: float) -> tuple[float, float]:
    """Minimum density and pressure over the volume and own-face points (unlimited)."""
    U = np.asarray(U)
    vol = np.einsum("iq,eis->eqs", ops.ref.phi_vol, U)
    ed = ops.topology.edges
    nface = ed.face_edge.shape[1]
    fb = ops.ref.phi_face[ed.face_side, np.arange(nface)[None, :]]
    face = np.einsum("efiq,eis->efqs", fb, U).reshape(U.shape[0], -1, 4)
    pr = np.concatenate([vol, face], axis=1)
    rho = pr[..., 0]
    p = (gamma - 1.0) * (pr[..., 3] - 0.5 * (pr[..., 1] ** 2 + pr[..., 2] ** 2) / np.where(rho != 0.0, rho, 1.0))
    return float(rho.min()), float(p.min())


def solve(backend, U0, *, length: float = 1.0) -> MarchResult:
    """Steady solve from ``U0`` with the backend's operators, flow and options."""
    opts = backend.opts
    scale = residual_scale(backend.flow, length)
    t0 = time.perf_counter()
    U, its, res, res0, conv, msg, hi, hr = march(np.asarray(U0, float), backend, opts, scale)
    wall = time.perf_counter() - t0
    rmin, pmin = probe_minima(U, backend.ops, backend.flow.gamma)
    if conv and (rmin <= 0.0 or pmin <= 0.0):
        conv = False
        msg = f"residual converged but the solution is not physical (min rho {rmin:.3e}, min p {pmin:.3e})"
    return MarchResult(U, conv, its, res, res0, scale, msg, hi, hr, wall, rmin, pmin,
                       backend.limiter_activity(), int(backend.n_mean_repaired))
