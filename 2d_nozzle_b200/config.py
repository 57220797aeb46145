"""Operating point, march options and the step-size rule.

The backend reads flow and option objects by attribute name only, so it works
with the reference's ``FlowConditions`` / ``SolverOptions``
(src/config.py:44-419) or with the stand-ins here, which carry the same field
names and defaults for machines where the reference is not installed.

The step-size constants restate src/timestepping/step.py:34-183: the measured
stability limits, the fallback growth rule above the measured orders, the 30%
margin, ``euler`` at ``p = 0`` and ``ssprk3`` above, and
``dt_e = cfl / (2p + 1) * 2 A_e / max(sum_f s_f l_f, 1e-10)``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, replace

FLUXES = ("roe", "hllc", "ausmup")
FLUX_IDS = {"roe": 0, "hllc": 1, "ausmup": 2}
SCHEMES = ("euler", "ssprk3")
FLOOR = 1e-10

_STABILITY = {"ssprk3": (1.437, 2.337, 2.240), "euler": (1.169, 1.337, 0.775)}
_FALLBACK = {"ssprk3": ("grow", 1.32), "euler": ("flat", 0.70)}
CFL_MARGIN = 0.7


@dataclass(frozen=True)
class FlowConditions:
    gamma: float = 1.4
    Rgas: float = 0.4
    total_temperature: float = 1.0
    total_pressure: float = 1.0
    back_pressure_ratio: float = 0.15
    inflow_angle: float = 0.0
    entropy_fix: float = 0.05
    flux: str = "roe"
    hllc_low_mach: float = 0.0
    backflow: bool = False
    allow_shock_in_nozzle: bool = False

    def __post_init__(self):
        if self.flux not in FLUXES:
            raise ValueError(f"flux must be one of {sorted(FLUXES)}, got {self.flux!r}")
        if self.gamma <= 1.0:
            raise ValueError("gamma must exceed 1")

    @property
    def back_pressure(self) -> float:
        return self.back_pressure_ratio * self.total_pressure

    @property
    def stagnation_sound_speed(self) -> float:
        return math.sqrt(self.gamma * self.Rgas * self.total_temperature)

    @property
    def stagnation_density(self) -> float:
        return self.gamma * self.total_pressure / self.stagnation_sound_speed**2

    def replace(self, **kw) -> FlowConditions:
        return replace(self, **kw)


@dataclass(frozen=True)
class SolverOptions:
    cfl: float | None = None
    tolerance: float = 1e-6
    max_iterations: int = 200_000
    scheme: str | None = None
    limiter: str = "positivity"
    tvb_constant: float = 50.0
    positivity_cfl: float = 0.0
    initial_condition: str = "quasi1d"
    p_continuation: bool = False
    check_interval: int = 50
    print_interval: int = 500
    divergence_factor: float = 1e4
    stall_window: int = 40
    stall_ratio: float = 0.98

    def __post_init__(self):
        if self.scheme is not None and self.scheme not in SCHEMES:
            raise ValueError(f"unknown scheme {self.scheme!r}; choose from {SCHEMES}")
        if self.limiter not in ("none", "positivity", "superbee"):
            raise ValueError(f"unknown limiter {self.limiter!r}")

    def replace(self, **kw) -> SolverOptions:
        return replace(self, **kw)


def recommended_scheme(order: int) -> str:
    return "euler" if order < 1 else "ssprk3"


def stability_limit(order: int, scheme: str = "ssprk3") -> float:
    if scheme not in _STABILITY:
        raise ValueError(f"unknown scheme {scheme!r}; choose from {tuple(_STABILITY)}")
    table = _STABILITY[scheme]
    if order < len(table):
        return table[order]
    rule, k = _FALLBACK[scheme]
    return k if rule == "flat" else k * (2 * order + 1) / (order + 1)


def step_coefficient(order: int, cfl: float | None, scheme: str = "ssprk3") -> float:
    if cfl is None:
        cfl = CFL_MARGIN * stability_limit(order, scheme)
    return cfl / (2 * order + 1)


def component_weights(flow) -> tuple[float, float, float, float]:
    """``(1, 1/a_t, 1/a_t, 1/a_t^2)`` (src/backends/base.py:42-78)."""
    a_t = flow.stagnation_sound_speed
    return (1.0, 1.0 / a_t, 1.0 / a_t, 1.0 / a_t**2)


def residual_scale(flow, length: float) -> float:
    return float(flow.stagnation_density * flow.stagnation_sound_speed / max(length, 1e-30))
