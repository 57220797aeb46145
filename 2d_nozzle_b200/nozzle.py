"""Nozzle cases built on the host: contour, mesh, operators, quasi-1D initial state.

A sweep of design points has to be built where the reference solver is not
installed, so this module restates the pieces of its setup a solve needs, with
the same defaults and the same arithmetic:

* the contour families bell / smooth / conical / moc / bezier: a cubic-Hermite
  converging section with zero end slopes and a diverging section per family
  (src/geometry/contour.py:112-311), plus ``bezier8``, a smooth wall with eight
  Gaussian-free radial control offsets (no counterpart in the reference);
* the throat-clustered axial node distribution, refined by subdivision
  (src/geometry/mesh.py:213-272,442-464) and ``y = r * y_wall(x)``
  (src/geometry/mesh.py:467-490);
* isentropic quasi-1D theory: the area-Mach relation inverted by bisection,
  the critical back-pressure ratios, the shock-free test and the quasi-1D
  solution in each regime (src/physics/quasi1d.py:61-401);
* the L2 projection of that solution, with a transverse velocity from the wall
  slope, as the initial state (src/timestepping/initialize.py:41-102).
"""

from __future__ import annotations

import math
from dataclasses import asdict, dataclass, field, replace

import numpy as np

from . import mesh as msh
from .config import FlowConditions, SolverOptions
from .operators import build_operators

ANALYTIC_THROAT_X = 0.13880048
ANALYTIC_THROAT_Y = 0.13989434
ANALYTIC_INLET_Y = 0.15
ANALYTIC_AREA_RATIO = 0.35 / ANALYTIC_THROAT_Y
CONTOURS = ("bell", "smooth", "conical", "moc", "bezier", "bezier8")


@dataclass(frozen=True)
class Geometry:
    area_ratio: float = ANALYTIC_AREA_RATIO
    throat_x: float = ANALYTIC_THROAT_X
    throat_half_height: float = ANALYTIC_THROAT_Y
    inlet_half_height: float = ANALYTIC_INLET_Y
    length: float = 1.0
    contour: str = "bell"
    theta_initial_deg: float | None = None
    theta_exit_deg: float = 0.0
    bezier_w1: float = 0.55
    bezier_w2: float = 0.90
    # bezier8: radial offsets of eight interior control points, as fractions of
    # the throat half-height, added to a smooth diverging wall
    offsets: tuple = field(default_factory=lambda: (0.0,) * 8)

    def __post_init__(self):
        if self.contour not in CONTOURS:
            raise ValueError(f"unknown contour {self.contour!r}; choose from {CONTOURS}")
        if self.area_ratio <= 1.0 or not 0.0 < self.throat_x < 1.0:
            raise ValueError("area_ratio must exceed 1 and throat_x lie in (0, 1)")

    def theta_initial(self) -> float:
        if self.contour in ("smooth", "bezier8"):
            return 0.0
        if self.theta_initial_deg is not None:
            return math.radians(float(self.theta_initial_deg))
        if self.contour == "moc":
            return math.radians(30.0)
        y_th = self.throat_half_height
        span = max(self.length * (1.0 - self.throat_x), 1e-12)
        return math.atan(1.6 * (y_th * self.area_ratio - y_th) / span)

    def wall(self, x):
        return wall_half_height(np.asarray(x, dtype=float), self)

    def throat_location(self) -> float:
        return float(self.throat_x) * self.length

    def throat_height(self) -> float:
        return float(self.throat_half_height)

    def replace(self, **kw) -> Geometry:
        return replace(self, **kw)

    def as_dict(self) -> dict:
        return asdict(self)


def _hermite(s, y0, y1, m0, m1):
    s2 = s * s
    s3 = s2 * s
    return (2.0 * s3 - 3.0 * s2 + 1.0) * y0 + (s3 - 2.0 * s2 + s) * m0 + (-2.0 * s3 + 3.0 * s2) * y1 + (s3 - s2) * m1


BEZIER8_DEGREE = 9  # ten control points: the throat, eight free, the exit


def _bernstein(n, k, t):
    return math.comb(n, k) * t**k * (1.0 - t) ** (n - k)


def wall_half_height(x, geom: Geometry):
    xi = x / geom.length
    y_th, y_in = geom.throat_half_height, geom.inlet_half_height
    y_ex = y_th * geom.area_ratio
    x_th = geom.throat_x
    y_conv = _hermite(np.clip(xi / x_th, 0.0, 1.0), y_in, y_th, 0.0, 0.0)
    span = 1.0 - x_th
    s = np.clip((xi - x_th) / span, 0.0, 1.0)
    dx_ds = span * geom.length
    c = geom.contour
    if c == "conical":
        y_div = y_th + (y_ex - y_th) * s
    elif c in ("bell", "smooth", "moc"):
        y_div = _hermite(s, y_th, y_ex, math.tan(geom.theta_initial()) * dx_ds,
                         math.tan(math.radians(geom.theta_exit_deg)) * dx_ds)
    elif c == "bezier":
        c1 = y_th + geom.bezier_w1 * (y_ex - y_th)
        c2 = y_th + geom.bezier_w2 * (y_ex - y_th)
        u = 1.0 - s
        y_div = u**3 * y_th + 3.0 * u**2 * s * c1 + 3.0 * u * s**2 * c2 + s**3 * y_ex
    else:  # bezier8: smooth Hermite wall plus a degree-9 Bezier bump that vanishes at both ends
        base = _hermite(s, y_th, y_ex, 0.0, math.tan(math.radians(geom.theta_exit_deg)) * dx_ds)
        bump = sum(_bernstein(BEZIER8_DEGREE, k + 1, s) * geom.offsets[k] for k in range(8))
        y_div = base + y_th * bump
    return np.where(xi <= x_th, y_conv, y_div)


def bezier8_sensitivity(x, geom: Geometry) -> np.ndarray:
    """``d y_wall / d offset_k`` at ``x``, shape ``(8, len(x))`` (zero upstream of the throat)."""
    xi = np.asarray(x, float) / geom.length
    s = np.clip((xi - geom.throat_x) / (1.0 - geom.throat_x), 0.0, 1.0)
    out = np.stack([geom.throat_half_height * _bernstein(BEZIER8_DEGREE, k + 1, s) for k in range(8)])
    return np.where(xi[None, :] <= geom.throat_x, 0.0, out)


# ------------------------------------------------------- design variables
#: Differentiable design variables of a contour (src/geometry/contour.py:55-65),
#: plus the eight radial offsets of the bezier8 family.
DESIGN_PARAMETERS = ("area_ratio", "throat_x", "throat_half_height", "inlet_half_height", "theta_initial",
                     "theta_exit", "bezier_w1", "bezier_w2", "length")
BEZIER8_PARAMETERS = tuple(f"offset_{k}" for k in range(8))


def design_params(geom: Geometry) -> dict:
    """The design variables as a flat dict, wall angles in radians (src/geometry/contour.py:170-188)."""
    out = {
        "area_ratio": float(geom.area_ratio),
        "throat_x": float(geom.throat_x),
        "throat_half_height": float(geom.throat_half_height),
        "inlet_half_height": float(geom.inlet_half_height),
        "theta_initial": float(geom.theta_initial()),
        "theta_exit": math.radians(float(geom.theta_exit_deg)),
        "bezier_w1": float(geom.bezier_w1),
        "bezier_w2": float(geom.bezier_w2),
        "length": float(geom.length),
    }
    if geom.contour == "bezier8":
        out.update({f"offset_{k}": float(geom.offsets[k]) for k in range(8)})
    return out


def geometry_with(geom: Geometry, params: dict) -> Geometry:
    """The geometry at these design variables (src/geometry/contour.py:190-204)."""
    fields = {}
    for key, value in params.items():
        if key == "theta_initial":
            fields["theta_initial_deg"] = math.degrees(float(value))
        elif key == "theta_exit":
            fields["theta_exit_deg"] = math.degrees(float(value))
        elif key in BEZIER8_PARAMETERS:
            continue
        elif key in DESIGN_PARAMETERS:
            fields[key] = float(value)
        else:
            raise ValueError(f"{key!r} is not a design parameter; use {DESIGN_PARAMETERS + BEZIER8_PARAMETERS}")
    if any(k in params for k in BEZIER8_PARAMETERS):
        offs = list(geom.offsets)
        for k in range(8):
            if f"offset_{k}" in params:
                offs[k] = float(params[f"offset_{k}"])
        fields["offsets"] = tuple(offs)
    return replace(geom, **fields)


def _as_array(a, xp):
    # arrays are used as they are: torch.asarray would hand a tensor back with
    # requires_grad switched off, cutting the gradient through it
    return a if hasattr(a, "shape") else xp.asarray(a)


def wall_from_params(x, params: dict, contour: str, xp=np):
    """Wall half-height from a design-variable dict, every operation through ``xp``.

    Restates src/geometry/contour.py:264-311 (plus the bezier8 family) so that
    ``xp = torch`` with tensor parameters gives a differentiable contour; the
    wall angles are independent variables here, as in the reference's
    parameterisation.
    """
    if contour not in CONTOURS:
        raise ValueError(f"unknown contour {contour!r}; choose from {CONTOURS}")
    length = params.get("length", 1.0)
    xi = _as_array(x, xp) / length
    y_th = params["throat_half_height"]
    y_in = params["inlet_half_height"]
    y_ex = y_th * params["area_ratio"]
    x_th = params["throat_x"]
    y_conv = _hermite(xp.clip(xi / x_th, 0.0, 1.0), y_in, y_th, 0.0, 0.0)
    span = 1.0 - x_th
    s = xp.clip((xi - x_th) / span, 0.0, 1.0)
    dx_ds = span * length
    if contour == "conical":
        y_div = y_th + (y_ex - y_th) * s
    elif contour in ("bell", "smooth", "moc"):
        y_div = _hermite(s, y_th, y_ex, xp.tan(params["theta_initial"]) * dx_ds,
                         xp.tan(params["theta_exit"]) * dx_ds)
    elif contour == "bezier":
        c1 = y_th + params["bezier_w1"] * (y_ex - y_th)
        c2 = y_th + params["bezier_w2"] * (y_ex - y_th)
        u = 1.0 - s
        y_div = u**3 * y_th + 3.0 * u**2 * s * c1 + 3.0 * u * s**2 * c2 + s**3 * y_ex
    else:
        base = _hermite(s, y_th, y_ex, 0.0, xp.tan(params["theta_exit"]) * dx_ds)
        bump = sum(_bernstein(BEZIER8_DEGREE, k + 1, s) * params[f"offset_{k}"] for k in range(8))
        y_div = base + y_th * bump
    return xp.where(xi <= x_th, y_conv, y_div)


def node_coords_from_params(x_frac, r_frac, params: dict, contour: str, xp=np):
    """Node coordinates ``(x, r y_wall(x))`` of the frozen logical grid (src/geometry/mesh.py:467-490)."""
    length = params.get("length", 1.0)
    x = _as_array(x_frac, xp) * length
    yw = wall_from_params(x, params, contour, xp)
    nr, nx = len(r_frac), len(x_frac)
    xx = xp.broadcast_to(x[None, :], (nr, nx))
    yy = _as_array(r_frac, xp)[:, None] * yw[None, :]
    return xp.stack([xx.reshape(-1), yy.reshape(-1)], -1)


# ---------------------------------------------------------------- node grids
def clustered_distribution(n_intervals, x_throat, strength, width):
    if strength < 1.0:
        raise ValueError("cluster strength must be >= 1")
    fine = np.linspace(0.0, 1.0, 20001)
    h = 1.0 + (strength - 1.0) * (1.0 - np.exp(-(((fine - x_throat) / width) ** 2)))
    dens = 1.0 / h
    cdf = np.concatenate([[0.0], np.cumsum(0.5 * (dens[1:] + dens[:-1]) * np.diff(fine))])
    cdf /= cdf[-1]
    x = np.interp(np.linspace(0.0, 1.0, n_intervals + 1), cdf, fine)
    x[0], x[-1] = 0.0, 1.0
    return x


def subdivide(base, n_sub):
    if n_sub == 1:
        return base.copy()
    frac = np.arange(n_sub) / n_sub
    out = np.concatenate([base[i] * (1.0 - frac) + base[i + 1] * frac for i in range(base.size - 1)] + [base[-1:]])
    return out


def x_distribution(n_nodes, nx_base, n_sub, spacing, x_throat, strength, width):
    if spacing == "uniform":
        base = np.linspace(0.0, 1.0, nx_base + 1)
    elif spacing == "throat":
        base = clustered_distribution(nx_base, x_throat, strength, width)
    elif spacing == "inlet":
        a, b = 0.7, 1.2
        v = np.logspace(a, b, nx_base + 1)
        base = (v - 10.0**a) / (10.0**b - 10.0**a)
    else:
        raise ValueError(f"unknown x_spacing {spacing!r}")
    x = subdivide(base, n_sub)
    assert x.size == n_nodes
    return x


# ---------------------------------------------------------------- quasi-1D
def area_over_throat(M, g):
    M = np.maximum(np.asarray(M, float), 1e-12)
    return (1.0 / M) * (2.0 / (g + 1.0) * (1.0 + 0.5 * (g - 1.0) * M * M)) ** ((g + 1.0) / (2.0 * (g - 1.0)))


def pressure_ratio(M, g):
    M = np.asarray(M, float)
    return (1.0 + 0.5 * (g - 1.0) * M * M) ** (-g / (g - 1.0))


def temperature_ratio(M, g):
    M = np.asarray(M, float)
    return 1.0 / (1.0 + 0.5 * (g - 1.0) * M * M)


def mach_from_pressure_ratio(r, g):
    r = np.clip(np.asarray(r, float), 1e-300, 1.0)
    return np.sqrt(2.0 / (g - 1.0) * (r ** (-(g - 1.0) / g) - 1.0))


def mach_from_area(ar, g, supersonic=False, tol=1e-13):
    ar_in = ar
    ar = np.atleast_1d(np.asarray(ar, float))
    if np.any(ar < 1.0 - 1e-9):
        raise ValueError("A/A* must be >= 1")
    ar = np.maximum(ar, 1.0)
    if supersonic:
        lo, hi = np.ones_like(ar), np.full_like(ar, 1.2)
        for _ in range(200):
            need = area_over_throat(hi, g) < ar
            if not np.any(need):
                break
            hi = np.where(need, hi * 1.5, hi)
    else:
        lo, hi = np.full_like(ar, 1e-10), np.ones_like(ar)
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        small = area_over_throat(mid, g) < ar
        if supersonic:
            lo, hi = np.where(small, mid, lo), np.where(small, hi, mid)
        else:
            hi, lo = np.where(small, mid, hi), np.where(small, lo, mid)
        if np.all(hi - lo < tol):
            break
    out = 0.5 * (lo + hi)
    return out if np.ndim(ar_in) else float(out[0])


def shock_static_ratio(M1, g):
    return (2.0 * g * M1 * M1 - (g - 1.0)) / (g + 1.0)


def shock_total_ratio(M1, g):
    t1 = ((g + 1.0) * 0.5 * M1 * M1 / (1.0 + 0.5 * (g - 1.0) * M1 * M1)) ** (g / (g - 1.0))
    t2 = (2.0 * g / (g + 1.0) * M1 * M1 - (g - 1.0) / (g + 1.0)) ** (1.0 / (g - 1.0))
    return t1 / t2


def critical_ratios(area_ratio, g=1.4):
    """``(first, second, third)``: choking, shock at the exit, design."""
    m_sub = float(mach_from_area(area_ratio, g, supersonic=False))
    m_sup = float(mach_from_area(area_ratio, g, supersonic=True))
    third = float(pressure_ratio(m_sup, g))
    return float(pressure_ratio(m_sub, g)), third * float(shock_static_ratio(m_sup, g)), third


def is_shock_free(area_ratio, pb, g=1.4) -> bool:
    first, second, _ = critical_ratios(area_ratio, g)
    return pb < second or pb >= first


def realised_area_ratio(geom: Geometry) -> float:
    return float(geom.wall(np.asarray([geom.length]))[0]) / geom.throat_height()


@dataclass
class Quasi1D:
    x: np.ndarray
    density: np.ndarray
    velocity: np.ndarray
    pressure: np.ndarray
    regime: str


def solve_quasi1d(geom: Geometry, flow, n_points=601) -> Quasi1D:
    g = flow.gamma
    x = np.linspace(0.0, geom.length, n_points)
    area = 2.0 * np.asarray(geom.wall(x), float)
    x_th = geom.throat_location()
    a_th = 2.0 * geom.throat_height()
    a_ex = 2.0 * float(geom.wall(np.asarray([geom.length]))[0])
    first, second, third = critical_ratios(a_ex / a_th, g)
    pb = flow.back_pressure_ratio
    pt = flow.total_pressure
    pt_local = np.full_like(x, pt)
    if pb >= first:
        regime = "subsonic"
        m_exit = float(mach_from_pressure_ratio(pb, g))
        a_star = a_ex / float(area_over_throat(m_exit, g))
        mach = mach_from_area(np.maximum(area / a_star, 1.0), g, supersonic=False)
    else:
        regime = "shock-in-nozzle" if pb > second else "choked"
        a_star = a_th
        ratio = np.maximum(area / a_star, 1.0)
        mach = np.where(x > x_th, mach_from_area(ratio, g, supersonic=True), mach_from_area(ratio, g, supersonic=False))
        if regime == "shock-in-nozzle":

            def p_exit(xs):
                a1 = 2.0 * float(geom.wall(np.asarray([xs]))[0])
                m1 = float(mach_from_area(a1 / a_star, g, supersonic=True))
                r = float(shock_total_ratio(m1, g))
                m_e = float(mach_from_area(a_ex / (a_star / r), g, supersonic=False))
                return float(pressure_ratio(m_e, g)) * r

            lo, hi = x_th + 1e-9 * geom.length, geom.length
            for _ in range(200):
                mid = 0.5 * (lo + hi)
                if p_exit(mid) > pb:
                    lo = mid
                else:
                    hi = mid
                if hi - lo < 1e-12 * geom.length:
                    break
            xs = 0.5 * (lo + hi)
            a1 = 2.0 * float(geom.wall(np.asarray([xs]))[0])
            m1 = float(mach_from_area(a1 / a_star, g, supersonic=True))
            r = float(shock_total_ratio(m1, g))
            behind = x > xs
            mach = np.where(behind, mach_from_area(np.maximum(area / (a_star / r), 1.0), g, supersonic=False), mach)
            pt_local = np.where(behind, pt * r, pt)
    p = pt_local * pressure_ratio(mach, g)
    T = flow.total_temperature * temperature_ratio(mach, g)
    rho = p / (flow.Rgas * T)
    vx = mach * np.sqrt(g * flow.Rgas * T)
    return Quasi1D(x, rho, vx, p, regime)


# ------------------------------------------------------------------ cases
def project(values, ops):
    """L2 projection of point values at the volume quadrature points."""
    rhs = np.einsum("iq,eq,eqs->eis", ops.ref.phi_vol, ops.weighted_det, values)
    return np.einsum("eij,ejs->eis", ops.inv_mass, rhs)


def quasi1d_initial(ops, flow, geom: Geometry):
    sol = solve_quasi1d(geom, flow)
    xy = np.asarray(ops.xy_vol)
    x, y = xy[..., 0], xy[..., 1]
    rho = np.interp(x, sol.x, sol.density)
    vx = np.interp(x, sol.x, sol.velocity)
    p = np.interp(x, sol.x, sol.pressure)
    yw = np.asarray(geom.wall(x))
    h = 1e-6 * geom.length
    slope = (np.asarray(geom.wall(x + h)) - np.asarray(geom.wall(np.maximum(x - h, 0.0)))) / (h + np.minimum(x, h))
    vy = vx * np.clip(y / np.maximum(yw, 1e-30), 0.0, 1.0) * slope
    rhoE = p / (flow.gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)
    return project(np.stack([rho, rho * vx, rho * vy, rhoE], axis=-1), ops)


@dataclass
class Case:
    geometry: Geometry
    flow: object
    options: object
    topology: object
    node_coords: np.ndarray
    operators: object
    grids: dict

    def initial_state(self):
        return quasi1d_initial(self.operators, self.flow, self.geometry)


class ShockInNozzle(ValueError):
    """The operating point stands a normal shock in the diverging section."""


WALL_FAMILIES = {"conical": 0, "bell": 1, "smooth": 1, "moc": 1, "bezier": 2, "bezier8": 3}


def wall_parameters(geom: Geometry) -> np.ndarray:
    """The numbers the device evaluates ``wall_half_height`` from (the header's NZB_WALL_PARAMS layout):
    family, length, throat x, 1 - throat x, throat / inlet / exit half-heights, the Hermite end slopes,
    the Bezier control heights, the difference step h = 1e-6 L and the eight bezier8 offsets -- each
    formed as ``wall_half_height`` forms it."""
    y_th, y_in = geom.throat_half_height, geom.inlet_half_height
    y_ex = y_th * geom.area_ratio
    x_th = geom.throat_x
    span = 1.0 - x_th
    dx_ds = span * geom.length
    m0 = m1 = 0.0
    if geom.contour in ("bell", "smooth", "moc"):
        m0 = math.tan(geom.theta_initial()) * dx_ds
        m1 = math.tan(math.radians(geom.theta_exit_deg)) * dx_ds
    elif geom.contour == "bezier8":
        m1 = math.tan(math.radians(geom.theta_exit_deg)) * dx_ds
    c1 = y_th + geom.bezier_w1 * (y_ex - y_th)
    c2 = y_th + geom.bezier_w2 * (y_ex - y_th)
    out = [float(WALL_FAMILIES[geom.contour]), geom.length, x_th, span, y_th, y_in, y_ex, m0, m1, c1, c2,
           1e-6 * geom.length] + [float(v) for v in geom.offsets]
    return np.asarray(out, float)


def quasi1d_table(geom: Geometry, flow) -> np.ndarray:
    """(4, n): the quasi-1D solution's x, density, axial velocity and pressure, as the initial state reads it."""
    sol = solve_quasi1d(geom, flow)
    return np.ascontiguousarray(np.stack([sol.x, sol.density, sol.velocity, sol.pressure]).astype(float))


def build_case(*, element="tri", order=1, refine=0, nx=14, nr=5, x_spacing="throat", cluster_strength=3.0,
               cluster_width=0.12, flow=None, options=None, check_shock=True, lean=False, geometry_order=1,
               **geom_kw) -> Case:
    """A nozzle case with the reference's defaults (src/api.py:159-210).  ``geometry_order`` 2 gives
    curved (quadratic) elements whose interior and mid-edge nodes follow the wall, as the reference's
    build_nozzle_mesh places them (src/geometry/mesh.py:493-521).

    Raises :class:`ShockInNozzle` for an operating point in the shocked band
    unless ``flow.allow_shock_in_nozzle`` -- the reference's refusal
    (src/api.py:320-334).
    """
    geom = Geometry(**geom_kw)
    flow = flow or FlowConditions()
    options = options or SolverOptions()
    if check_shock and not (is_shock_free(realised_area_ratio(geom), flow.back_pressure_ratio, flow.gamma)
                            or getattr(flow, "allow_shock_in_nozzle", False)):
        raise ShockInNozzle(f"back_pressure_ratio={flow.back_pressure_ratio:.4f} stands a normal shock in the nozzle")
    if geometry_order < 1:
        raise ValueError(f"geometry_order (Q) must be >= 1, got {geometry_order}")
    topo, _, r_frac = msh.channel_topology(element, nx=nx, nr=nr, refine=refine, geometry_order=geometry_order)
    x_frac = x_distribution(topo.logical["nx_nodes"], nx, geometry_order * 2**refine, x_spacing,
                            geom.throat_location() / geom.length, cluster_strength, cluster_width)
    coords = msh.channel_coords(x_frac, r_frac, geom.wall, geom.length)
    # lean: no per-element operator arrays on the host -- the device builds the metric terms and the
    # initial state from the node coordinates (DeviceMesh.set_geometry, nzb_initial_state)
    ops = build_operators(topo, coords, order, lean=lean)
    return Case(geom, flow, options, topo, coords, ops, {"x_frac": x_frac, "r_frac": r_frac})
