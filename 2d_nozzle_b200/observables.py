"""Integral observables of a converged state: thrust, mass flow, exit Mach number.

Restates the parity observables of src/post/postprocess.py:56-75,155-171,193-255:
the solution traced onto one tagged boundary with the owner-side basis, the
axial momentum flux ``int (rho vx vn + p nx) ds``, the mass flux
``int rho vn ds`` and the area-averaged exit Mach number, all for the full
planar nozzle (twice the meshed half channel).
"""

from __future__ import annotations

import numpy as np

from .config import FLOOR
from .mesh import INFLOW, OUTFLOW


def _primitives(U, g):
    rho = np.maximum(U[..., 0], FLOOR)
    vx, vy = U[..., 1] / rho, U[..., 2] / rho
    p = np.maximum((g - 1.0) * (U[..., 3] - 0.5 * rho * (vx * vx + vy * vy)), FLOOR)
    return rho, vx, vy, p


def boundary_trace(U, ops, tag: int):
    """``(state (n, nqf, 4), normal (n, nqf, 2), ds (n, nqf))`` on one tagged boundary."""
    ed = ops.topology.edges
    sl = ops.topology.tag_slice(tag)
    phi = np.asarray(ops.ref.phi_face)[0][ed.bedge_face[sl]]
    state = np.einsum("kiq,kis->kqs", phi, np.asarray(U)[ed.bedge_elem[sl]])
    g = ops.n_interior + np.arange(sl.start, sl.stop)
    ds = np.asarray(ops.edge_jac)[g] * np.asarray(ops.ref.w_face)[None, :]
    return state, np.asarray(ops.edge_normal)[g], ds


def _momentum(tr, g):
    state, n, ds = tr
    rho, vx, vy, p = _primitives(state, g)
    vn = vx * n[..., 0] + vy * n[..., 1]
    return float(((rho * vx * vn + p * n[..., 0]) * ds).sum())


def _mass(tr, g):
    state, n, ds = tr
    rho, vx, vy, _ = _primitives(state, g)
    return float((rho * (vx * n[..., 0] + vy * n[..., 1]) * ds).sum())


def performance(U, ops, flow) -> dict:
    """Thrust (momentum form), inlet mass flow and area-averaged exit Mach number."""
    g = flow.gamma
    inlet, outlet = boundary_trace(U, ops, INFLOW), boundary_trace(U, ops, OUTFLOW)
    thrust = 2.0 * (_momentum(outlet, g) + _momentum(inlet, g))
    mdot_in = 2.0 * -_mass(inlet, g)
    mdot_out = 2.0 * _mass(outlet, g)
    rho, vx, vy, p = _primitives(outlet[0], g)
    mach = np.sqrt((vx * vx + vy * vy) * rho / (g * p))
    ds = outlet[2]
    return {
        "thrust": thrust,
        "mass_flow_in": mdot_in,
        "mass_flow_out": mdot_out,
        "exit_mach": float((mach * ds).sum() / ds.sum()),
    }
