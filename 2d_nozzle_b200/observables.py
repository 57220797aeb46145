"""Integral observables of a converged state: thrust, mass flow, exit averages, entropy error.

Restates the parity observables of src/post/postprocess.py:56-75,155-192,193-263:
the solution traced onto one tagged boundary with the owner-side basis, the
axial momentum flux ``int (rho vx vn + p nx) ds``, the wall-pressure thrust,
the mass flux ``int rho vn ds``, the area-averaged exit Mach number, pressure
and temperature, and the RMS entropy deviation, all for the full planar nozzle
(twice the meshed half channel).

Both paths reduce a state to the same eleven per-instance sums (the columns
``capi.OBS_*``) and :func:`from_sums` forms the metrics from them:
:func:`sums` on the host from a host state, :class:`DeviceObservables` with one
launch of the device kernel over every instance of a mesh or batch bucket, so
a sweep's observables need no state copied back.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import capi
from .config import FLOOR
from .mesh import INFLOW, OUTFLOW, WALL


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


def entropy_reference(flow) -> float:
    """``s_t = p_t^(1 - gamma) (R T_t)^gamma`` (src/post/postprocess.py:184)."""
    g = flow.gamma
    return flow.total_pressure ** (1.0 - g) * (flow.Rgas * flow.total_temperature) ** g


def sums(U, ops, flow) -> np.ndarray:
    """The eleven integrals of ``capi.OBS_*`` from a host state ``(E, NP, 4)``."""
    g = flow.gamma
    out = np.zeros(capi.NOBS)
    for tag in (OUTFLOW, INFLOW):
        state, n, ds = boundary_trace(U, ops, tag)
        rho, vx, vy, p = _primitives(state, g)
        vn = vx * n[..., 0] + vy * n[..., 1]
        mom = float(((rho * vx * vn + p * n[..., 0]) * ds).sum())
        mass = float((rho * vn * ds).sum())
        if tag == OUTFLOW:
            out[capi.OBS_MOM_OUT], out[capi.OBS_MASS_OUT] = mom, mass
            out[capi.OBS_EXIT_LEN] = float(ds.sum())
            out[capi.OBS_EXIT_MACH] = float((np.sqrt((vx * vx + vy * vy) * rho / (g * p)) * ds).sum())
            out[capi.OBS_EXIT_P] = float((p * ds).sum())
            out[capi.OBS_EXIT_T] = float((p / (flow.Rgas * rho) * ds).sum())
        else:
            out[capi.OBS_MOM_IN], out[capi.OBS_MASS_IN] = mom, mass
    state, n, ds = boundary_trace(U, ops, WALL)
    out[capi.OBS_WALL_PX] = float((_primitives(state, g)[3] * n[..., 0] * ds).sum())
    uq = np.einsum("iq,eis->eqs", np.asarray(ops.ref.phi_vol), np.asarray(U))
    rho, _, _, p = _primitives(uq, g)
    ratio = (p / rho**g) / entropy_reference(flow)
    out[capi.OBS_ENTROPY] = float(((ratio - 1.0) ** 2 * np.asarray(ops.weighted_det)).sum())
    out[capi.OBS_AREA] = float(np.asarray(ops.elem_area).sum())
    return out


def ideal_thrust(geom, flow) -> float:
    """Quasi-1D axial force of the same geometry, momentum form, full nozzle
    (src/post/postprocess.py:258-263); ``A(x) = 2 y_wall(x)``."""
    from .nozzle import solve_quasi1d

    q = solve_quasi1d(geom, flow)
    area = 2.0 * np.asarray(geom.wall(np.asarray([q.x[0], q.x[-1]])), float)
    rho, vx, p = q.density, q.velocity, q.pressure
    return float((rho[-1] * vx[-1] ** 2 + p[-1]) * area[-1] - (rho[0] * vx[0] ** 2 + p[0]) * area[0])


def from_sums(s, flow, geom=None) -> dict:
    """The metrics of the reference's ``performance()`` from one instance's sums.

    ``geom`` (the nozzle geometry) adds the throat-normalised coefficients, the
    quasi-1D ideal thrust and the efficiency (src/post/postprocess.py:193-255).
    """
    s = np.asarray(s, float)
    half_to_full = 2.0
    thrust = half_to_full * (s[capi.OBS_MOM_OUT] + s[capi.OBS_MOM_IN])
    thrust_wall = half_to_full * -s[capi.OBS_WALL_PX]
    denom = abs(thrust) if abs(thrust) > 0.0 else 1.0
    mdot_in = half_to_full * -s[capi.OBS_MASS_IN]
    mdot_out = half_to_full * s[capi.OBS_MASS_OUT]
    area_e = s[capi.OBS_EXIT_LEN]
    a_t = flow.stagnation_sound_speed
    out = {
        "thrust": float(thrust),
        "thrust_wall": float(thrust_wall),
        "thrust_imbalance": float(abs(thrust - thrust_wall) / denom),
        "mass_flow_in": float(mdot_in),
        "mass_flow_out": float(mdot_out),
        "mass_imbalance": float(abs(mdot_out - mdot_in) / (abs(mdot_in) if mdot_in else 1.0)),
        "entropy_error": float(math.sqrt(s[capi.OBS_ENTROPY] / s[capi.OBS_AREA])),
        "exit_mach": float(s[capi.OBS_EXIT_MACH] / area_e),
        "exit_pressure_ratio": float(s[capi.OBS_EXIT_P] / area_e / flow.total_pressure),
        "exit_temperature_ratio": float(s[capi.OBS_EXIT_T] / area_e / flow.total_temperature),
        "specific_thrust": float(thrust / mdot_in) if mdot_in else float("nan"),
        "specific_thrust_ratio": float(thrust / mdot_in / a_t) if mdot_in else float("nan"),
    }
    out["exit_mach_area_averaged"] = out["exit_mach"]
    if geom is not None:
        a_throat = 2.0 * geom.throat_height()
        ideal = ideal_thrust(geom, flow)
        out["thrust_coefficient"] = float(thrust / (flow.total_pressure * a_throat))
        out["discharge_coefficient"] = float(mdot_in / (flow.stagnation_density * a_t * a_throat))
        out["ideal_thrust"] = ideal
        out["thrust_efficiency"] = float(thrust / ideal) if ideal else float("nan")
    return out


def performance(U, ops, flow, geom=None) -> dict:
    """Thrust (momentum and wall forms), mass flows, exit averages and entropy error of a host state."""
    return from_sums(sums(U, ops, flow), flow, geom)


def segments(parts) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
    """``(bedges, bseg, eseg)`` of ``nzb_obs_args`` for meshes laid out one after another.

    ``parts``: per instance ``(ops, element offset, edge offset)`` in the
    concatenated numbering; an instance's inflow, outflow and wall edges are
    its boundary edges of those tags (edges number interior first, then the
    boundary by tag).
    """
    bedges, bseg, eseg = [], [0], []
    for ops, e_off, k_off in parts:
        topo = ops.topology
        for tag in (INFLOW, OUTFLOW, WALL):
            sl = topo.tag_slice(tag)
            bedges.append(k_off + ops.n_interior + np.arange(sl.start, sl.stop))
        bseg.append(bseg[-1] + sum(len(b) for b in bedges[-3:]))
        eseg.append(e_off)
    eseg.append(parts[-1][1] + int(parts[-1][0].n_elem))
    cat = np.concatenate(bedges) if bedges else np.zeros(0, int)
    return cat.astype(np.int32), np.asarray(bseg, np.int32), np.asarray(eseg, np.int32)


class DeviceObservables:
    """Per-instance observable sums of a device mesh (or bucket) in one launch.

    ``parts`` as for :func:`segments`; a single mesh is ``[(ops, 0, 0)]``.
    """

    def __init__(self, dmesh, phys, parts, flows):
        import torch

        self.torch = torch
        self.dmesh, self.phys = dmesh, phys
        self.flows = list(flows)
        if len(self.flows) != len(parts):
            raise ValueError("one flow per instance")
        if len({(f.gamma, f.Rgas, entropy_reference(f)) for f in self.flows}) != 1:
            raise ValueError("a launch takes one gas (gamma, R, s_t) for all its instances")
        b, bs, es = segments(parts)
        dev = dmesh.device
        self._b = torch.as_tensor(b if len(b) else np.zeros(1, np.int32), device=dev)
        self._bs = torch.as_tensor(bs, device=dev)
        self._es = torch.as_tensor(es, device=dev)
        self.n = len(parts)
        self.out = torch.empty((self.n, capi.NOBS), dtype=torch.float64, device=dev)
        a = capi.ObsArgs()
        a.n_seg = self.n
        a.bedges, a.bseg, a.eseg = self._b.data_ptr(), self._bs.data_ptr(), self._es.data_ptr()
        a.r_gas = float(self.flows[0].Rgas)
        a.s_t = float(entropy_reference(self.flows[0]))
        a.out = self.out.data_ptr()
        self.args = a

    def launch(self, U_soa, stream=None) -> None:
        """Queue the sums of the device state ``(4, NP, E)`` (no synchronisation)."""
        torch = self.torch
        st = stream if stream is not None else torch.cuda.current_stream(self.dmesh.device)
        self.args.U = U_soa.data_ptr()
        lib = capi.load()
        capi.check(lib.nzb_observables(self.dmesh.c_ref, C.byref(self.phys), C.byref(self.args),
                                       st.cuda_stream), "nzb_observables")

    def sums(self, U_soa, stream=None) -> np.ndarray:
        """``(n_instances, NOBS)`` sums on the host."""
        self.launch(U_soa, stream)
        return self.out.cpu().numpy()

    def performance(self, U_soa, geoms=None, stream=None) -> list[dict]:
        s = self.sums(U_soa, stream)
        geoms = geoms if geoms is not None else [None] * self.n
        return [from_sums(s[i], self.flows[i], geoms[i]) for i in range(self.n)]
