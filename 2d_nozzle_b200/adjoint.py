"""Exact design sensitivities by the discrete adjoint, on the device.

Restates src/sensitivity.py for the B200 kernels.  For a scalar objective J
(thrust, thrust coefficient, exit Mach number, mass flow, exit pressure) and
design variables a, the converged state satisfies R(U, a) = 0 and

    dJ/da = dJ/da|_U - lam^T dR/da,     (dR/dU)^T lam = (dJ/dU)^T,

with R the unfolded residual (M dU/dt = -R).  lam comes from the reference's
pseudo-time march dlam/dtau = -M^-1 ((dR/dU)^T lam - dJ/dU): classical RK4,
the local step frozen from the converged state with the SSP-RK3 coefficient at
the forward solve's cfl, the defect's RMS checked every ``check_interval``
steps against ``tolerance`` times the seed's (src/sensitivity.py:289-383).

Every product with a transposed Jacobian is a hand-written CUDA kernel
(``nzb_vjp`` for the state, ``nzb_vjp_coords`` for node coordinates and back
pressure), and the march is a CUDA graph of fused RK4-stage kernels
(``nzb_adjoint_*``).  :class:`ResidualFunction` exposes R(U, X, p_back) to
PyTorch as a ``torch.autograd.Function`` whose backward calls those kernels.
The objectives (boundary integrals) and the map from design variables to node
coordinates are small computations written in torch, so their derivatives
come from torch's autograd, as the reference takes them from JAX.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
from dataclasses import dataclass

import numpy as np
import torch

from . import capi
from . import nozzle as nz
from .backend import B200Backend
from .config import SolverOptions, step_coefficient
from .autotune import choose_variant, context_for, set_struct_variant, tail_elements
from .layout import DeviceMesh, face_tangent_table, physics_struct
from .march import solve as march_solve
from .mesh import INFLOW, OUTFLOW
from .operators import build_operators

OBJECTIVES = ("thrust", "thrust_coefficient", "exit_mach", "mass_flow", "exit_pressure")
FLOW_DESIGN_PARAMETERS = ("back_pressure",)
STATUS = {0: "running", 1: "converged", 2: "non-finite", 5: "max_iterations"}


def to_soa(U):
    """(E, NP, 4) tensor -> flat (4, NP, E) tensor, the device layout."""
    return U.permute(2, 1, 0).contiguous().reshape(-1)


def from_soa(a, E, NP):
    """Flat (4, NP, E) tensor -> (E, NP, 4)."""
    return a.reshape(4, NP, E).permute(2, 1, 0).contiguous()


class AdjointModel:
    """One mesh on the device, with what the transposed products need."""

    def __init__(self, ops, flow, opts, device=None, variants: str = "auto"):
        self.ops, self.flow, self.opts = ops, flow, opts
        self.lib = capi.load()
        self.mesh = DeviceMesh(ops, device)
        self.variants = context_for(self.mesh.E, variants)
        choose_variant(self.mesh, self.variants)
        self.device = self.mesh.device
        self.E, self.NP, self.NV = self.mesh.E, self.mesh.np_, self.mesh.nf
        self.phys = physics_struct(flow, opts, ops.ref)
        self.dgs = np.ascontiguousarray(face_tangent_table(ops.ref).ravel())  # host: passed by value to the kernel
        self.elem_nodes = np.ascontiguousarray(np.asarray(ops.topology.elem_nodes)[:, : self.NV])
        self.elem_nodes_t = torch.as_tensor(self.elem_nodes, device=self.device)
        self.X0 = torch.as_tensor(np.asarray(ops.node_coords, float), device=self.device)
        # per-block partial sums of the defect: room for the most blocks any variant launches (32 elements
        # per block); slots past the launched blocks stay zero
        self._partial = torch.zeros(max(int(self.lib.nzb_element_blocks(self.mesh.c_ref)), (self.E + 31) // 32),
                                    dtype=torch.float64, device=self.device)
        self._other = (None, None)  # (coordinates, DeviceMesh) of the last mesh built away from X0

    @property
    def stream(self):
        return self.mesh.stream()

    def physics_at(self, p_back):
        ph = capi.Physics()
        C.memmove(C.byref(ph), C.byref(self.phys), C.sizeof(capi.Physics))
        if p_back is not None:
            ph.p_back = float(p_back)
        return ph

    def mesh_at(self, X):
        """The device mesh at node coordinates X (this model's own when X is its base coordinates)."""
        # coordinates from the torch and NumPy contour code can differ in the last bit
        if X is None or (X.shape == self.X0.shape and torch.allclose(X.detach().to(self.device), self.X0,
                                                                     rtol=1e-14, atol=1e-15)):
            return self.mesh
        # the metric terms at X are rebuilt on the device (nzb_geometry); the connectivity is this mesh's
        Xd = X.detach().to(device=self.device, dtype=torch.float64)
        if self._other[0] is None or not torch.equal(self._other[0], Xd):
            mesh = self._other[1]
            if mesh is None:
                mesh = DeviceMesh(self.ops, self.device)
                choose_variant(mesh, self.variants)
            mesh.set_geometry(Xd, self.elem_nodes_t)
            self._other = (Xd.clone(), mesh)
        return self._other[1]

    def verts(self, X):
        """(2 NV, E) vertex coordinates of every element."""
        Xe = X.detach().to(self.device)[self.elem_nodes_t]  # (E, NV, 2)
        return torch.cat([Xe[:, :, 0].T, Xe[:, :, 1].T], 0).contiguous()

    # -- kernels -------------------------------------------------------------------
    def residual(self, U_soa, X=None, p_back=None):
        """(R, wave) at (U, X, p_back); R unfolded, SoA."""
        mesh = self.mesh_at(X)
        ph = self.physics_at(p_back)
        out = torch.empty_like(U_soa)
        wave = torch.empty(self.E, dtype=torch.float64, device=self.device)
        capi.check(self.lib.nzb_residual(C.byref(mesh.c), C.byref(ph), 0, U_soa.data_ptr(), out.data_ptr(),
                                         wave.data_ptr(), self.stream), "nzb_residual")
        return out, wave

    def _vjp(self, mode, U_soa, lam_soa, seed_soa=None, out=None, p_back=None, X=None):
        a = capi.AdjointArgs()
        a.mode = mode
        a.U, a.lam = U_soa.data_ptr(), lam_soa.data_ptr()
        a.seed = seed_soa.data_ptr() if seed_soa is not None else None
        a.out = out.data_ptr() if out is not None else None
        if mode == capi.ADJ_DEFECT:
            a.norm_partial = self._partial.data_ptr()
        ph = self.physics_at(p_back)
        capi.check(self.lib.nzb_vjp(C.byref(self.mesh_at(X).c), C.byref(ph), C.byref(a), self.stream), "nzb_vjp")

    def vjp_state(self, U_soa, lam_soa, p_back=None, X=None):
        """(dR/dU)^T lam, SoA."""
        out = torch.empty_like(U_soa)
        self._vjp(capi.ADJ_VJP, U_soa, lam_soa, out=out, p_back=p_back, X=X)
        return out

    def adjoint_rate(self, U_soa, lam_soa, seed_soa):
        """-M^-1 ((dR/dU)^T lam - seed), SoA."""
        out = torch.empty_like(U_soa)
        self._vjp(capi.ADJ_RATE, U_soa, lam_soa, seed_soa, out=out)
        return out

    def defect_rms(self, U_soa, lam_soa, seed_soa) -> float:
        """rms((dR/dU)^T lam - seed) over every entry."""
        res = torch.zeros(1, dtype=torch.float64, device=self.device)
        self._vjp(capi.ADJ_DEFECT, U_soa, lam_soa, seed_soa)
        capi.check(self.lib.nzb_norm_finalize(self._partial.data_ptr(), self._partial.numel(), 4.0 * self.E * self.NP,
                                              res.data_ptr(), self.stream), "nzb_norm_finalize")
        return float(res.item())

    def vjp_coords_vertices(self, U_soa, lam_soa, X=None, p_back=None):
        """Per element vertex (2, NV, E) d(lam . R)/dX and per element (E) d(lam . R)/dp_back."""
        X = self.X0 if X is None else X
        ph = self.physics_at(p_back)
        gvert = torch.empty(2 * self.NV * self.E, dtype=torch.float64, device=self.device)
        gpb = torch.empty(self.E, dtype=torch.float64, device=self.device)
        verts = self.verts(X)
        capi.check(self.lib.nzb_vjp_coords(C.byref(self.mesh_at(X).c), C.byref(ph), U_soa.data_ptr(),
                                           lam_soa.data_ptr(), verts.data_ptr(), self.dgs.ctypes.data, gvert.data_ptr(),
                                           gpb.data_ptr(), self.stream), "nzb_vjp_coords")
        return gvert.reshape(2, self.NV, self.E), gpb

    def vjp_coords(self, U_soa, lam_soa, X=None, p_back=None):
        """((dR/dX)^T lam as an (N_nodes, 2) tensor, (dR/dp_back)^T lam as a float)."""
        X = self.X0 if X is None else X
        gv, gpb = self.vjp_coords_vertices(U_soa, lam_soa, X, p_back)
        # element vertices -> nodes, summed in a fixed order on the host (E x NV entries)
        gv = gv.cpu().numpy()
        g = np.zeros((X.shape[0], 2))
        np.add.at(g[:, 0], self.elem_nodes.T, gv[0])
        np.add.at(g[:, 1], self.elem_nodes.T, gv[1])
        return torch.as_tensor(g, device=X.device), float(np.sum(gpb.cpu().numpy()))


class _Residual(torch.autograd.Function):
    @staticmethod
    def forward(ctx, model, U, X, p_back):
        R, _ = model.residual(U.detach().contiguous(), X.detach(), float(p_back))
        ctx.model = model
        ctx.save_for_backward(U.detach(), X.detach(), p_back.detach())
        return R

    @staticmethod
    def backward(ctx, gR):
        U, X, pb = ctx.saved_tensors
        m = ctx.model
        gR = gR.contiguous()
        gU = gX = gpb = None
        if ctx.needs_input_grad[1]:
            gU = m.vjp_state(U, gR, float(pb), X)
        if ctx.needs_input_grad[2] or ctx.needs_input_grad[3]:
            g, gp = m.vjp_coords(U, gR, X, float(pb))
            gX = g.to(dtype=X.dtype, device=X.device)
            gpb = torch.tensor(gp, dtype=pb.dtype, device=pb.device)
        return None, gU, gX, gpb


def ResidualFunction(model: AdjointModel, U_soa, X, p_back):
    """``R(U, X, p_back)`` (unfolded, SoA) as a differentiable torch function over the CUDA kernels.

    U_soa: the (4, NP, E) device state, flat; X: (N_nodes, 2) node coordinates;
    p_back: a 0-d tensor.  The forward runs the residual kernel on the mesh at
    X; the backward runs ``nzb_vjp`` (for U) and ``nzb_vjp_coords`` (for X and
    p_back).  The forward of src/sensitivity.py:230-234, the backward of
    ``jax.vjp`` on it (src/sensitivity.py:313-317,453-458).
    """
    return _Residual.apply(model, U_soa, X, p_back)


class AdjointMarch:
    """The adjoint pseudo-time march of one linearisation, as one device object."""

    def __init__(self, model: AdjointModel, U_soa, seed_soa, cfl):
        self.model = model
        lib = model.lib
        E, NP, dev = model.E, model.NP, model.device
        self.U, self.seed = U_soa.contiguous(), seed_soa.contiguous()
        n = 4 * NP * E
        z = lambda: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
        self.lam, self.Y1, self.Y2, self.f0, self.f1, self.f2 = (z() for _ in range(6))
        _, wave = model.residual(self.U)
        self.dt = torch.empty(E, dtype=torch.float64, device=dev)
        coef = step_coefficient(model.ops.ref.order, cfl, "ssprk3")
        capi.check(lib.nzb_local_dt(model.mesh.c_ref, wave.data_ptr(), coef, self.dt.data_ptr(), model.stream),
                   "nzb_local_dt")
        self.t = {
            "begin": torch.zeros(1, dtype=torch.int64, device=dev),
            "end": torch.full((1,), E, dtype=torch.int64, device=dev),
            "count": torch.full((1,), 4.0 * E * NP, dtype=torch.float64, device=dev),
            "elem_norm": torch.zeros(E, dtype=torch.float64, device=dev),
            "status": torch.zeros(1, dtype=torch.int32, device=dev),
            "iterations": torch.zeros(1, dtype=torch.int32, device=dev),
            "res0": torch.zeros(1, dtype=torch.float64, device=dev),
            "res": torch.zeros(1, dtype=torch.float64, device=dev),
            "n_running": torch.zeros(1, dtype=torch.int32, device=dev),
        }
        bf = capi.AdjointBuffers()
        bf.U, bf.seed, bf.lam = self.U.data_ptr(), self.seed.data_ptr(), self.lam.data_ptr()
        bf.Y1, bf.Y2 = self.Y1.data_ptr(), self.Y2.data_ptr()
        bf.f0, bf.f1, bf.f2 = self.f0.data_ptr(), self.f1.data_ptr(), self.f2.data_ptr()
        bf.dt = self.dt.data_ptr()
        self.bf = bf
        self.handle = None
        self.ph = model.physics_at(None)

    def _create(self, tolerance, max_iterations):
        am = capi.AdjointMarch()
        am.n_inst = 1
        for f, k in (("inst_begin", "begin"), ("inst_end", "end"), ("inst_count", "count"), ("elem_norm", "elem_norm"),
                     ("status", "status"), ("iterations", "iterations"), ("res0", "res0"), ("res", "res"),
                     ("n_running", "n_running")):
            setattr(am, f, self.t[k].data_ptr())
        am.tolerance = float(tolerance)
        am.max_iterations = int(max_iterations)
        offs = np.zeros(1, np.int64)
        h = capi.P()
        capi.check(self.model.lib.nzb_adjoint_create(1, self.model.mesh.c_ref, C.byref(self.ph), C.byref(self.bf),
                                                     offs.ctypes.data, C.byref(am), C.byref(h)), "nzb_adjoint_create")
        self.am = am
        self.handle = h.value

    def __del__(self):
        if getattr(self, "handle", None):
            self.model.lib.nzb_adjoint_destroy(self.handle)

    def run(self, n_steps: int) -> tuple[int, float, float, int]:
        capi.check(self.model.lib.nzb_adjoint_run(self.handle, int(n_steps), self.model.stream), "nzb_adjoint_run")
        return (int(self.t["status"].item()), float(self.t["res"].item()), float(self.t["res0"].item()),
                int(self.t["iterations"].item()))

    def solve(self, *, tolerance=1e-8, max_iterations=100_000, check_interval=100):
        """``(lam (SoA), residual / residual_0, iterations, converged)``, as src/sensitivity.py:289-383."""
        if max_iterations < 1 or check_interval < 1:
            raise ValueError("max_iterations and check_interval must be at least 1")
        if self.handle is None:
            self._create(tolerance, max_iterations)
        self.lam.zero_()
        for k in ("status", "iterations"):
            self.t[k].zero_()
        status, res, res0, it = self.run(0)
        if res0 == 0.0:
            return self.lam, 0.0, 0, True
        while status == 0 and it < max_iterations:
            status, res, res0, it = self.run(min(check_interval, max_iterations - it))
        return self.lam, res / res0, it, status == 1


# ---------------------------------------------------------------- objectives
def boundary_geometry(model: AdjointModel, X, tag):
    """Owner element, owner face, unit normal (n, 2) and ds (n, NQF) of one tagged boundary, from X in torch.

    The tangent of a straight edge is sum_v dgeom_dsigma[f, v] X_v, its length
    |t| = |dX/dsigma|, the outward normal (t_y, -t_x) / |t| and ds = w_q |t|
    (src/spatial/operators.py:296-303, src/post/postprocess.py:56-75).
    """
    ed = model.ops.topology.edges
    sl = model.ops.topology.tag_slice(tag)
    belem = np.asarray(ed.bedge_elem)[sl]
    bface = np.asarray(ed.bedge_face)[sl]
    T = torch.as_tensor(face_tangent_table(model.ops.ref), device=X.device)[torch.as_tensor(bface, device=X.device)]
    Xo = X[torch.as_tensor(model.elem_nodes[belem], device=X.device)]  # (n, NV, 2)
    t = torch.einsum("nv,nvd->nd", T[:, : model.NV], Xo)
    jac = torch.sqrt(t[:, 0] ** 2 + t[:, 1] ** 2)
    normal = torch.stack([t[:, 1], -t[:, 0]], -1) / jac[:, None]
    w = torch.as_tensor(np.asarray(model.ops.ref.w_face), device=X.device)
    return belem, bface, normal, jac[:, None] * w[None, :]


def boundary_state(model: AdjointModel, U, belem, bface):
    """The state at a boundary's face points with the owner-side basis: (n, NQF, 4)."""
    phi = torch.as_tensor(np.asarray(model.ops.ref.phi_face)[0][bface], device=U.device)  # (n, NP, NQF)
    return torch.einsum("kiq,kis->kqs", phi, U[torch.as_tensor(belem, device=U.device)])


def _primitives(W, g):
    rho = torch.clamp(W[..., 0], min=1e-10)
    vx, vy = W[..., 1] / rho, W[..., 2] / rho
    p = torch.clamp((g - 1.0) * (W[..., 3] - 0.5 * rho * (vx * vx + vy * vy)), min=1e-10)
    return rho, vx, vy, p


def objective_value(model: AdjointModel, U, X, name: str, params: dict):
    """A named objective of the (E, NP, 4) state U on coordinates X, in torch (src/sensitivity.py:96-130).

    thrust = 2 (int_out + int_in) (rho vx vn + p nx) ds; thrust_coefficient =
    thrust / (p_t 2 throat_half_height); mass_flow = -2 int_in rho vn ds;
    exit_mach / exit_pressure: area averages over the outflow boundary.
    """
    g = model.flow.gamma
    pt = model.flow.total_pressure
    if name not in OBJECTIVES:
        raise ValueError(f"unknown objective {name!r}; choose from {OBJECTIVES}")

    def trace(tag):
        be, bf, n, ds = boundary_geometry(model, X, tag)
        return boundary_state(model, U, be, bf), n, ds

    if name in ("thrust", "thrust_coefficient"):
        total = 0.0
        for tag in (OUTFLOW, INFLOW):
            W, n, ds = trace(tag)
            rho, vx, vy, p = _primitives(W, g)
            vn = vx * n[:, None, 0] + vy * n[:, None, 1]
            total = total + ((rho * vx * vn + p * n[:, None, 0]) * ds).sum()
        thrust = 2.0 * total
        if name == "thrust":
            return thrust
        return thrust / (pt * 2.0 * params["throat_half_height"])
    if name == "mass_flow":
        W, n, ds = trace(INFLOW)
        rho, vx, vy, _ = _primitives(W, g)
        return -2.0 * (rho * (vx * n[:, None, 0] + vy * n[:, None, 1]) * ds).sum()
    W, n, ds = trace(OUTFLOW)
    rho, vx, vy, p = _primitives(W, g)
    area = ds.sum()
    if name == "exit_mach":
        mach = torch.sqrt(vx * vx + vy * vy) / torch.sqrt(g * p / rho)
        return (mach * ds).sum() / area
    return (p * ds).sum() / area / pt


# ---------------------------------------------------------------- the case
@dataclass
class DifferentiableCase:
    """A nozzle problem set up for differentiation with respect to its design (src/sensitivity.py:134-460).

    The mesh topology and the logical grids are frozen; node coordinates, every
    metric term, the residual and the objective follow the design variables.
    """

    topology: object
    x_frac: np.ndarray
    r_frac: np.ndarray
    geometry: nz.Geometry
    flow: object
    order: int
    options: SolverOptions
    device: object = None

    # -- parameters ---------------------------------------------------------------
    def default_params(self) -> dict:
        p = dict(nz.design_params(self.geometry))
        p["back_pressure"] = float(self.flow.back_pressure)
        return p

    def params_for(self, names) -> dict:
        full = self.default_params()
        missing = [n for n in names if n not in full]
        if missing:
            raise ValueError(f"unknown design parameter(s) {missing}; choose from {tuple(full)}")
        return {n: full[n] for n in names}

    def _merged(self, params) -> dict:
        merged = dict(self.default_params())
        merged.update(params)
        return merged

    def node_coords(self, params, xp=np):
        full = self._merged(params)
        if xp is torch:
            dev = self.device if self.device is not None else "cuda"
            x = torch.as_tensor(self.x_frac, device=dev)
            r = torch.as_tensor(self.r_frac, device=dev)
            return nz.node_coords_from_params(x, r, full, self.geometry.contour, xp=torch)
        return nz.node_coords_from_params(self.x_frac, self.r_frac, {k: float(v) for k, v in full.items()},
                                          self.geometry.contour)

    def operators(self, params=None):
        return build_operators(self.topology, self.node_coords(params or {}), self.order)

    def _flow_with(self, params):
        full = self._merged(params)
        return dataclasses.replace(self.flow, back_pressure_ratio=float(full["back_pressure"]) / self.flow.total_pressure)

    def case_at(self, params=None) -> nz.Case:
        """A concrete case at these design variables on the frozen grid (src/sensitivity.py:253-267)."""
        params = dict(params or {})
        geom = nz.geometry_with(self.geometry, {k: v for k, v in params.items() if k != "back_pressure"})
        flow = self._flow_with(params)
        coords = self.node_coords(params)
        ops = build_operators(self.topology, coords, self.order)
        return nz.Case(geom, flow, self.options, self.topology, coords, ops,
                       {"x_frac": self.x_frac, "r_frac": self.r_frac})

    # -- solves --------------------------------------------------------------------
    def solve_forward(self, params=None, U0=None):
        """Converge the flow at these design variables on the frozen grid (src/sensitivity.py:269-287)."""
        cs = self.case_at(params)
        bk = B200Backend(cs.operators, cs.flow, self.options, device=self.device)
        res = march_solve(bk, cs.initial_state() if U0 is None else U0, length=float(cs.geometry.length))
        res.case = cs
        return res

    def model(self, cs) -> AdjointModel:
        return AdjointModel(cs.operators, cs.flow, self.options, self.device)

    def adjoint_solve(self, U, params, seed, *, tolerance=1e-8, max_iterations=100_000, check_interval=100,
                      model=None):
        """Solve (dR/dU)^T lam = seed by the pseudo-time march; ``(lam (E, NP, 4), rel. residual, iterations,
        converged)`` (src/sensitivity.py:289-383)."""
        m = model or self.model(self.case_at(params))
        Ut = torch.as_tensor(np.asarray(U, float), device=m.device)
        seed_t = torch.as_tensor(seed, dtype=torch.float64, device=m.device)
        am = AdjointMarch(m, to_soa(Ut), to_soa(seed_t), self.options.cfl)
        lam, rel, its, ok = am.solve(tolerance=tolerance, max_iterations=max_iterations, check_interval=check_interval)
        return from_soa(lam, m.E, m.NP), rel, its, ok

    def value_and_gradient(self, objective="thrust", params=None, *, names=None, U0=None, adjoint_tolerance=1e-8):
        """Objective value and its exact gradient (src/sensitivity.py:386-460): ``(value, grad, forward)``."""
        params = dict(params or {})
        if names is None:
            names = tuple(params.keys()) or ("area_ratio",)
        base = self.params_for(names)
        base.update({k: v for k, v in params.items() if k in names})
        fwd = self.solve_forward(base, U0=U0)
        if not fwd.converged:
            raise RuntimeError(f"the forward solve did not converge, so no gradient can be taken: {fwd.message}")
        m = self.model(fwd.case)
        dev = m.device
        U = torch.as_tensor(np.asarray(fwd.U, float), device=dev)

        # dJ/dU and the explicit dJ/da at fixed U
        P = {k: torch.tensor(float(v), dtype=torch.float64, device=dev, requires_grad=True) for k, v in base.items()}
        full = {k: (P[k] if k in P else torch.tensor(float(v), dtype=torch.float64, device=dev))
                for k, v in self._merged({}).items()}
        Ug = U.clone().requires_grad_(True)
        X = self.node_coords(full, xp=torch)
        J = objective_value(m, Ug, X, objective, full)
        grads = torch.autograd.grad(J, [Ug] + list(P.values()), allow_unused=True)
        J_U = grads[0]
        J_a = {k: (float(gk) if gk is not None else 0.0) for k, gk in zip(P, grads[1:])}

        lam, rel, its, ok = self.adjoint_solve(fwd.U, base, J_U.detach().cpu().numpy(),
                                               tolerance=adjoint_tolerance, model=m)
        if not ok:
            raise RuntimeError(f"the adjoint march stalled at relative residual {rel:.2e} after {its} iterations")

        # lam^T dR/da through the node coordinates and the back pressure
        X = self.node_coords(full, xp=torch)
        pb = full["back_pressure"]
        R = ResidualFunction(m, to_soa(U), X, pb)
        L = (to_soa(lam.to(dev)) * R).sum()
        rg = torch.autograd.grad(L, list(P.values()), allow_unused=True)
        R_a = {k: (float(gk) if gk is not None else 0.0) for k, gk in zip(P, rg)}
        grad = {k: J_a[k] - R_a[k] for k in base}
        self.last_adjoint = {"iterations": its, "relative_residual": rel, "lambda": lam}
        return float(J.detach()), grad, fwd


def differentiable_case(*, element="tri", order=1, refine=0, flow=None, options=None, device=None, **overrides):
    """A :class:`DifferentiableCase` (src/sensitivity.py:473-509).

    Keyword shortcuts as ``solve_nozzle`` takes them: fields of FlowConditions
    (``back_pressure_ratio``, ``flux`` ...) and of SolverOptions
    (``tolerance``, ``cfl`` ...) override ``flow`` / ``options``; the rest are
    geometry and mesh arguments of the case builder.
    """
    from .config import FlowConditions

    flow_f = {f.name for f in dataclasses.fields(FlowConditions)}
    opt_f = {f.name for f in dataclasses.fields(SolverOptions)}
    fkw = {k: v for k, v in overrides.items() if k in flow_f}
    okw = {k: v for k, v in overrides.items() if k in opt_f}
    gkw = {k: v for k, v in overrides.items() if k not in flow_f and k not in opt_f}
    flow = dataclasses.replace(flow or FlowConditions(), **fkw)
    options = dataclasses.replace(options or SolverOptions(), **okw)
    cs = nz.build_case(element=element, order=order, refine=refine, flow=flow, options=options, **gkw)
    return DifferentiableCase(cs.topology, np.asarray(cs.grids["x_frac"]), np.asarray(cs.grids["r_frac"]), cs.geometry,
                              cs.flow, order, cs.options, device)


def finite_difference_gradient(case: DifferentiableCase, objective="thrust", params=None, *, names=None,
                               step=1e-6, U0=None):
    """Central differences of the converged objective (src/sensitivity.py:515-555): two forward solves per
    variable, each from the quasi-1D state (or U0) on the frozen grid."""
    params = dict(params or {})
    names = tuple(names or params.keys() or ("area_ratio",))
    base = case.params_for(names)
    base.update({k: v for k, v in params.items() if k in names})

    def evaluate(p):
        fwd = case.solve_forward(p, U0=U0)
        if not fwd.converged:
            raise RuntimeError(f"forward solve did not converge at {p}: {fwd.message}")
        m = AdjointModel(fwd.case.operators, fwd.case.flow, case.options, case.device)
        U = torch.as_tensor(np.asarray(fwd.U, float), device=m.device)
        full = {k: torch.tensor(float(v), dtype=torch.float64, device=m.device) for k, v in case._merged(p).items()}
        return float(objective_value(m, U, case.node_coords(full, xp=torch), objective, full))

    grad = {}
    for k in names:
        h = step * max(1.0, abs(float(base[k])))
        up, dn = dict(base), dict(base)
        up[k] = float(base[k]) + h
        dn[k] = float(base[k]) - h
        grad[k] = (evaluate(up) - evaluate(dn)) / (2.0 * h)
    return grad


def check_gradient(case: DifferentiableCase, objective="thrust", params=None, *, names=None, step=1e-6,
                   rtol=1e-3) -> dict:
    """Adjoint against central differences, variable by variable (src/sensitivity.py:558-592)."""
    _, adj, _ = case.value_and_gradient(objective, params, names=names)
    fd = finite_difference_gradient(case, objective, params, names=names, step=step)
    out = {}
    for k in adj:
        scale = max(abs(fd[k]), 1e-12)
        out[k] = {"adjoint": adj[k], "fd": fd[k], "rel_err": abs(adj[k] - fd[k]) / scale,
                  "ok": abs(adj[k] - fd[k]) <= rtol * scale + 1e-10}
    return out




# ---------------------------------------------------------------- many members at once
class ObjectiveSpace:
    """What :func:`objective_value` reads of one mesh: its operators, flow and element vertices."""

    def __init__(self, ops, flow):
        self.ops, self.flow = ops, flow
        self.NV = 3 if ops.ref.kind == "tri" else 4
        self.elem_nodes = np.ascontiguousarray(np.asarray(ops.topology.elem_nodes)[:, : self.NV])


@dataclass
class MemberGradient:
    value: float
    grad: dict | None
    forward_status: str
    forward_iterations: int
    adjoint_converged: bool
    adjoint_iterations: int
    adjoint_residual: float


class BatchGradient:
    """Objective gradients of many design members of one case, marched together.

    Per member this is :meth:`DifferentiableCase.value_and_gradient`
    (src/sensitivity.py:386-460); all members' forward solves run as one
    batched march (:class:`~.batch.BatchSolver`), all adjoint marches as one
    ``nzb_adjoint`` object over the same concatenated mesh (each member retires
    when its own defect meets the tolerance), and one ``nzb_vjp_coords`` launch
    gives every member's ``lam^T dR/dX``.  The members share the case's
    topology, order and solver options; they differ in design variables.
    """

    def __init__(self, case: DifferentiableCase, members, objective="thrust", names=None, device=None,
                 variants: str = "batch", compact: bool = True):
        """``compact``: late in the marches, launch only the blocks that hold elements of members still
        marching (the same kernels on the same elements: the same bits)."""
        from .batch import Instance

        self.variants = variants
        self.compact = bool(compact)

        self.case = case
        self.members = [dict(m) for m in members]
        if not self.members:
            raise ValueError("no members")
        self.objective = objective
        self.names = tuple(names or self.members[0].keys())
        self.device = torch.device(device if device is not None else (case.device or "cuda"))
        self.cases = [case.case_at(m) for m in self.members]
        self.instances = [Instance(cs.operators, cs.flow, case.options, cs.initial_state(), float(cs.geometry.length), cs.geometry)
                          for cs in self.cases]

    def _params(self, i):
        merged = self.case._merged(self.members[i])
        P = {k: torch.tensor(float(merged[k]), dtype=torch.float64, device=self.device, requires_grad=True)
             for k in self.names}
        full = {k: P[k] if k in P else torch.tensor(float(v), dtype=torch.float64, device=self.device)
                for k, v in merged.items()}
        return P, full

    # adjoint status of a member whose forward solve has not retired yet (the kernels skip it), and the
    # status a running member is parked at while newly started members take their first defect
    WAITING, PARKED = 8, 9

    def run(self, *, adjoint_tolerance=1e-8, max_iterations=100_000, check_interval=100,
            overlap: bool = True) -> list[MemberGradient]:
        """Every member's value and gradient.

        ``overlap`` starts a member's adjoint march as soon as its own forward
        solve has converged, while the slower members' forward solves go on:
        each round queues one forward chunk (the forward check interval) on the
        current stream and one adjoint chunk (``check_interval`` RK4 steps) on a
        second stream, so the two run side by side on the device; between
        rounds the members whose forward solves retired get their seeds and
        frozen local steps and join the adjoint march.  ``overlap=False`` runs
        every forward solve to retirement first, then every adjoint.  With
        ``variants="single"`` a member's gradient is the same, bit for bit,
        either way: its seed, step and march depend on its own converged state
        only.  In the default batch context the forward and adjoint marches
        switch to the single-solve variants for their tails (few elements still
        marching), at a point that depends on the whole batch, so the two
        orders agree to round-off.
        """
        from .batch import BatchSolver, blocks_of

        import time

        lib = capi.load()
        dev = self.device
        clock = [time.perf_counter()]
        self.timings = {}

        def lap(name):
            torch.cuda.synchronize(dev)
            clock.append(time.perf_counter())
            self.timings[name] = self.timings.get(name, 0.0) + clock[-1] - clock[-2]

        fwd = BatchSolver(self.instances, device=dev, variants=self.variants, compact=self.compact)
        if len(fwd.meshes) != 1:
            raise NotImplementedError("the members of one batch share the element kind and order")
        dm = fwd.meshes[0]
        S0 = fwd.buffers[0][1][0]
        E, NP, NV, n = dm.E, dm.np_, dm.nf, len(self.members)
        main = torch.cuda.current_stream(dev)
        side = torch.cuda.Stream(dev)
        spans = [(int(fwd.local[i]), int(fwd.local[i]) + cs.operators.n_elem) for i, cs in enumerate(self.cases)]
        values = [float("nan")] * n
        J_a = [None] * n

        # the adjoint march over the forward's concatenated mesh: it reads the forward state buffer, whose
        # slices freeze when their members retire; every member waits until its forward solve converges
        size = 4 * NP * E
        z = lambda: torch.zeros(size, dtype=torch.float64, device=dev)  # noqa: E731
        seed_soa, lam, Y1, Y2, f0, f1, f2, scratch = (z() for _ in range(8))
        wave = torch.zeros(E, dtype=torch.float64, device=dev)
        dt = torch.zeros(E, dtype=torch.float64, device=dev)
        dt_new = torch.zeros(E, dtype=torch.float64, device=dev)
        status = torch.full((n,), self.WAITING, dtype=torch.int32, device=dev)
        mesh = capi.Mesh()
        C.memmove(C.byref(mesh), C.byref(dm.c), C.sizeof(capi.Mesh))
        mesh.inst_status = status.data_ptr()
        ph = fwd.phys[0]
        bf = capi.AdjointBuffers()
        bf.U, bf.seed, bf.lam, bf.Y1, bf.Y2 = (t.data_ptr() for t in (S0, seed_soa, lam, Y1, Y2))
        bf.f0, bf.f1, bf.f2, bf.dt = (t.data_ptr() for t in (f0, f1, f2, dt))
        t = {"elem_norm": torch.zeros(E, dtype=torch.float64, device=dev),
             "iterations": torch.zeros(n, dtype=torch.int32, device=dev),
             "res0": torch.zeros(n, dtype=torch.float64, device=dev),
             "res": torch.zeros(n, dtype=torch.float64, device=dev),
             "n_running": torch.zeros(1, dtype=torch.int32, device=dev)}
        am = capi.AdjointMarch()
        am.n_inst = n
        am.inst_begin, am.inst_end, am.inst_count = (fwd.t[k].data_ptr() for k in ("begin", "end", "count"))
        am.elem_norm, am.status = t["elem_norm"].data_ptr(), status.data_ptr()
        am.iterations, am.res0, am.res = (t[k].data_ptr() for k in ("iterations", "res0", "res"))
        am.n_running = t["n_running"].data_ptr()
        am.tolerance = float(adjoint_tolerance)
        am.max_iterations = int(max_iterations)
        offs = np.zeros(1, np.int64)
        elem_count = np.asarray([hi - lo for lo, hi in spans], np.int64)
        handles = {}  # adjoint march object -> its block list (kept alive with it)

        def variant_mesh(context):
            mc = capi.Mesh()
            C.memmove(C.byref(mc), C.byref(mesh), C.sizeof(capi.Mesh))
            if context is not None:
                set_struct_variant(mc, dm.kind, dm.order, context)
            return mc

        def blocks_for(context, mask):
            W = int(lib.nzb_block_width(C.byref(variant_mesh(context)), 1))
            return blocks_of([spans[i] for i in range(n) if mask[i]] if mask is not None else [(0, E)], W)

        def adjoint_handle(context, mask):
            """An adjoint march object over the shared buffers: the bucket's batch variant, or that of
            ``context``; with ``mask``, launching only the blocks that hold those members' elements.
            Returns the object and the blocks one launch spans."""
            mc = variant_mesh(context)
            blocks = blocks_for(context, mask)
            keep = None
            if mask is not None:
                keep = torch.as_tensor(blocks if blocks.size else np.zeros(1, np.int32), device=dev)
                mc.vjp_blocks, mc.n_vjp_blocks = keep.data_ptr(), int(blocks.size)
            hh = capi.P()
            capi.check(lib.nzb_adjoint_create(1, C.byref(mc), C.byref(ph), C.byref(bf), offs.ctypes.data,
                                              C.byref(am), C.byref(hh)), "nzb_adjoint_create")
            handles[hh.value] = keep
            return hh.value, int(blocks.size)

        # Late in the march (few members left, or few blocks holding them) the adjoint switches to the
        # single-solve variant and to a march object that lists only the blocks of members still
        # marching or yet to start, as the forward batch does (BatchSolver._retarget).
        first_h, launched = adjoint_handle(None, None)
        cur = [first_h]
        tail_at = tail_elements() if self.variants == "batch" else 0
        in_tail = False
        self.tail_switched = {"forward": None, "adjoint": None}
        self.compactions = {"forward": 0, "adjoint": 0}
        coef = step_coefficient(self.cases[0].operators.ref.order, self.case.options.cfl, "ssprk3")
        started = np.zeros(n, bool)
        elem_inst = dm.elem_inst_t

        def start(members, fst):
            """Seeds, frozen steps and first defects of members whose forward solves have retired."""
            conv = [i for i in members if fst[i] == 1]
            for i in members:
                started[i] = True
            if not conv:
                return
            U_all = dm.unpack(S0)
            seed = dm.unpack(seed_soa)
            for i in conv:  # dJ/dU and the explicit dJ/da (boundary integrals in torch)
                lo, hi = spans[i]
                P, full = self._params(i)
                Ui = U_all[lo:hi].clone().requires_grad_(True)
                X = self.case.node_coords(full, xp=torch)
                J = objective_value(ObjectiveSpace(self.cases[i].operators, self.cases[i].flow), Ui, X, self.objective,
                                    full)
                g = torch.autograd.grad(J, [Ui] + list(P.values()), allow_unused=True)
                seed[lo:hi] = g[0]
                values[i] = float(J.detach())
                J_a[i] = {k: float(gk) if gk is not None else 0.0 for k, gk in zip(P, g[1:])}
            seed_soa.copy_(to_soa(seed))
            # the frozen local step of the new members from their converged states (the residual runs on
            # their elements only), written into their slices of dt
            idx = torch.as_tensor(conv, dtype=torch.int32, device=dev)
            only = torch.ones(n, dtype=torch.int32, device=dev)
            only[idx.long()] = 0
            one = capi.Mesh()
            C.memmove(C.byref(one), C.byref(mesh), C.sizeof(capi.Mesh))
            one.inst_status = only.data_ptr()
            capi.check(lib.nzb_residual(C.byref(one), C.byref(ph), 0, S0.data_ptr(), scratch.data_ptr(),
                                        wave.data_ptr(), main.cuda_stream), "nzb_residual")
            capi.check(lib.nzb_local_dt(C.byref(one), wave.data_ptr(), coef, dt_new.data_ptr(), main.cuda_stream),
                       "nzb_local_dt")
            new_elem = torch.isin(elem_inst, idx)
            dt.copy_(torch.where(new_elem, dt_new, dt))
            # first defect (res0) of the new members alone: the running ones are parked meanwhile
            running = status == 0
            status.copy_(torch.where(running, torch.full_like(status, self.PARKED), status))
            status[idx.long()] = 0
            capi.check(lib.nzb_adjoint_run(cur[0], 0, main.cuda_stream), "nzb_adjoint_run")
            status.copy_(torch.where(running, torch.zeros_like(status), status))

        try:
            fwd_running = fwd.step_chunk(1, True)
            fchunk = min(max(1, fwd.opts.check_interval), fwd.opts.max_iterations)
            adj_running = 0
            # forward chunks per round: as many as take about as long as one adjoint chunk, so neither
            # stream waits long for the other at the round's end (re-measured every round)
            per_round = 1
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
            while True:
                fst = fwd.t["status"].cpu().numpy()
                new = [i for i in range(n) if not started[i] and fst[i] != 0]
                if new and (overlap or not fwd_running):
                    if not overlap:
                        lap("forward")
                    start(new, fst)
                    adj_running = int((status == 0).sum().item())
                # the adjoint stream starts after this round's set-up, before the forward chunks are queued,
                # so the two run side by side
                side.wait_stream(main)
                nf = 0
                if fwd_running:
                    ev[0].record(main)
                    for _ in range(per_round if adj_running else 1):
                        if fwd.done >= fwd.opts.max_iterations:
                            break
                        fwd.launch_chunk(min(fchunk, fwd.opts.max_iterations - fwd.done), False)
                        nf += 1
                    ev[1].record(main)
                if adj_running:
                    ev[2].record(side)
                    capi.check(lib.nzb_adjoint_run(cur[0], check_interval, side.cuda_stream), "nzb_adjoint_run")
                    ev[3].record(side)
                main.wait_stream(side)
                if not fwd_running and not adj_running:
                    break
                if fwd_running:
                    fwd_running = fwd.n_running() if fwd.done < fwd.opts.max_iterations else 0
                    fwd._retarget(fwd_running)
                    self.tail_switched["forward"] = fwd.tail_switched_at
                    self.compactions["forward"] = fwd.compactions
                if adj_running:
                    adj_running = int(t["n_running"].item())
                    if adj_running:
                        # members marching, still in their forward solve, or converged and not started yet
                        fst_now = fwd.t["status"].cpu().numpy()
                        mask = (status.cpu().numpy() == 0) | (fst_now == 0) | ((fst_now == 1) & ~started)
                        tail = in_tail or (tail_at > 0 and int(elem_count[mask].sum()) <= tail_at)
                        need = int(blocks_for("single" if tail else None, mask).size)
                        if tail != in_tail or (self.compact and 2 * need <= launched):
                            old_h = cur[0]
                            cur[0], launched = adjoint_handle("single" if tail else None,
                                                              mask if self.compact else None)
                            lib.nzb_adjoint_destroy(old_h)
                            del handles[old_h]
                            self.compactions["adjoint"] += 1
                            if tail and not in_tail:
                                in_tail = True
                                self.tail_switched["adjoint"] = int(t["iterations"].max().item())
                    if nf:
                        t_f = ev[0].elapsed_time(ev[1]) / nf
                        t_a = ev[2].elapsed_time(ev[3])
                        per_round = max(1, min(64, int(round(t_a / max(t_f, 1e-3)))))
            lap("adjoint" if not overlap else "forward+adjoint")
        finally:
            for hh in list(handles):
                lib.nzb_adjoint_destroy(hh)
            handles.clear()
        fres = fwd.results(with_state=False)
        ast = status.cpu().numpy()
        its = t["iterations"].cpu().numpy()
        rel = (t["res"] / torch.where(t["res0"] > 0, t["res0"], torch.ones_like(t["res0"]))).cpu().numpy()

        # lam^T dR/dX of every member whose adjoint converged, in one launch
        include = torch.where(status == 1, 0, 7).to(torch.int32)
        mesh.inst_status = include.data_ptr()
        verts_h = np.concatenate([np.asarray(cs.operators.node_coords)[ObjectiveSpace(cs.operators, cs.flow).elem_nodes]
                                  for cs in self.cases])  # (E, NV, 2)
        verts = torch.as_tensor(np.ascontiguousarray(np.concatenate([verts_h[:, :, 0].T, verts_h[:, :, 1].T])),
                                device=dev)
        gvert = torch.zeros(2 * NV * E, dtype=torch.float64, device=dev)
        gpb = torch.zeros(E, dtype=torch.float64, device=dev)
        dgs = np.ascontiguousarray(face_tangent_table(self.cases[0].operators.ref).ravel())
        stream = dm.stream()
        capi.check(lib.nzb_vjp_coords(C.byref(mesh), C.byref(ph), S0.data_ptr(), lam.data_ptr(), verts.data_ptr(),
                                      dgs.ctypes.data, gvert.data_ptr(), gpb.data_ptr(), stream), "nzb_vjp_coords")
        gv = gvert.reshape(2, NV, E).cpu().numpy()
        gp = gpb.cpu().numpy()

        out = []
        for i, cs in enumerate(self.cases):
            grad = None
            if ast[i] == 1:
                lo, hi = spans[i]
                en = ObjectiveSpace(cs.operators, cs.flow).elem_nodes
                g = np.zeros((np.asarray(cs.operators.node_coords).shape[0], 2))
                np.add.at(g[:, 0], en.T, gv[0][:, lo:hi])
                np.add.at(g[:, 1], en.T, gv[1][:, lo:hi])
                P, full = self._params(i)
                X = self.case.node_coords(full, xp=torch)
                L = (torch.as_tensor(g, device=dev) * X).sum() + float(np.sum(gp[lo:hi])) * full["back_pressure"]
                rg = torch.autograd.grad(L, list(P.values()), allow_unused=True)
                grad = {k: J_a[i][k] - (float(gk) if gk is not None else 0.0) for k, gk in zip(P, rg)}
            out.append(MemberGradient(values[i], grad, fres[i].status, fres[i].iterations, bool(ast[i] == 1),
                                      int(its[i]), float(rel[i])))
        lap("contraction")
        return out


__all__ = ["OBJECTIVES", "FLOW_DESIGN_PARAMETERS", "AdjointModel", "AdjointMarch", "ResidualFunction",
           "DifferentiableCase", "differentiable_case", "objective_value", "finite_difference_gradient",
           "check_gradient", "face_tangent_table", "to_soa", "from_soa", "BatchGradient", "MemberGradient",
           "ObjectiveSpace"]
