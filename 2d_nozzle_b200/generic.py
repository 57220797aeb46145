"""The drop-in backend for orders above 3 and curved (Q = 2) elements.

``B200Backend(ops, flow, opts)`` returns this class when the mesh is outside
what the specialised kernels are instantiated for (straight-sided elements of
order 0..3).  It runs the ``nzb_gen_*`` kernels (csrc/generic.cuh) on the
reference's own per-element operators (src/spatial/operators.py:139-206),
uploaded once in the reference's layout: an edge pass and an element pass per
rate, the positivity limiter in place, the SSP-RK3 / forward-Euler stages with
the local step and the weighted norm -- the reference's compiled step
(src/backends/numba_backend.py:283-337) on the GPU.  The interface is the
reference's ``Backend`` (src/backends/base.py:81-201), as ``B200Backend``'s.

With ``device_metrics=True`` (or lean operators) the coordinate-dependent
operators are built on the device from the node coordinates instead
(``nzb_gen_geometry``, csrc/gen_geometry.cuh): the curved (Q = 2) metric terms
at every volume and face point, the inverse mass matrices and the folded
operators.

The limiter is the positivity limiter (``nzb_gen_limit``) or the Superbee
slope limiter followed by it (``nzb_gen_superbee``), as the reference's
``apply_limiter`` runs them.

``initial_state`` projects the quasi-1D state on the device
(``nzb_gen_initial_state``, csrc/gen_initial.cuh), curved elements included.

``performance`` integrates the parity observables on the device
(``nzb_gen_observables``, csrc/gen_observe.cuh).

Not here: batches and the adjoint, which take straight elements of order 0..3.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from .backend import B200Backend
from .config import SCHEMES, recommended_scheme
from .layout import physics_struct


def needs_generic(ops) -> bool:
    """Whether a mesh is outside the specialised kernels: order above 3 or curved elements."""
    from .layout import MAX_ORDER

    return int(ops.ref.order) > MAX_ORDER or int(getattr(ops.topology, "geometry_order", 1)) != 1


class GenericB200Backend(B200Backend):
    name = "b200"

    def __init__(self, ops, flow, opts, *, device=None, variants: str = "auto", device_metrics: bool = False, **_):
        """``device_metrics``: build the coordinate-dependent operators (gradients, inverse mass, folded
        operators, edge normals and Jacobians, areas, mean weights) on the device from the node
        coordinates (``nzb_gen_geometry``) instead of uploading the host's; ``ops`` may then be lean."""
        import torch

        self.torch = torch
        self.ops, self.flow, self.opts = ops, flow, opts
        if opts.limiter not in ("positivity", "superbee", "none"):
            raise ValueError(f"unknown limiter {opts.limiter!r}")
        self.scheme = recommended_scheme(ops.ref.order) if opts.scheme is None else opts.scheme
        if self.scheme not in SCHEMES:
            raise ValueError(f"unknown scheme {self.scheme!r}; choose from {SCHEMES}")
        # lean operators (no per-element gradients) get theirs built on the device
        device_metrics = bool(device_metrics) or getattr(ops, "grad_x", None) is None \
            or getattr(ops, "face_basis_m", None) is None
        self.device_built = bool(device_metrics)
        self.n_limited = 0
        self.n_mean_repaired = 0
        self.n_limit_calls = 0
        a_t = flow.stagnation_sound_speed
        self.component_weight = np.array([1.0, 1.0 / a_t, 1.0 / a_t, 1.0 / a_t**2]).reshape(1, 1, 4)
        self.lib = capi.load()
        dev = torch.device(device if device is not None else "cuda")
        if dev.type != "cuda":
            raise capi.NativeError("the B200 backend runs on a CUDA device only")
        self.device = dev
        ref, topo = ops.ref, ops.topology
        ed = topo.edges
        E, NP = int(ops.n_elem), int(ref.n_basis)
        NQV, NQF = int(np.asarray(ref.phi_vol).shape[1]), int(np.asarray(ref.w_face).shape[0])
        NF = int(np.asarray(ed.face_edge).shape[1])
        n_int, n_bnd = int(ops.n_interior), int(ops.n_boundary)
        self.E, self.NP, self.n_edge = E, NP, n_int + n_bnd
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, float)), device=dev)  # noqa: E731
        i32 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a).astype(np.int32)), device=dev)  # noqa: E731
        be, bf = np.asarray(ed.bedge_elem), np.asarray(ed.bedge_face)
        side = np.asarray(ed.face_side)
        self._arr = {
            "phi_vol": f64(ref.phi_vol), "phi_face": f64(ref.phi_face), "w_face": f64(ref.w_face),
            "face_edge": i32(ed.face_edge), "face_side": i32(side),
            "face_sign": f64(np.where(side == 0, 1.0, -1.0)),
            "edge_elem": i32(np.concatenate([np.asarray(ed.iedge_elem).reshape(-1, 2), np.stack([be, be], 1)])),
            "edge_face": i32(np.concatenate([np.asarray(ed.iedge_face).reshape(-1, 2), np.stack([bf, bf], 1)])),
            "edge_tag": i32(np.asarray(ed.bedge_tag) if n_bnd else np.zeros(1)),
        }
        if device_metrics:
            self._build_operators(ops, dev, E, NP, NQV, NQF, NF, n_int + n_bnd, f64, i32)
        else:
            for k in ("grad_x", "grad_y", "grad_x_m", "grad_y_m", "face_basis_m", "edge_normal", "edge_jac",
                      "edge_length", "elem_area", "mean_weights"):
                self._arr[k] = f64(getattr(ops, k))
        m = capi.GenMesh()
        m.np, m.nqv, m.nqf, m.nface = NP, NQV, NQF, NF
        m.n_elem, m.n_int, m.n_bnd = E, n_int, n_bnd
        for k, t in self._arr.items():
            if k != "inv_mass":
                setattr(m, k, t.data_ptr())
        self.gm = m
        self._gm = C.byref(m)
        if device_metrics:
            capi.check(self.lib.nzb_gen_geometry(self._gm, C.byref(self._geo_args), self._stream), "nzb_gen_geometry")
            if int(self._bad.item()):
                raise ValueError(f"{int(self._bad.item())} quadrature point(s) have a non-positive Jacobian")
        self.phys = physics_struct(flow, opts, ref)
        self._phys_ref = C.byref(self.phys)
        z = lambda n: torch.zeros(n, dtype=torch.float64, device=dev)  # noqa: E731
        n = E * NP * 4
        self._S = [z(n) for _ in range(3)]
        self._F = [z(n) for _ in range(3)]
        self._wave, self._dt = z(E), z(E)
        self._fw, self._smax = z(self.n_edge * NQF * 4), z(self.n_edge)
        self._nb = int(self.lib.nzb_gen_blocks(self._gm))
        self._partial = z(self._nb)
        self._res = z(1)
        self._counters = torch.zeros(2, dtype=torch.int64, device=dev)
        self._minv = self._arr["inv_mass"].view(E, NP, NP) if device_metrics else None
        if opts.limiter == "superbee":
            # each element's share of the domain area, as the reference forms it (A_e / sum A)
            area = self._arr["elem_area"].cpu().numpy()
            self._share = f64(area / area.sum())
            self._means, self._scale = z(4 * E), z(4)
        self._obs = None
        self._solvers = {}

    def _build_operators(self, ops, dev, E, NP, NQV, NQF, NF, n_edge, f64, i32):
        """Output arrays and arguments of nzb_gen_geometry (the coordinate-dependent operators built on
        the device from the topology's geometry nodes and the node coordinates)."""
        import torch

        ref, topo = ops.ref, ops.topology
        X = np.asarray(ops.node_coords, float)
        en = np.asarray(topo.elem_nodes)
        NG = int(en.shape[1])
        if en.shape[0] != E or en.min() < 0 or en.max() >= X.shape[0]:
            raise ValueError("elem_nodes must index the node coordinates, one row per element")
        side = np.asarray(topo.edges.face_side)
        if side.min(initial=0) < 0 or side.max(initial=0) > 1:
            raise ValueError("face_side must be 0 or 1")
        shapes = {"dgeom_dxi_vol": (NG, NQV), "dgeom_deta_vol": (NG, NQV), "dphi_dxi_vol": (NP, NQV),
                  "dphi_deta_vol": (NP, NQV), "w_vol": (NQV,), "dgeom_dsigma_face": (NF, NG, NQF)}
        for name, shape in shapes.items():
            if np.asarray(getattr(ref, name)).shape != shape:
                raise ValueError(f"reference table {name} has shape {np.asarray(getattr(ref, name)).shape}, "
                                 f"expected {shape}")
        z = lambda *shape: torch.zeros(shape, dtype=torch.float64, device=dev)  # noqa: E731
        self._arr.update({
            "grad_x": z(E, NP, NQV), "grad_y": z(E, NP, NQV), "grad_x_m": z(E, NP, NQV), "grad_y_m": z(E, NP, NQV),
            "face_basis_m": z(E, NF, NP, NQF), "inv_mass": z(E, NP, NP), "elem_area": z(E), "mean_weights": z(E, NP),
            "edge_normal": z(n_edge, NQF, 2), "edge_jac": z(n_edge, NQF), "edge_length": z(n_edge),
        })
        self._geo_in = {"X": f64(X), "elem_nodes": i32(en), "w_vol": f64(ref.w_vol), "dphi_dxi": f64(ref.dphi_dxi_vol),
                        "dphi_deta": f64(ref.dphi_deta_vol), "dgeom_dxi": f64(ref.dgeom_dxi_vol),
                        "dgeom_deta": f64(ref.dgeom_deta_vol), "dgeom_dsigma": f64(ref.dgeom_dsigma_face)}
        self._bad = torch.zeros(1, dtype=torch.int32, device=dev)
        a = capi.GenGeometryArgs()
        a.ng = NG
        for k, t in self._geo_in.items():
            setattr(a, k, t.data_ptr())
        for k in ("grad_x", "grad_y", "grad_x_m", "grad_y_m", "face_basis_m", "inv_mass", "elem_area", "mean_weights",
                  "edge_normal", "edge_jac", "edge_length"):
            setattr(a, k, self._arr[k].data_ptr())
        a.bad = self._bad.data_ptr()
        self._geo_args = a
        self.h2d_bytes = sum(t.numel() * t.element_size() for t in self._geo_in.values())

    # -- helpers ----------------------------------------------------------------
    @property
    def _stream(self):
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def _put(self, U, dst):
        t = self.torch.as_tensor(np.ascontiguousarray(np.asarray(U, float)).reshape(-1), device=self.device)
        if t.numel() != dst.numel():
            raise ValueError(f"state has {t.numel()} values, expected {dst.numel()} ((E, NP, 4) = ({self.E}, {self.NP}, 4))")
        dst.copy_(t)
        return dst

    def _get(self, t) -> np.ndarray:
        return t.detach().to("cpu").numpy().reshape(self.E, self.NP, 4)

    def _rate_into(self, src, out, unfolded=0):
        capi.check(self.lib.nzb_gen_rate(self._gm, self._phys_ref, unfolded, src.data_ptr(), out.data_ptr(),
                                         self._wave.data_ptr(), self._fw.data_ptr(), self._smax.data_ptr(),
                                         self._stream), "nzb_gen_rate")

    def _limit_into(self, t):
        if not self._limiter_on():
            return
        if self.opts.limiter == "superbee" and self.ops.ref.order > 0:
            capi.check(self.lib.nzb_gen_superbee(self._gm, self._phys_ref, t.data_ptr(), self._share.data_ptr(),
                                                 self._means.data_ptr(), self._scale.data_ptr(),
                                                 self._counters.data_ptr(), self._stream), "nzb_gen_superbee")
        else:
            capi.check(self.lib.nzb_gen_limit(self._gm, self._phys_ref, t.data_ptr(), self._counters.data_ptr(),
                                              self._stream), "nzb_gen_limit")

    def _update(self, stage, V, U0, F, out, a=0.0, b=1.0):
        args = capi.GenUpdateArgs()
        args.stage = stage
        args.dt_factor = self.positivity_scale() * _step_coefficient(self.ops.ref.order, self.opts.cfl, self.scheme)
        args.a, args.b = a, b
        args.V, args.F, args.wave, args.dt, args.out = (x.data_ptr() for x in (V, F, self._wave, self._dt, out))
        args.U0 = U0.data_ptr() if U0 is not None else None
        args.partial = self._partial.data_ptr() if stage == 1 else None
        capi.check(self.lib.nzb_gen_update(self._gm, self._phys_ref, C.byref(args), self._stream), "nzb_gen_update")
        if stage == 1:
            capi.check(self.lib.nzb_norm_finalize(self._partial.data_ptr(), self._nb, 4.0 * self.E * self.NP,
                                                  self._res.data_ptr(), self._stream), "nzb_norm_finalize")

    # -- primitives -----------------------------------------------------------
    def _eval(self, U, unfolded):
        src = self._put(U, self._S[0])
        self._rate_into(src, self._S[1], unfolded)
        return self._get(self._S[1]), self._wave.detach().cpu().numpy()

    def residual(self, U):
        """``(R, wave)`` with ``M dU/dt = -R`` (src/backends/base.py:118-120)."""
        return self._eval(U, 1)

    def rate(self, U):
        """``(-M^-1 R, wave)``: the folded operators, one pass."""
        return self._eval(U, 0)

    def inverse_mass(self, R):
        if self._minv is None:
            self._minv = self.torch.as_tensor(np.ascontiguousarray(np.asarray(self.ops.inv_mass, float)), device=self.device)
        Rt = self._put(R, self._S[0]).view(self.E, self.NP, 4)
        return self.torch.bmm(self._minv, Rt).cpu().numpy()

    def limit(self, U):
        if not self._limiter_on():
            return np.asarray(U)
        st = self._put(U, self._S[0])
        self._limit_into(st)
        out = self._get(st)
        self._take_counters(1)
        return out

    def limit_flags(self, U):
        raise NotImplementedError("per-element limiter flags come from the specialised kernels (order <= 3, straight)")

    def norm(self, A) -> float:
        t = self._put(A, self._S[0]).view(-1, 4)
        w = self.torch.as_tensor(self.component_weight.reshape(4), device=self.device)
        return float(((t * w) ** 2).mean().sqrt().item())

    def initial_state(self, geometry, host: bool = True):
        """The quasi-1D initial state of this mesh (src/timestepping/initialize.py:41-102, the reference's
        ``initial_condition="quasi1d"``) projected on the device (``nzb_gen_initial_state``) from the node
        coordinates, the nozzle ``geometry`` and this backend's flow: the reference-layout (E, NP, 4) host
        array, or with ``host=False`` the device tensor of that layout."""
        from .nozzle import quasi1d_table, wall_parameters

        torch = self.torch
        ops, ref = self.ops, self.ops.ref
        dev = self.device
        f64 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, float)), device=dev)  # noqa: E731
        X = np.asarray(ops.node_coords, float)
        en = np.asarray(ops.topology.elem_nodes)
        if en.shape[0] != self.E or en.min() < 0 or en.max() >= X.shape[0]:
            raise ValueError("elem_nodes must index the node coordinates, one row per element")
        NG, NQV = int(en.shape[1]), int(np.asarray(ref.phi_vol).shape[1])
        for name in ("geom_vol", "dgeom_dxi_vol", "dgeom_deta_vol"):
            if np.asarray(getattr(ref, name)).shape != (NG, NQV):
                raise ValueError(f"reference table {name} does not match the elements' {NG} geometry nodes")
        if self._minv is None:
            self._minv = f64(ops.inv_mass)
        table = quasi1d_table(geometry, self.flow)
        keep = {"X": f64(X), "elem_nodes": torch.as_tensor(np.ascontiguousarray(en.astype(np.int32)), device=dev),
                "geom_vol": f64(ref.geom_vol), "dgeom_dxi": f64(ref.dgeom_dxi_vol), "dgeom_deta": f64(ref.dgeom_deta_vol),
                "w_vol": f64(ref.w_vol), "wall": f64(wall_parameters(geometry)), "q1d": f64(table)}
        out = torch.empty(self.E * self.NP * 4, dtype=torch.float64, device=dev)
        a = capi.GenInitialArgs()
        a.ng = NG
        for k, t in keep.items():
            setattr(a, k, t.data_ptr())
        a.inv_mass = self._minv.data_ptr()
        a.n_q1d = int(table.shape[1])
        a.out = out.data_ptr()
        capi.check(self.lib.nzb_gen_initial_state(self._gm, self._phys_ref, C.byref(a), self._stream),
                   "nzb_gen_initial_state")
        if host:
            return self._get(out)
        torch.cuda.current_stream(dev).synchronize()  # the inputs above are freed on return
        return out.view(self.E, self.NP, 4)

    def performance(self, U, geom=None) -> dict:
        """The performance() metrics of a state (src/post/postprocess.py:193-255), integrated on the device
        (``nzb_gen_observables``); ``geom`` adds the throat-normalised coefficients and the ideal thrust."""
        from .observables import entropy_reference, from_sums

        torch = self.torch
        if self._obs is None:
            ops, ref = self.ops, self.ops.ref
            dev = self.device
            f64 = lambda a: torch.as_tensor(np.ascontiguousarray(np.asarray(a, float)), device=dev)  # noqa: E731
            en = np.asarray(ops.topology.elem_nodes)
            X = np.asarray(ops.node_coords, float)
            if en.shape[0] != self.E or en.min() < 0 or en.max() >= X.shape[0]:
                raise ValueError("elem_nodes must index the node coordinates, one row per element")
            self._obs = {"X": f64(X), "elem_nodes": torch.as_tensor(np.ascontiguousarray(en.astype(np.int32)), device=dev),
                         "dgeom_dxi": f64(ref.dgeom_dxi_vol), "dgeom_deta": f64(ref.dgeom_deta_vol),
                         "w_vol": f64(ref.w_vol), "out": torch.zeros(capi.NOBS, dtype=torch.float64, device=dev)}
        src = self._put(U, self._S[0])
        a = capi.GenObsArgs()
        a.ng = int(np.asarray(self.ops.topology.elem_nodes).shape[1])
        for k in ("X", "elem_nodes", "dgeom_dxi", "dgeom_deta", "w_vol", "out"):
            setattr(a, k, self._obs[k].data_ptr())
        a.U = src.data_ptr()
        a.s_t = entropy_reference(self.flow)
        a.r_gas = float(self.flow.Rgas)
        capi.check(self.lib.nzb_gen_observables(self._gm, self._phys_ref, C.byref(a), self._stream),
                   "nzb_gen_observables")
        return from_sums(self._obs["out"].cpu().numpy(), self.flow, geom)

    def step_record(self, U, scheme: str | None = None):
        raise NotImplementedError("stage-by-stage limiter flags come from the specialised kernels")

    # -- the march ---------------------------------------------------------------
    def run_device(self, n_steps: int, scheme: str | None = None) -> None:
        """Advance the device-resident state (``self._S[0]``) by ``n_steps``: per stage a rate (edge and element
        passes), the update and the limiter in place, as the reference's fused step orders them."""
        scheme = scheme or self.scheme
        S0, S1, S2 = self._S
        F0, F1, F2 = self._F
        for _ in range(int(n_steps)):
            self._rate_into(S0, F0)
            if scheme == "euler":
                self._update(1, S0, None, F0, S1)
                self._limit_into(S1)
                S0.copy_(S1)
                continue
            self._update(1, S0, None, F0, S2)
            self._limit_into(S2)
            self._rate_into(S2, F1)
            self._update(2, S2, S0, F1, S1, 0.75, 0.25)
            self._limit_into(S1)
            self._rate_into(S1, F2)
            self._update(3, S1, S0, F2, S0, 1.0 / 3.0, 2.0 / 3.0)
            self._limit_into(S0)

    def run(self, U, n_steps: int, scheme: str):
        """Advance ``n_steps`` steps; returns a fresh ``(U, residual of the last step)``."""
        if scheme not in SCHEMES:
            raise ValueError(f"unknown scheme {scheme!r}; choose from {SCHEMES}")
        self._put(U, self._S[0])
        self.run_device(n_steps, scheme)
        out = self._get(self._S[0])
        res = float(self._res.item())
        self._take_counters((3 if scheme == "ssprk3" else 1) * int(n_steps))
        return out, res


def _step_coefficient(order, cfl, scheme):
    from .config import step_coefficient

    return step_coefficient(order, cfl, scheme)
