"""The drop-in backend: the reference's ``Backend`` interface on the B200 kernels.

Straight elements of order 0..3 run the specialised kernels here; other meshes
(orders above 3, curved elements) get :class:`~.generic.GenericB200Backend`
from the same constructor.

``B200Backend(ops, flow, opts)`` has the constructor, attributes and methods of
the reference's ``Backend`` (src/backends/base.py:81-201) -- ``residual``,
``inverse_mass``, ``limit``, ``time_step``, ``norm``, ``rate``,
``euler_step``, ``ssprk3_step``, ``make_step``, ``run``,
``positivity_scale``, ``limiter_activity``, ``asarray``, ``to_numpy``, the
counters ``n_limited`` / ``n_mean_repaired`` / ``n_limit_calls`` and the
resolved ``scheme`` -- so ``march`` / ``solve_steady`` / ``solve_nozzle`` /
``sweep`` drive it unchanged once ``get_backend`` returns it.

Arrays crossing the interface are host NumPy arrays in the reference layout
``(E, NP, 4)``, as the reference's backends return them.  ``run`` copies the
state in once and out once per chunk; every step in between runs on the device
as a captured CUDA graph of three fused stage kernels (the reference's
``NumbaBackend.run``, src/backends/numba_backend.py:283-337).

Configuration errors raise at construction, as the reference does
(src/backends/numba_backend.py:55-66, src/backends/base.py:181-186).
Numerical failure never raises: it shows up as a non-finite residual.
"""

from __future__ import annotations

import numpy as np

from . import capi
from .config import FLOOR, SCHEMES, recommended_scheme, step_coefficient
from .autotune import choose_variant, context_for
from .layout import DeviceMesh, physics_struct


class B200Backend:
    name = "b200"

    def __new__(cls, ops, flow, opts, **kw):
        # orders above 3 and curved elements run the kernels on the reference's per-element operators
        if cls is B200Backend:
            from .generic import GenericB200Backend, needs_generic

            if needs_generic(ops):
                return super().__new__(GenericB200Backend)
        return super().__new__(cls)

    def __init__(self, ops, flow, opts, *, device=None, force_general: bool = False, device_metrics: bool = False,
                 variants: str = "auto"):
        import torch

        self.torch = torch
        self.ops, self.flow, self.opts = ops, flow, opts
        if opts.limiter not in ("positivity", "superbee", "none"):
            raise ValueError(f"unknown limiter {opts.limiter!r}")
        self.scheme = recommended_scheme(ops.ref.order) if opts.scheme is None else opts.scheme
        if self.scheme not in SCHEMES:
            raise ValueError(f"unknown scheme {self.scheme!r}; choose from {SCHEMES}")
        self.n_limited = 0
        self.n_mean_repaired = 0
        self.n_limit_calls = 0
        a_t = flow.stagnation_sound_speed
        self.component_weight = np.array([1.0, 1.0 / a_t, 1.0 / a_t, 1.0 / a_t**2]).reshape(1, 1, 4)

        self.lib = capi.load()
        # device_metrics: operators built without inverse mass matrices (lean) get their metric
        # terms from the node coordinates on the device
        self.mesh = DeviceMesh(ops, device, force_general=force_general, device_metrics=device_metrics)
        self.phys = physics_struct(flow, opts, ops.ref)
        self._phys_ref = capi.C.byref(self.phys)
        d = self.mesh.device
        E = self.mesh.E
        self._S = [self.mesh.state() for _ in range(3)]
        self._dt = torch.zeros(E, dtype=torch.float64, device=d)
        self._wave = torch.zeros(E, dtype=torch.float64, device=d)
        self._partial = torch.zeros(int(self.lib.nzb_norm_blocks(E)), dtype=torch.float64, device=d)
        self._res = torch.zeros(1, dtype=torch.float64, device=d)
        self._counters = torch.zeros(2, dtype=torch.int64, device=d)
        self._solvers: dict[str, int] = {}
        self._obs = None
        # fused or edge-pass face fluxes, fixed per element type
        # launch variants: the latency choice for a mesh that cannot fill the GPU, else the throughput one
        choose_variant(self.mesh, context_for(self.mesh.E, variants))

    def __del__(self):
        lib = getattr(self, "lib", None)
        for h in getattr(self, "_solvers", {}).values():
            if lib is not None and h:
                lib.nzb_solver_destroy(h)

    # -- helpers -------------------------------------------------------------
    @property
    def _stream(self):
        return self.mesh.stream()

    def _host(self, t) -> np.ndarray:
        return t.detach().to("cpu").numpy()

    def _limiter_on(self) -> bool:
        return self.opts.limiter != "none" and self.ops.ref.order > 0

    def _take_counters(self, calls: int) -> None:
        if not self._limiter_on():
            return
        c = self._host(self._counters)
        self._counters.zero_()
        self.n_limited += int(c[0])
        self.n_mean_repaired += int(c[1])
        self.n_limit_calls += calls

    def positivity_scale(self) -> float:
        pc = getattr(self.opts, "positivity_cfl", 0.0)
        if pc > 0.0 and self.opts.limiter != "none" and self.ops.ref.order > 0:
            return float(pc)
        return 1.0

    def limiter_activity(self) -> float:
        if self.n_limit_calls == 0:
            return float("nan")
        return self.n_limited / self.n_limit_calls

    def asarray(self, A):
        return np.asarray(A)

    def to_numpy(self, A) -> np.ndarray:
        return np.asarray(A)

    # -- primitives -----------------------------------------------------------
    def _eval(self, U, op):
        src = self.mesh.pack(U, self._S[0])
        out = self._S[1]
        capi.check(self.lib.nzb_residual(self.mesh.c_ref, self._phys_ref, op, src.data_ptr(), out.data_ptr(),
                                         self._wave.data_ptr(), self._stream), "nzb_residual")
        return self._host(self.mesh.unpack(out)), self._host(self._wave)

    def residual(self, U):
        """``(R, wave)`` with ``M dU/dt = -R`` (src/backends/base.py:118-120)."""
        return self._eval(U, 0)

    def rate(self, U):
        """``(-M^-1 R, wave)`` in one fused pass."""
        return self._eval(U, 1)

    def inverse_mass(self, R):
        src = self.mesh.pack(R, self._S[0])
        out = self._S[1]
        capi.check(self.lib.nzb_inverse_mass(self.mesh.c_ref, src.data_ptr(), out.data_ptr(), self._stream), "nzb_inverse_mass")
        return self._host(self.mesh.unpack(out))

    def limit(self, U):
        if not self._limiter_on():
            return np.asarray(U)
        st = self.mesh.pack(U, self._S[0])
        capi.check(self.lib.nzb_limit(self.mesh.c_ref, self._phys_ref, st.data_ptr(), self._counters.data_ptr(), None,
                                      self._stream), "nzb_limit")
        out = self._host(self.mesh.unpack(st))
        self._take_counters(1)
        return out

    def limit_flags(self, U):
        """Limit ``U`` and also return per-element flags (bit 0 scaled, bit 1 mean repaired)."""
        st = self.mesh.pack(U, self._S[0])
        flags = self.torch.zeros(self.mesh.E, dtype=self.torch.uint8, device=self.mesh.device)
        if self._limiter_on():
            capi.check(self.lib.nzb_limit(self.mesh.c_ref, self._phys_ref, st.data_ptr(), self._counters.data_ptr(),
                                          flags.data_ptr(), self._stream), "nzb_limit")
            self._take_counters(1)
        return self._host(self.mesh.unpack(st)), self._host(flags)

    def time_step(self, wave_sum):
        coef = step_coefficient(self.ops.ref.order, self.opts.cfl, self.scheme)
        dt = coef * 2.0 * np.asarray(self.ops.elem_area) / np.maximum(np.asarray(wave_sum), FLOOR)
        return self.positivity_scale() * dt[:, None, None]

    def norm(self, A) -> float:
        src = self.mesh.pack(A, self._S[0])
        w = np.ascontiguousarray(self.component_weight.reshape(-1))
        capi.check(self.lib.nzb_norm(src.data_ptr(), self.mesh.E, self.mesh.np_, w.ctypes.data, self._partial.data_ptr(),
                                     self._res.data_ptr(), self._stream), "nzb_norm")
        return float(self._host(self._res)[0])

    def initial_state(self, geometry, host: bool = True):
        """The quasi-1D initial state of this mesh (src/timestepping/initialize.py:41-102, the reference's
        ``initial_condition="quasi1d"``), projected on the device (``nzb_initial_state``) from the node
        coordinates, the nozzle ``geometry`` and this backend's flow: the reference-layout (E, NP, 4) host
        array, or with ``host=False`` the device (4, NP, E) state."""
        from .nozzle import quasi1d_table, wall_parameters

        S = self.mesh.initial_state(self.phys, wall_parameters(geometry)[None], [quasi1d_table(geometry, self.flow)],
                                    np.asarray(self.ops.node_coords, float), np.asarray(self.ops.topology.elem_nodes))
        return self._host(self.mesh.unpack(S)) if host else S

    def performance(self, U, geom=None) -> dict:
        """The performance() metrics of a state (src/post/postprocess.py:193-255), integrated on the
        device; ``geom`` adds the throat-normalised coefficients and the ideal thrust."""
        from .observables import DeviceObservables

        if self._obs is None:
            self._obs = DeviceObservables(self.mesh, self.phys, [(self.ops, 0, 0)], [self.flow])
        src = self.mesh.pack(U, self._S[0])
        return self._obs.performance(src, [geom])[0]

    # -- integrators (host composition of the primitives, src/backends/base.py:155-190)
    def euler_step(self, U):
        F0, wave = self.rate(U)
        dt = self.time_step(wave)
        res = self.norm(F0)
        return self.limit(U + dt * F0), res

    def ssprk3_step(self, U):
        F0, wave = self.rate(U)
        dt = self.time_step(wave)
        res = self.norm(F0)
        U1 = self.limit(U + dt * F0)
        F1, _ = self.rate(U1)
        U2 = self.limit(0.75 * U + 0.25 * (U1 + dt * F1))
        F2, _ = self.rate(U2)
        U3 = (1.0 / 3.0) * U + (2.0 / 3.0) * (U2 + dt * F2)
        return self.limit(U3), res

    def make_step(self, scheme: str):
        if scheme == "euler":
            return self.euler_step
        if scheme == "ssprk3":
            return self.ssprk3_step
        raise ValueError(f"unknown scheme {scheme!r}; choose from {SCHEMES}")

    def step_record(self, U, scheme: str | None = None):
        """One step through the fused stage kernels, stage by stage.

        Returns ``(U_new, residual, flags)`` with ``flags`` of shape
        ``(stages, E)``: bit 0 = the limiter scaled the element at that stage,
        bit 1 = its cell mean was repaired.  Same kernels as :meth:`run`.
        """
        torch = self.torch
        scheme = scheme or self.scheme
        S0, S1, S2 = self._S
        self.mesh.pack(U, S0)
        E = self.mesh.E
        n_st = 3 if scheme == "ssprk3" else 1
        flags = torch.zeros((n_st, E), dtype=torch.uint8, device=self.mesh.device)
        factor = self.positivity_scale() * step_coefficient(self.ops.ref.order, self.opts.cfl, self.scheme)
        plan = [(S0, None, S2 if n_st == 3 else S1, 1, 0.0, 1.0)]
        if n_st == 3:
            plan += [(S2, S0, S1, 2, 0.75, 0.25), (S1, S0, S0, 3, 1.0 / 3.0, 2.0 / 3.0)]
        for k, (V, U0, out, stage, a, b) in enumerate(plan):
            args = capi.StageArgs()
            args.V, args.out, args.dt = V.data_ptr(), out.data_ptr(), self._dt.data_ptr()
            args.U0 = U0.data_ptr() if U0 is not None else None
            args.norm_partial = self._partial.data_ptr() if stage == 1 else None
            args.counters = self._counters.data_ptr()
            args.flags = flags[k].data_ptr()
            args.dt_factor, args.a, args.b, args.stage = factor, a, b, stage
            capi.check(self.lib.nzb_stage(self.mesh.c_ref, self._phys_ref, capi.C.byref(args), self._stream), "nzb_stage")
            if stage == 1:
                nb = int(self.lib.nzb_element_blocks(self.mesh.c_ref))
                capi.check(self.lib.nzb_norm_finalize(self._partial.data_ptr(), nb, 4.0 * E * self.mesh.np_,
                                                      self._res.data_ptr(), self._stream), "nzb_norm_finalize")
        final = S0 if n_st == 3 else S1
        out = self._host(self.mesh.unpack(final))
        self._take_counters(n_st)
        return out, float(self._host(self._res)[0]), self._host(flags)

    # -- the fused march -------------------------------------------------------
    def _solver(self, scheme: str) -> int:
        if scheme in self._solvers:
            return self._solvers[scheme]
        buf = capi.Buffers()
        buf.S0, buf.S1, buf.S2 = (s.data_ptr() for s in self._S)
        buf.dt = self._dt.data_ptr()
        buf.norm_partial = self._partial.data_ptr()
        buf.res = self._res.data_ptr()
        buf.counters = self._counters.data_ptr()
        factor = self.positivity_scale() * step_coefficient(self.ops.ref.order, self.opts.cfl, self.scheme)
        h = capi.P()
        capi.check(self.lib.nzb_solver_create(self.mesh.c_ref, self._phys_ref, capi.C.byref(buf), 1 if scheme == "ssprk3" else 0,
                                              factor, capi.C.byref(h)), "nzb_solver_create")
        self._solvers[scheme] = h.value
        return h.value

    def run_device(self, n_steps: int, scheme: str | None = None) -> None:
        """Advance the device-resident state (``self._S[0]``) by ``n_steps``; no copies."""
        h = self._solver(scheme or self.scheme)
        capi.check(self.lib.nzb_solver_run(h, int(n_steps), self._stream), "nzb_solver_run")

    def run(self, U, n_steps: int, scheme: str):
        """Advance ``n_steps`` steps; returns a fresh ``(U, residual of the last step)``."""
        if scheme not in SCHEMES:
            raise ValueError(f"unknown scheme {scheme!r}; choose from {SCHEMES}")
        self.mesh.pack(U, self._S[0])
        self.run_device(n_steps, scheme)
        out = self._host(self.mesh.unpack(self._S[0]))
        res = float(self._host(self._res)[0])
        self._take_counters((3 if scheme == "ssprk3" else 1) * int(n_steps))
        return out, res
