"""The reference's compiled CPU step restated in C (``cpu_step.c``) -- TEST INFRASTRUCTURE.

Only ``bench.py``'s CPU-baseline legs and the tests that check it against the
NumPy oracle use this; the product never loads it.  ``CpuStepper(ops, flow,
opts)`` takes the host operators (the reference's ``Operators`` attribute
names) and mirrors ``NumbaBackend`` (src/backends/numba_backend.py:48-337):
the same arrays in the reference layout, the same constants, and ``run(U, n,
scheme) -> (U_new, res)`` advancing ``n`` fused steps with the limiter after
every stage.  ``set_threads`` fixes the OpenMP thread count (the reference's
``numba.set_num_threads``).

``build()`` compiles the library with gcc (``-O3``, FMA contraction and
reassociation allowed, as the reference compiles with fastmath; OpenMP) into
``oracle/_lib``.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "cpu_step.c")
LIB = os.path.join(HERE, "_lib", "libcpu_step.so")
FLAGS = ["-O3", "-march=x86-64-v3", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=fast", "-fno-math-errno",
         "-fno-trapping-math", "-fno-signed-zeros", "-fassociative-math", "-freciprocal-math"]


def build(force: bool = False) -> str:
    if not force and os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    tmp = f"{LIB}.tmp{os.getpid()}"
    subprocess.run(["gcc", *FLAGS, SRC, "-o", tmp, "-lm"], check=True)
    os.replace(tmp, LIB)
    return LIB


P, I32, I64, D = C.c_void_p, C.c_int32, C.c_int64, C.c_double


class Case(C.Structure):
    _fields_ = [("n_elem", I64), ("n_int", I64), ("n_bnd", I64), ("nbf", I32), ("nqv", I32), ("nqf", I32),
                ("nface", I32)] + [(n, P) for n in (
                    "phi_vol", "phi_face", "w_face", "grad_x_m", "grad_y_m", "face_basis_m", "face_edge", "face_side",
                    "face_sign", "edge_normal", "edge_jac", "edge_length", "elem_area", "mean_weights", "iedge_elem",
                    "iedge_face", "bedge_elem", "bedge_face", "bedge_tag")] + [(n, D) for n in (
                        "gamma", "efix", "low_mach", "rho_t_bf", "p_t_bf", "band_bf", "at2", "at", "rho_t", "ca", "sa",
                        "p_back")] + [("flux_id", I32), ("limiter", I32)] + [(n, D) for n in (
                            "rho_floor", "p_floor", "fraction", "lebesgue")] + [("steps", I32), ("pad", I32),
                                                                               ("dt_factor", D), ("weight", D * 4)] + [
        (n, P) for n in ("fw", "smax", "wave", "dt", "F0", "F1", "F2", "S0", "S1", "S2")]


_LIB = None


def load():
    global _LIB
    if _LIB is None:
        lib = C.CDLL(build())
        lib.cpu_run.argtypes = [C.POINTER(Case), P, P, C.c_int, C.c_int, C.POINTER(D), C.POINTER(I64)]
        lib.cpu_run.restype = C.c_int
        lib.cpu_rate.argtypes = [C.POINTER(Case), P, P]
        lib.cpu_rate.restype = C.c_int
        lib.cpu_set_threads.argtypes = [C.c_int]
        lib.cpu_max_threads.restype = C.c_int
        _LIB = lib
    return _LIB


def set_threads(n: int) -> None:
    load().cpu_set_threads(int(n))


FLUX_IDS = {"roe": 0, "hllc": 1, "ausmup": 2}
SSPRK3_LIMITS = (1.437, 2.337, 2.240)
EULER_LIMITS = (1.169, 1.337, 0.775)


def step_coefficient(order: int, cfl, scheme: str) -> float:
    """cfl / (2p + 1), cfl defaulting to 0.7 x the measured stability limit (src/timestepping/step.py:123-168)."""
    if cfl is None:
        table = SSPRK3_LIMITS if scheme == "ssprk3" else EULER_LIMITS
        lim = table[order] if order < len(table) else (0.70 if scheme == "euler" else 1.32 * (2 * order + 1) / (order + 1))
        cfl = 0.7 * lim
    return cfl / (2 * order + 1)


class CpuStepper:
    def __init__(self, ops, flow, opts):
        if opts.limiter == "superbee":
            raise NotImplementedError("the C port runs the positivity limiter only")
        if flow.flux not in FLUX_IDS:
            raise NotImplementedError(f"flux {flow.flux!r}")
        lib = load()
        self.lib = lib
        ref, ed = ops.ref, ops.topology.edges
        self.order = int(ref.order)
        self.scheme = opts.scheme or ("euler" if self.order < 1 else "ssprk3")
        c64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64))  # noqa: E731
        i64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int64))  # noqa: E731
        keep = {
            "phi_vol": c64(ref.phi_vol), "phi_face": c64(ref.phi_face), "w_face": c64(ref.w_face),
            "grad_x_m": c64(ops.grad_x_m), "grad_y_m": c64(ops.grad_y_m), "face_basis_m": c64(ops.face_basis_m),
            "face_edge": i64(ed.face_edge), "face_side": i64(ed.face_side), "face_sign": c64(ops.face_sign),
            "edge_normal": c64(ops.edge_normal), "edge_jac": c64(ops.edge_jac), "edge_length": c64(ops.edge_length),
            "elem_area": c64(ops.elem_area), "mean_weights": c64(ops.mean_weights),
            "iedge_elem": i64(ed.iedge_elem), "iedge_face": i64(ed.iedge_face), "bedge_elem": i64(ed.bedge_elem),
            "bedge_face": i64(ed.bedge_face), "bedge_tag": i64(ed.bedge_tag),
        }
        E, nbf = int(ops.n_elem), int(ref.n_basis)
        nqv, nqf = int(np.asarray(ref.phi_vol).shape[1]), int(np.asarray(ref.w_face).shape[0])
        nface = int(np.asarray(ed.face_edge).shape[1])
        n_edge = int(ops.n_edges_total)
        work = {"fw": np.zeros(n_edge * nqf * 4), "smax": np.zeros(n_edge), "wave": np.zeros(E), "dt": np.zeros(E)}
        for k in ("F0", "F1", "F2", "S0", "S1", "S2"):
            work[k] = np.zeros(E * nbf * 4)
        self._keep = {**keep, **work}
        self.work = work
        c = Case()
        c.n_elem, c.n_int, c.n_bnd = E, int(ops.n_interior), int(ops.n_boundary)
        c.nbf, c.nqv, c.nqf, c.nface = nbf, nqv, nqf, nface
        for k, a in self._keep.items():
            setattr(c, k, a.ctypes.data)
        g = float(flow.gamma)
        c.gamma, c.efix, c.low_mach = g, float(flow.entropy_fix), float(getattr(flow, "hllc_low_mach", 0.0))
        c.rho_t_bf = float(flow.stagnation_density) if getattr(flow, "backflow", False) else 0.0
        c.p_t_bf, c.band_bf = float(flow.total_pressure), 0.05
        at = float(flow.stagnation_sound_speed)
        c.at, c.at2, c.rho_t = at, at * at, float(flow.stagnation_density)
        c.ca, c.sa = float(np.cos(flow.inflow_angle)), float(np.sin(flow.inflow_angle))
        c.p_back = float(flow.back_pressure)
        c.flux_id = FLUX_IDS[flow.flux]
        c.limiter = 1 if (opts.limiter == "positivity" and self.order > 0) else 0
        c.rho_floor, c.p_floor = 1e-8 * float(flow.stagnation_density), 1e-8 * float(flow.total_pressure)
        c.fraction, c.steps = 1e-8, 12
        phi_v, phi_f = np.asarray(ref.phi_vol), np.asarray(ref.phi_face)
        c.lebesgue = float(max(np.abs(phi_v).sum(axis=0).max(), np.abs(phi_f).sum(axis=2).max()))
        pc = getattr(opts, "positivity_cfl", 0.0)
        pscale = float(pc) if (pc > 0.0 and opts.limiter != "none" and self.order > 0) else 1.0
        c.dt_factor = pscale * step_coefficient(self.order, opts.cfl, self.scheme)
        for s, w in enumerate((1.0, 1.0 / at, 1.0 / at, 1.0 / at**2)):
            c.weight[s] = w
        self.c = c
        self.shape = (E, nbf, 4)
        self.counters = np.zeros(2, np.int64)

    def run(self, U, n_steps: int, scheme: str | None = None):
        """Advance ``n_steps`` steps from ``U`` (E, NP, 4); returns a fresh array and the last step's residual."""
        scheme = scheme or self.scheme
        U = np.ascontiguousarray(np.asarray(U, dtype=np.float64))
        if U.shape != self.shape:
            raise ValueError(f"U has shape {U.shape}, expected {self.shape}")
        out = np.empty_like(U)
        res = D(0.0)
        cnt = (I64 * 2)(0, 0)
        rc = self.lib.cpu_run(C.byref(self.c), U.ctypes.data, out.ctypes.data, int(n_steps),
                              1 if scheme == "ssprk3" else 0, C.byref(res), cnt)
        if rc != 0:
            raise RuntimeError(f"cpu_run returned {rc}")
        self.counters += np.array([cnt[0], cnt[1]])
        return out, float(res.value)

    def rate(self, U):
        """``(-M^-1 R, wave)`` of ``U``."""
        U = np.ascontiguousarray(np.asarray(U, dtype=np.float64))
        out = np.empty_like(U)
        if self.lib.cpu_rate(C.byref(self.c), U.ctypes.data, out.ctypes.data) != 0:
            raise RuntimeError("cpu_rate failed")
        return out, self.work["wave"].copy()
