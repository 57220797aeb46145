"""ctypes binding of ``include/nozzle_b200.h``.

The library is loaded from the package's ``_lib`` directory (built by
:mod:`.build`).  A missing or unloadable library raises immediately: there is
no CPU fallback anywhere in this package.
"""

from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# NZB_LIBRARY names another build of the same library (e.g. one compiled with
# different launch bounds); by default the in-tree build is loaded.
LIB_PATH = os.environ.get("NZB_LIBRARY") or os.path.join(_HERE, "_lib", "libnozzle_b200.so")

P = C.c_void_p
I64 = C.c_int64
I32 = C.c_int32


class Mesh(C.Structure):
    _fields_ = [
        ("kind", I32),
        ("order", I32),
        ("affine", I32),
        ("edge_pass", I32),
        ("n_elem", I64),
        ("n_edge", I64),
        ("geo", P),
        ("minv", P),
        ("area", P),
        ("face_nbr", P),
        ("face_code", P),
        ("face_edge", P),
        ("edge_geo", P),
        ("elem_inst", P),
        ("inst_status", P),
        ("inst_p_back", P),
        ("edge_conn", P),
        ("edge_flux", P),
        ("edge_speed", P),
        ("elem_share", P),
        ("lim_means", P),
        ("lim_scale", P),
        ("split", I32),
        ("n_inst", I32),
        ("vjp_split", I32),
        ("reserved", I32),
        ("fwd_blocks", P),
        ("n_fwd_blocks", I64),
        ("vjp_blocks", P),
        ("n_vjp_blocks", I64),
    ]


class Physics(C.Structure):
    _fields_ = [
        ("gamma", C.c_double),
        ("entropy_fix", C.c_double),
        ("hllc_low_mach", C.c_double),
        ("flux", I32),
        ("limiter", I32),
        ("in_cos", C.c_double),
        ("in_sin", C.c_double),
        ("in_at2", C.c_double),
        ("in_at", C.c_double),
        ("in_rho_t", C.c_double),
        ("p_back", C.c_double),
        ("bf_rho_t", C.c_double),
        ("bf_p_t", C.c_double),
        ("bf_band", C.c_double),
        ("lim_fraction", C.c_double),
        ("rho_floor", C.c_double),
        ("p_floor", C.c_double),
        ("lebesgue", C.c_double),
        ("lim_steps", I32),
        ("reserved", I32),
        ("norm_w", C.c_double * 4),
        ("tvb_constant", C.c_double),
    ]


class StageArgs(C.Structure):
    _fields_ = [
        ("V", P),
        ("U0", P),
        ("out", P),
        ("dt", P),
        ("norm_partial", P),
        ("elem_norm", P),
        ("counters", P),
        ("flags", P),
        ("dt_factor", C.c_double),
        ("a", C.c_double),
        ("b", C.c_double),
        ("stage", I32),
        ("reserved", I32),
    ]


class Buffers(C.Structure):
    _fields_ = [
        ("S0", P),
        ("S1", P),
        ("S2", P),
        ("dt", P),
        ("norm_partial", P),
        ("res", P),
        ("counters", P),
    ]


class BatchMarch(C.Structure):
    _fields_ = [
        ("n_inst", I64),
        ("inst_begin", P),
        ("inst_end", P),
        ("inst_count", P),
        ("inst_tol", P),
        ("elem_norm", P),
        ("status", P),
        ("iterations", P),
        ("res0", P),
        ("res", P),
        ("window", P),
        ("window_count", P),
        ("n_running", P),
        ("divergence_factor", C.c_double),
        ("stall_ratio", C.c_double),
        ("stall_window", I32),
        ("max_iterations", I32),
    ]


class AdjointArgs(C.Structure):
    _fields_ = [
        ("mode", I32),
        ("stage", I32),
        ("U", P),
        ("lam", P),
        ("seed", P),
        ("out", P),
        ("lam0", P),
        ("dt", P),
        ("f0", P),
        ("f1", P),
        ("f2", P),
        ("norm_partial", P),
        ("elem_norm", P),
    ]


class AdjointBuffers(C.Structure):
    _fields_ = [
        ("U", P),
        ("seed", P),
        ("lam", P),
        ("Y1", P),
        ("Y2", P),
        ("f0", P),
        ("f1", P),
        ("f2", P),
        ("dt", P),
    ]


class AdjointMarch(C.Structure):
    _fields_ = [
        ("n_inst", I64),
        ("inst_begin", P),
        ("inst_end", P),
        ("inst_count", P),
        ("elem_norm", P),
        ("status", P),
        ("iterations", P),
        ("res0", P),
        ("res", P),
        ("n_running", P),
        ("tolerance", C.c_double),
        ("max_iterations", I32),
        ("reserved", I32),
    ]


ADJ_VJP, ADJ_DEFECT, ADJ_RATE, ADJ_RK4 = 0, 1, 2, 3


class ObsArgs(C.Structure):
    _fields_ = [
        ("U", P),
        ("n_seg", I32),
        ("reserved", I32),
        ("bedges", P),
        ("bseg", P),
        ("eseg", P),
        ("r_gas", C.c_double),
        ("s_t", C.c_double),
        ("out", P),
    ]


class GeometryArgs(C.Structure):
    _fields_ = [
        ("X", P),
        ("elem_nodes", P),
        ("edge_conn", P),
        ("dgs", C.c_double * 16),
        ("geo", P),
        ("minv", P),
        ("area", P),
        ("edge_geo", P),
    ]


class GenMesh(C.Structure):
    _fields_ = [("np", I32), ("nqv", I32), ("nqf", I32), ("nface", I32), ("n_elem", I64), ("n_int", I64),
                ("n_bnd", I64)] + [(n, P) for n in (
                    "phi_vol", "phi_face", "w_face", "grad_x", "grad_y", "grad_x_m", "grad_y_m", "face_basis_m",
                    "face_edge", "face_side", "face_sign", "edge_elem", "edge_face", "edge_tag", "edge_normal",
                    "edge_jac", "edge_length", "elem_area", "mean_weights")]


class GenGeometryArgs(C.Structure):
    _fields_ = [("ng", I32), ("reserved", I32)] + [
        (n, P) for n in ("X", "elem_nodes", "w_vol", "dphi_dxi", "dphi_deta", "dgeom_dxi", "dgeom_deta", "dgeom_dsigma",
                         "grad_x", "grad_y", "grad_x_m", "grad_y_m", "face_basis_m", "inv_mass", "elem_area",
                         "mean_weights", "edge_normal", "edge_jac", "edge_length", "bad")]


class GenInitialArgs(C.Structure):
    _fields_ = [("ng", I32), ("reserved", I32)] + [
        (n, P) for n in ("X", "elem_nodes", "geom_vol", "dgeom_dxi", "dgeom_deta", "w_vol", "inv_mass", "wall", "q1d")] + [
        ("n_q1d", I64), ("out", P)]


class GenObsArgs(C.Structure):
    _fields_ = [("ng", I32), ("reserved", I32)] + [
        (n, P) for n in ("X", "elem_nodes", "dgeom_dxi", "dgeom_deta", "w_vol", "U")] + [
        ("s_t", C.c_double), ("r_gas", C.c_double), ("out", P)]


class GenUpdateArgs(C.Structure):
    _fields_ = [("stage", I32), ("pad", I32), ("dt_factor", C.c_double), ("a", C.c_double), ("b", C.c_double)] + [
        (n, P) for n in ("V", "U0", "F", "wave", "dt", "out", "partial")]


NZB_WALL_PARAMS = 20


class InitialArgs(C.Structure):
    _fields_ = [
        ("verts", P),
        ("wall", P),
        ("q1d", P),
        ("q1d_begin", P),
        ("out", P),
    ]


# column of each per-instance sum of nzb_observables
(OBS_MOM_OUT, OBS_MOM_IN, OBS_WALL_PX, OBS_MASS_IN, OBS_MASS_OUT, OBS_EXIT_LEN, OBS_EXIT_MACH, OBS_EXIT_P,
 OBS_EXIT_T, OBS_ENTROPY, OBS_AREA) = range(11)
NOBS = 11

# (name, restype, argtypes) of every exported symbol
SIGNATURES = [
    ("nzb_version", C.c_int, []),
    ("nzb_last_error", C.c_char_p, []),
    ("nzb_table_size", I64, [C.c_int, C.c_int]),
    ("nzb_upload_tables", C.c_int, [C.c_int, C.c_int, P, I64]),
    ("nzb_pack_state", C.c_int, [P, P, I64, C.c_int, P, P]),
    ("nzb_unpack_state", C.c_int, [P, P, I64, C.c_int, P, P]),
    ("nzb_residual", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), C.c_int, P, P, P, P]),
    ("nzb_inverse_mass", C.c_int, [C.POINTER(Mesh), P, P, P]),
    ("nzb_observables", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(ObsArgs), P]),
    ("nzb_geometry", C.c_int, [C.POINTER(Mesh), C.POINTER(GeometryArgs), P]),
    ("nzb_initial_state", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(InitialArgs), P]),
    ("nzb_gen_rate", C.c_int, [C.POINTER(GenMesh), C.POINTER(Physics), C.c_int, P, P, P, P, P, P]),
    ("nzb_gen_limit", C.c_int, [C.POINTER(GenMesh), C.POINTER(Physics), P, P, P]),
    ("nzb_gen_update", C.c_int, [C.POINTER(GenMesh), C.POINTER(Physics), C.POINTER(GenUpdateArgs), P]),
    ("nzb_gen_blocks", I64, [C.POINTER(GenMesh)]),
    ("nzb_gen_geometry", C.c_int, [C.POINTER(GenMesh), C.POINTER(GenGeometryArgs), P]),
    ("nzb_gen_superbee", C.c_int, [C.POINTER(GenMesh), C.POINTER(Physics), P, P, P, P, P, P]),
    ("nzb_gen_initial_state", C.c_int, [C.POINTER(GenMesh), C.POINTER(Physics), C.POINTER(GenInitialArgs), P]),
    ("nzb_gen_observables", C.c_int, [C.POINTER(GenMesh), C.POINTER(Physics), C.POINTER(GenObsArgs), P]),
    ("nzb_limit", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), P, P, P, P]),
    ("nzb_stage", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(StageArgs), P]),
    ("nzb_norm_blocks", I64, [I64]),
    ("nzb_element_blocks", I64, [C.POINTER(Mesh)]),
    ("nzb_block_width", I64, [C.POINTER(Mesh), I32]),
    ("nzb_norm_finalize", C.c_int, [P, I64, C.c_double, P, P]),
    ("nzb_norm", C.c_int, [P, I64, C.c_int, P, P, P, P]),
    ("nzb_norm_noalloc", C.c_int, [P, I64, C.c_int, P, P, P]),
    ("nzb_solver_create", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(Buffers), C.c_int, C.c_double, C.POINTER(P)]),
    ("nzb_solver_run", C.c_int, [P, C.c_int, P]),
    ("nzb_solver_destroy", C.c_int, [P]),
    ("nzb_batch_create", C.c_int, [C.c_int, C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(Buffers), P, P,
                                   C.POINTER(BatchMarch), C.POINTER(P)]),
    ("nzb_batch_run", C.c_int, [P, C.c_int, C.c_int, P]),
    ("nzb_batch_destroy", C.c_int, [P]),
    ("nzb_vjp", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(AdjointArgs), P]),
    ("nzb_vjp_coords", C.c_int, [C.POINTER(Mesh), C.POINTER(Physics), P, P, P, P, P, P, P]),
    ("nzb_local_dt", C.c_int, [C.POINTER(Mesh), P, C.c_double, P, P]),
    ("nzb_adjoint_create", C.c_int, [C.c_int, C.POINTER(Mesh), C.POINTER(Physics), C.POINTER(AdjointBuffers), P,
                                     C.POINTER(AdjointMarch), C.POINTER(P)]),
    ("nzb_adjoint_run", C.c_int, [P, C.c_int, P]),
    ("nzb_adjoint_destroy", C.c_int, [P]),
]

_lib = None


class NativeError(RuntimeError):
    pass


def load(path: str = LIB_PATH):
    """Load the library once and declare every signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise NativeError(
            f"{path} is missing; build it with `python 2d_nozzle_b200/build.py` (nvcc, sm_100a). "
            "This backend has no CPU fallback."
        )
    lib = C.CDLL(path)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int, what: str) -> None:
    if rc != 0:
        msg = _lib.nzb_last_error().decode(errors="replace") if _lib is not None else "library not loaded"
        raise NativeError(f"{what} failed ({rc}): {msg}")
