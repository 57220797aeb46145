"""Device layout: reference-element tables and the per-mesh arrays the kernels read.

:func:`element_tables` flattens one (kind, order) slot of the constant-memory
table in the order ``csrc/shapes.cuh`` declares.  :class:`DeviceMesh` turns an
``Operators``-like object (the reference's, or :mod:`.operators`') into
structure-of-arrays device tensors and the ``nzb_mesh`` descriptor.

Two geometry layouts:

* affine -- straight-sided triangles: ``(5, E)`` = xi_x, xi_y, eta_x, eta_y,
  det per element (40 B), the volume and mass operators coming from the
  constant tables because ``M_e = det_e M_ref`` exactly;
* general -- any element (bilinear quadrilaterals): the reference's
  per-element weighted gradients ``grad_x``, ``grad_y`` and inverse mass
  matrices, stored index-major / element-minor so a warp reads them coalesced.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import capi
from . import refelem as re
from .config import FLUX_IDS, component_weights
from .operators import affine_inverse_jacobian, is_affine

KIND_IDS = {"tri": 0, "quad": 1}
MAX_ORDER = 3


def element_tables(ref) -> np.ndarray:
    """The constant-memory slot of one reference element (see csrc/shapes.cuh)."""
    kind, p = ref.kind, ref.order
    w = np.asarray(ref.w_vol)
    phi = np.asarray(ref.phi_vol)
    wxi = np.asarray(ref.dphi_dxi_vol) * w[None, :]
    weta = np.asarray(ref.dphi_deta_vol) * w[None, :]
    mref = np.einsum("iq,jq,q->ij", phi, phi, w)
    minv = np.linalg.inv(mref)
    f0 = 2 if kind == "tri" else 0  # the edge along eta = 0, walked in +xi
    nodes = re.edge_node_ids(kind, p, f0)
    e1d = np.asarray(ref.phi_face)[0, f0][nodes, :]
    wf = np.asarray(ref.w_face)
    mw = (phi @ w) / w.sum()
    pf = np.asarray(ref.phi_face)  # (2, NF, NP, NQF)
    return np.ascontiguousarray(np.concatenate([phi.ravel(), wxi.ravel(), weta.ravel(), minv.ravel(), e1d.ravel(), wf, mw,
                                                pf.ravel()]))


def lebesgue_constant(ref) -> float:
    """max over probe points of sum_i |phi_i|: bounds every probe by the coefficients."""
    return float(max(np.abs(ref.phi_vol).sum(axis=0).max(), np.abs(ref.phi_face).sum(axis=2).max()))


_uploaded: set[tuple[int, int, int]] = set()


def ensure_tables(ref, device_index: int) -> None:
    lib = capi.load()
    key = (device_index, KIND_IDS[ref.kind], ref.order)
    if key in _uploaded:
        return
    tab = element_tables(ref)
    n = lib.nzb_table_size(key[1], key[2])
    if n != tab.size:
        raise capi.NativeError(f"table size {tab.size} does not match the library's {n} for {ref.kind} p={ref.order}")
    capi.check(lib.nzb_upload_tables(key[1], key[2], tab.ctypes.data, tab.size), "nzb_upload_tables")
    _uploaded.add(key)


def physics_struct(flow, opts, ref) -> capi.Physics:
    """Constants evaluated exactly as the reference evaluates them."""
    if flow.flux not in FLUX_IDS:
        raise NotImplementedError(f"the device kernels implement {sorted(FLUX_IDS)}, not flux={flow.flux!r}")
    g = float(flow.gamma)
    ph = capi.Physics()
    ph.gamma = g
    ph.entropy_fix = float(flow.entropy_fix)
    ph.hllc_low_mach = float(getattr(flow, "hllc_low_mach", 0.0))
    ph.flux = FLUX_IDS[flow.flux]
    ph.limiter = 1 if (opts.limiter == "positivity" and ref.order > 0) else 0
    at2 = g * float(flow.Rgas) * float(flow.total_temperature)
    ph.in_cos = float(np.cos(flow.inflow_angle))
    ph.in_sin = float(np.sin(flow.inflow_angle))
    ph.in_at2 = at2
    ph.in_at = float(np.sqrt(at2))
    ph.in_rho_t = g * float(flow.total_pressure) / at2
    ph.p_back = float(flow.back_pressure)
    ph.bf_rho_t = float(flow.stagnation_density) if getattr(flow, "backflow", False) else 0.0
    ph.bf_p_t = float(flow.total_pressure)
    ph.bf_band = 0.05
    ph.lim_fraction = 1e-8
    ph.rho_floor = 1e-8 * float(flow.stagnation_density)
    ph.p_floor = 1e-8 * float(flow.total_pressure)
    ph.lebesgue = lebesgue_constant(ref)
    ph.lim_steps = 12
    for s, v in enumerate(component_weights(flow)):
        ph.norm_w[s] = v
    return ph


class DeviceMesh:
    """Device-resident geometry and connectivity of one mesh."""

    def __init__(self, ops, device=None, *, force_general: bool = False):
        import torch

        self.torch = torch
        self.device = torch.device(device if device is not None else "cuda")
        if self.device.type != "cuda":
            raise capi.NativeError("the B200 backend runs on a CUDA device only")
        ref = ops.ref
        if ref.kind not in KIND_IDS or not 0 <= ref.order <= MAX_ORDER:
            raise NotImplementedError(f"device kernels cover tri/quad p=0..{MAX_ORDER}, not {ref.kind} p={ref.order}")
        topo = ops.topology
        if topo.geometry_order != 1:
            raise NotImplementedError("device kernels take straight-sided (Q=1) elements")
        self.ref = ref
        self.kind, self.order = ref.kind, int(ref.order)
        self.np_ = int(ref.n_basis)
        self.nf = re.n_faces(ref.kind)
        self.E = int(ops.n_elem)
        self.affine = is_affine(ops) and not force_general
        idx = self.device.index if self.device.index is not None else torch.cuda.current_device()
        ensure_tables(ref, idx)

        def dev(a, dtype=torch.float64):
            return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device=self.device)

        E = self.E
        keep = {}
        if self.affine:
            keep["geo"] = dev(affine_inverse_jacobian(ops).T)
        else:
            if getattr(ops, "grad_x", None) is None:
                raise ValueError("general geometry needs the per-element operators (build_operators(..., lean=False))")
            keep["gx"] = dev(np.asarray(ops.grad_x).reshape(E, -1).T)
            keep["gy"] = dev(np.asarray(ops.grad_y).reshape(E, -1).T)
            keep["minv"] = dev(np.asarray(ops.inv_mass).reshape(E, -1).T)
            keep["mean_w"] = dev(np.asarray(ops.mean_weights).T)
        keep["area"] = dev(np.asarray(ops.elem_area))

        ed = topo.edges
        ni = ed.n_interior
        fe = np.asarray(ed.face_edge)
        side = np.asarray(ed.face_side)
        interior = fe < ni
        ke = np.where(interior, fe, 0)
        other = np.where(side == 0, 1, 0)
        nbr = np.where(interior, np.asarray(ed.iedge_elem)[ke, other], -1)
        nbr_face = np.where(interior, np.asarray(ed.iedge_face)[ke, other], 0)
        tag = np.where(interior, 0, np.asarray(ed.bedge_tag)[np.where(interior, 0, fe - ni)])
        code = side | (nbr_face << 1) | (tag << 4)
        keep["face_nbr"] = dev(nbr.T, torch.int32)
        keep["face_code"] = dev(code.T, torch.int32)
        keep["face_edge"] = dev(fe.T, torch.int32)

        nrm = np.asarray(ops.edge_normal)
        jac = np.asarray(ops.edge_jac)
        if np.abs(nrm - nrm[:, :1]).max() > 0.0 or np.abs(jac - jac[:, :1]).max() > 0.0:
            raise NotImplementedError("device kernels take straight edges (one normal per edge)")
        egeo = np.stack([nrm[:, 0, 0], nrm[:, 0, 1], jac[:, 0], np.asarray(ops.edge_length)], axis=1)
        keep["edge_geo"] = dev(egeo)
        self.n_edge = int(egeo.shape[0])
        self.arrays = keep

        m = capi.Mesh()
        m.kind = KIND_IDS[self.kind]
        m.order = self.order
        m.affine = 1 if self.affine else 0
        m.n_elem = E
        m.n_edge = self.n_edge
        for name in ("geo", "gx", "gy", "minv", "mean_w", "area", "face_nbr", "face_code", "face_edge", "edge_geo"):
            setattr(m, name, keep[name].data_ptr() if name in keep else None)
        self.c = m
        self.c_ref = C.byref(m)

    def state(self) -> object:
        """An uninitialised (4, NP, E) device state."""
        return self.torch.empty(4 * self.np_ * self.E, dtype=self.torch.float64, device=self.device)

    def stream(self) -> int:
        return self.torch.cuda.current_stream(self.device).cuda_stream

    def pack(self, U_host_or_dev, out=None):
        """(E, NP, 4) array (host or device) -> (4, NP, E) device state."""
        torch = self.torch
        src = torch.as_tensor(np.ascontiguousarray(U_host_or_dev) if isinstance(U_host_or_dev, np.ndarray) else U_host_or_dev,
                              dtype=torch.float64, device=self.device).contiguous()
        if tuple(src.shape) != (self.E, self.np_, 4):
            raise ValueError(f"state has shape {tuple(src.shape)}, expected {(self.E, self.np_, 4)}")
        dst = self.state() if out is None else out
        capi.check(capi.load().nzb_pack_state(src.data_ptr(), dst.data_ptr(), self.E, self.np_, None, self.stream()), "nzb_pack_state")
        return dst

    def unpack(self, soa):
        """(4, NP, E) device state -> (E, NP, 4) device tensor."""
        out = self.torch.empty((self.E, self.np_, 4), dtype=self.torch.float64, device=self.device)
        capi.check(capi.load().nzb_unpack_state(soa.data_ptr(), out.data_ptr(), self.E, self.np_, None, self.stream()), "nzb_unpack_state")
        return out

