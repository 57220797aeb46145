"""Host-side DG operators with the reference's attribute names.

:func:`build_operators` restates ``build_operators`` (src/spatial/operators.py:
209-342) in NumPy: per-element metrics, mass matrices and the M^-1-folded
operators, per-edge normals and jacobians, and the face gather map.  The object
it returns carries the same attribute names as the reference's ``Operators``
(src/spatial/operators.py:139-206), so the device packer in :mod:`.layout`
accepts either.

``lean=True`` skips the per-element operator arrays (``grad_*``, ``inv_mass``,
``face_basis*``), which cost ~7 GB at a million cubic triangles and which the
affine device path never reads: it carries the inverse Jacobian instead.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Any

import numpy as np

from . import refelem as re


@dataclass(frozen=True)
class Operators:
    ref: Any
    topology: Any
    node_coords: np.ndarray
    det_jac: np.ndarray
    weighted_det: np.ndarray
    grad_x: Any
    grad_y: Any
    inv_mass: Any
    grad_x_m: Any
    grad_y_m: Any
    face_basis_m: Any
    elem_area: np.ndarray
    mean_weights: np.ndarray
    xy_vol: Any
    edge_normal: np.ndarray
    edge_jac: np.ndarray
    edge_length: np.ndarray
    xy_face: Any
    face_edge: np.ndarray
    face_sign: np.ndarray
    face_basis: Any

    @property
    def n_elem(self) -> int:
        return int(self.topology.n_elem)

    @property
    def n_interior(self) -> int:
        return int(self.topology.edges.n_interior)

    @property
    def n_boundary(self) -> int:
        return int(self.topology.edges.n_boundary)

    @property
    def n_edges_total(self) -> int:
        return self.n_interior + self.n_boundary


def build_operators(topology, node_coords, order: int, *, lean: bool = False) -> Operators:
    rd = re.ref_tables(topology.kind, order, topology.geometry_order)
    X = np.asarray(node_coords, float)
    Xe = X[topology.elem_nodes]
    x_xi = Xe[:, :, 0] @ rd.dgeom_dxi_vol
    x_eta = Xe[:, :, 0] @ rd.dgeom_deta_vol
    y_xi = Xe[:, :, 1] @ rd.dgeom_dxi_vol
    y_eta = Xe[:, :, 1] @ rd.dgeom_deta_vol
    det = x_xi * y_eta - x_eta * y_xi
    if np.any(det <= 0.0):
        raise ValueError(f"{int(np.sum(det <= 0.0))} quadrature point(s) have a non-positive Jacobian")
    wdet = rd.w_vol[None, :] * det
    area = wdet.sum(axis=1)
    mean_w = np.einsum("iq,eq->ei", rd.phi_vol, wdet) / area[:, None]

    gx = gy = minv = gxm = gym = fbm = fb = xyv = None
    if not lean:
        inv = 1.0 / det
        xi_x, xi_y, eta_x, eta_y = y_eta * inv, -x_eta * inv, -y_xi * inv, x_xi * inv
        gx = wdet[:, None, :] * (rd.dphi_dxi_vol[None] * xi_x[:, None, :] + rd.dphi_deta_vol[None] * eta_x[:, None, :])
        gy = wdet[:, None, :] * (rd.dphi_dxi_vol[None] * xi_y[:, None, :] + rd.dphi_deta_vol[None] * eta_y[:, None, :])
        mass = np.einsum("iq,jq,eq->eij", rd.phi_vol, rd.phi_vol, wdet)
        minv = np.linalg.inv(mass)
        nface = topology.n_faces
        side = topology.edges.face_side
        fb = rd.phi_face[side, np.arange(nface)[None, :].repeat(topology.n_elem, axis=0)]
        gxm = np.einsum("eij,ejq->eiq", minv, gx)
        gym = np.einsum("eij,ejq->eiq", minv, gy)
        fbm = np.einsum("eij,efjq->efiq", minv, fb)
        xyv = np.einsum("nq,end->eqd", rd.geom_vol, Xe)

    ed = topology.edges
    own_e = np.concatenate([ed.iedge_elem[:, 0], ed.bedge_elem])
    own_f = np.concatenate([ed.iedge_face[:, 0], ed.bedge_face])
    Xo = Xe[own_e]
    tan = np.einsum("enq,end->eqd", rd.dgeom_dsigma_face[own_f], Xo)
    jac = np.sqrt(tan[..., 0] ** 2 + tan[..., 1] ** 2)
    normal = np.stack([tan[..., 1], -tan[..., 0]], axis=-1) / jac[..., None]
    length = (jac * rd.w_face[None, :]).sum(axis=1)
    xyf = np.einsum("enq,end->eqd", rd.geom_face[own_f], Xo)
    sign = np.where(ed.face_side == 0, 1.0, -1.0)
    return Operators(
        ref=rd,
        topology=topology,
        node_coords=X,
        det_jac=det,
        weighted_det=wdet,
        grad_x=gx,
        grad_y=gy,
        inv_mass=minv,
        grad_x_m=gxm,
        grad_y_m=gym,
        face_basis_m=fbm,
        elem_area=area,
        mean_weights=mean_w,
        xy_vol=xyv,
        edge_normal=normal,
        edge_jac=jac,
        edge_length=length,
        xy_face=xyf,
        face_edge=ed.face_edge,
        face_sign=sign,
        face_basis=fb,
    )


def affine_inverse_jacobian(ops) -> np.ndarray:
    """``(E, 5)``: ``xi_x, xi_y, eta_x, eta_y, det`` of straight-sided triangles.

    Taken at the first volume point; for a straight-sided triangle the
    geometry derivatives are the same at every point.
    """
    rd = ops.ref
    Xe = np.asarray(ops.node_coords)[ops.topology.elem_nodes]
    gxi, geta = rd.dgeom_dxi_vol[:, 0], rd.dgeom_deta_vol[:, 0]
    x_xi, x_eta = Xe[:, :, 0] @ gxi, Xe[:, :, 0] @ geta
    y_xi, y_eta = Xe[:, :, 1] @ gxi, Xe[:, :, 1] @ geta
    det = x_xi * y_eta - x_eta * y_xi
    inv = 1.0 / det
    return np.stack([y_eta * inv, -x_eta * inv, -y_xi * inv, x_xi * inv, det], axis=1)


def is_affine(ops) -> bool:
    """True for straight-sided triangles, where M = det * M_ref exactly."""
    return ops.ref.kind == "tri" and ops.topology.geometry_order == 1
