"""The flattened index arithmetic of the generic path's device operator build (csrc/gen_geometry.cuh),
restated in NumPy on the CPU: the same element loop, the same flat offsets into the reference-layout
outputs, the same in-place Gauss-Jordan inverse.  Against the host build (the reference's operators, bit
for bit), every array agrees to round-off, so a layout slip in the kernel's offsets would show here
before the GPU runs it."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import rel
from test_oracle_generic import generic_ops


def _build(ops):
    r, topo, ed = ops.ref, ops.topology, ops.topology.edges
    X = np.asarray(ops.node_coords, float).ravel()
    en = np.asarray(topo.elem_nodes).astype(np.int64).ravel()
    NG = np.asarray(topo.elem_nodes).shape[1]
    E, NP = ops.n_elem, r.n_basis
    NQV, NQF, NF = np.asarray(r.phi_vol).shape[1], np.asarray(r.w_face).size, np.asarray(ed.face_edge).shape[1]
    dgx, dge = np.asarray(r.dgeom_dxi_vol).ravel(), np.asarray(r.dgeom_deta_vol).ravel()
    dpx, dpe = np.asarray(r.dphi_dxi_vol).ravel(), np.asarray(r.dphi_deta_vol).ravel()
    phi, w = np.asarray(r.phi_vol).ravel(), np.asarray(r.w_vol).ravel()
    pf, wf = np.asarray(r.phi_face).ravel(), np.asarray(r.w_face).ravel()
    side = np.asarray(ed.face_side).astype(np.int64).ravel()
    dgs = np.asarray(r.dgeom_dsigma_face).ravel()
    out = {k: np.zeros(n) for k, n in (("grad_x", E * NP * NQV), ("grad_y", E * NP * NQV), ("grad_x_m", E * NP * NQV),
                                       ("grad_y_m", E * NP * NQV), ("face_basis_m", E * NF * NP * NQF),
                                       ("inv_mass", E * NP * NP), ("elem_area", E), ("mean_weights", E * NP))}
    k_idx, q_idx = np.arange(NP * NQV), np.arange(NP * NQV) % NQV
    for e in range(E):
        nodes = en[e * NG:(e + 1) * NG]
        xg, yg = X[2 * nodes], X[2 * nodes + 1]
        x_xi = xg @ dgx.reshape(NG, NQV)
        x_eta = xg @ dge.reshape(NG, NQV)
        y_xi = yg @ dgx.reshape(NG, NQV)
        y_eta = yg @ dge.reshape(NG, NQV)
        det = x_xi * y_eta - x_eta * y_xi
        met = np.concatenate([y_eta / det, -x_eta / det, -y_xi / det, x_xi / det, w * det])
        wdet = met[4 * NQV:]
        area = wdet.sum()
        out["elem_area"][e] = area
        out["mean_weights"][e * NP:(e + 1) * NP] = phi.reshape(NP, NQV) @ wdet / area
        gx = wdet[q_idx] * (dpx[k_idx] * met[q_idx] + dpe[k_idx] * met[2 * NQV + q_idx])
        gy = wdet[q_idx] * (dpx[k_idx] * met[NQV + q_idx] + dpe[k_idx] * met[3 * NQV + q_idx])
        gb = e * NP * NQV
        out["grad_x"][gb:gb + NP * NQV], out["grad_y"][gb:gb + NP * NQV] = gx, gy
        P = phi.reshape(NP, NQV)
        M = ((P * wdet) @ P.T).ravel()
        for p in range(NP):  # the kernel's Gauss-Jordan, step by step
            piv = 1.0 / M[p * NP + p]
            col = M[np.arange(NP) * NP + p].copy()
            row = M[p * NP:(p + 1) * NP].copy()
            row[p] = 1.0
            M[p * NP:(p + 1) * NP] = row * piv
            for i in range(NP):
                if i != p:
                    cur = M[i * NP:(i + 1) * NP].copy()
                    cur[p] = 0.0
                    M[i * NP:(i + 1) * NP] = cur - col[i] * M[p * NP:(p + 1) * NP]
        out["inv_mass"][e * NP * NP:(e + 1) * NP * NP] = M
        Mi = M.reshape(NP, NP)
        out["grad_x_m"][gb:gb + NP * NQV] = (Mi @ gx.reshape(NP, NQV)).ravel()
        out["grad_y_m"][gb:gb + NP * NQV] = (Mi @ gy.reshape(NP, NQV)).ravel()
        fb = e * NF * NP * NQF
        for k in range(NF * NP * NQF):
            f, i, q = k // (NP * NQF), (k // NQF) % NP, k % NQF
            s = side[e * NF + f]
            out["face_basis_m"][fb + k] = Mi[i] @ pf[((s * NF + f) * NP + np.arange(NP)) * NQF + q]
    ee = np.concatenate([np.asarray(ed.iedge_elem).reshape(-1, 2), np.stack([ed.bedge_elem, ed.bedge_elem], 1)]).ravel()
    ef = np.concatenate([np.asarray(ed.iedge_face).reshape(-1, 2), np.stack([ed.bedge_face, ed.bedge_face], 1)]).ravel()
    NK = ee.size // 2
    nrm, jacs, lens = np.zeros(NK * NQF * 2), np.zeros(NK * NQF), np.zeros(NK)
    for k in range(NK):
        e, f = ee[2 * k], ef[2 * k]
        nodes = en[e * NG:(e + 1) * NG]
        for q in range(NQF):
            d = dgs[(f * NG + np.arange(NG)) * NQF + q]
            tx, ty = d @ X[2 * nodes], d @ X[2 * nodes + 1]
            jac = np.sqrt(tx * tx + ty * ty)
            nrm[(k * NQF + q) * 2:(k * NQF + q) * 2 + 2] = ty / jac, -tx / jac
            jacs[k * NQF + q] = jac
            lens[k] += jac * wf[q]
    out.update(edge_normal=nrm, edge_jac=jacs, edge_length=lens)
    return out


@pytest.mark.parametrize("kind,p,q", [("tri", 2, 2), ("quad", 2, 2), ("tri", 4, 1)])
def test_device_build_layout_restated(kind, p, q):
    ops, _ = generic_ops(kind, p, q)
    got = _build(ops)
    for name, v in got.items():
        assert rel(v, np.asarray(getattr(ops, name)).ravel()) < 1e-13, name
