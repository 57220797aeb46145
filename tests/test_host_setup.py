"""Host-side setup (reference tables, mesh numbering, operators) against the reference's own arrays."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TINY, golden, pkg, tiny_ops


@pytest.mark.parametrize("kind,p", TINY)
def test_mesh_numbering_matches_the_reference(kind, p):
    g = golden(f"tiny_{kind}_p{p}.npz")
    topo, _, _ = pkg("mesh").channel_topology(kind, refine=0)
    assert np.array_equal(topo.elem_nodes, g["elem_nodes"])
    ed = topo.edges
    for name in ("face_edge", "face_side", "iedge_elem", "bedge_tag"):
        assert np.array_equal(getattr(ed, name), g[name]), name


@pytest.mark.parametrize("kind,p", TINY)
def test_operators_match_the_reference(kind, p):
    ops, g = tiny_ops(kind, p)
    for name in ("grad_x_m", "grad_y_m", "face_basis_m", "inv_mass", "edge_normal", "edge_jac", "edge_length",
                 "elem_area", "mean_weights"):
        a, b = np.asarray(getattr(ops, name)), g[name]
        assert a.shape == b.shape, name
        assert np.abs(a - b).max() <= 1e-14 * max(np.abs(b).max(), 1.0), name


def test_structured_rectangle_counts():
    topo, xf, rf = pkg("mesh").channel_topology("tri", nx=20, nr=10)
    assert topo.n_elem == 400
    ed = topo.edges
    assert ed.n_interior + ed.n_boundary == (3 * 400 + ed.n_boundary) // 2
    counts = {t: s.stop - s.start for t, s in ed.tag_slices.items()}
    assert counts == {1: 10, 2: 10, 3: 20, 4: 20}


@pytest.mark.parametrize("kind", ["tri", "quad"])
@pytest.mark.parametrize("p", [0, 1, 2, 3])
def test_edge_nodes_lie_on_their_edge(kind, p):
    re = pkg("refelem")
    nodes = re.lagrange_nodes(kind, p)
    for f in range(re.n_faces(kind)):
        ids = re.edge_node_ids(kind, p, f)
        assert len(ids) == p + 1
        if p == 0:
            continue
        (x0, y0), (dx, dy) = re.edge_start_and_direction(kind, f)
        for j, n in enumerate(ids):
            assert np.allclose(nodes[n], [x0 + j / p * dx, y0 + j / p * dy])


def test_affine_inverse_jacobian_inverts_the_map():
    ops, _ = tiny_ops("tri", 2)
    J = pkg("operators").affine_inverse_jacobian(ops)
    det = np.asarray(ops.det_jac)[:, 0]
    assert np.allclose(J[:, 4], det, rtol=1e-14)
    # grad_x / (w det) = dphi/dxi xi_x + dphi/deta eta_x at every point
    rd = ops.ref
    gx = rd.dphi_dxi_vol[None] * J[:, 0, None, None] + rd.dphi_deta_vol[None] * J[:, 2, None, None]
    ref = np.asarray(ops.grad_x) / (rd.w_vol[None, None, :] * det[:, None, None])
    assert np.abs(gx - ref).max() < 1e-10 * np.abs(ref).max()
