"""Device-built metric terms (nzb_geometry) against the host build of the same node coordinates."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TINY, pkg, rel, tiny_ops

pytestmark = pytest.mark.gpu


def perturbed(ops, seed=0, amount=0.05):
    """Node coordinates with every node moved by a small random fraction of the mesh spacing."""
    X = np.asarray(ops.node_coords, float).copy()
    h = float(np.sqrt(np.asarray(ops.elem_area).min()))
    X += np.random.default_rng(seed).uniform(-amount * h, amount * h, X.shape)
    return X


def compare(dm, host):
    arrays = {k: dm.arrays[k].cpu().numpy() for k in ("geo", "area", "edge_geo")}
    assert rel(arrays["geo"], host["geo"]) < 1e-13
    assert rel(arrays["area"], host["area"]) < 1e-13
    assert rel(arrays["edge_geo"], host["edge_geo"]) < 1e-13
    if "minv" in host:
        assert rel(dm.arrays["minv"].cpu().numpy(), host["minv"]) < 1e-11


@pytest.mark.parametrize("kind,p", TINY)
def test_device_geometry_matches_the_host_build(cuda, kind, p):
    lay, opm = pkg("layout"), pkg("operators")
    ops, g = tiny_ops(kind, p)
    for general in ((False, True) if kind == "tri" else (False,)):
        for X in (np.asarray(ops.node_coords, float), perturbed(ops)):
            ops_x = opm.build_operators(ops.topology, X, p)
            host = lay.host_arrays(ops_x, force_general=general)
            dm = lay.DeviceMesh(ops, force_general=general)  # built at the base coordinates
            dm.set_geometry(X, np.asarray(ops.topology.elem_nodes)[:, :dm.nf])
            compare(dm, host)


@pytest.mark.parametrize("kind,p", [("tri", 2), ("quad", 3)])
def test_residual_on_a_device_built_mesh(cuda, kind, p):
    """The residual at moved coordinates: device-built metrics vs a host-built mesh."""
    cfg, opm = pkg("config"), pkg("operators")
    ops, g = tiny_ops(kind, p)
    X = perturbed(ops, seed=3)
    flow, opts = cfg.FlowConditions(flux="hllc"), cfg.SolverOptions()
    ref = pkg("backend").B200Backend(opm.build_operators(ops.topology, X, p), flow, opts)
    bk = pkg("backend").B200Backend(ops, flow, opts)
    bk.mesh.set_geometry(X, np.asarray(ops.topology.elem_nodes)[:, :bk.mesh.nf])
    R_ref, w_ref = ref.residual(g["U"])
    R, w = bk.residual(g["U"])
    assert rel(R, R_ref) < 1e-12 and rel(w, w_ref) < 1e-12


def test_lean_operators_with_device_metrics(cuda):
    """Operators built without inverse mass matrices: the device builds them, the residual is unchanged."""
    cfg, opm = pkg("config"), pkg("operators")
    ops, g = tiny_ops("quad", 3)
    lean = opm.build_operators(ops.topology, ops.node_coords, 3, lean=True)
    flow, opts = cfg.FlowConditions(flux="roe"), cfg.SolverOptions()
    ref = pkg("backend").B200Backend(ops, flow, opts)
    bk = pkg("backend").B200Backend(lean, flow, opts, device_metrics=True)
    assert rel(bk.mesh.arrays["minv"].cpu().numpy(), ref.mesh.arrays["minv"].cpu().numpy()) < 1e-11
    R_ref, _ = ref.residual(g["U"])
    R, _ = bk.residual(g["U"])
    assert rel(R, R_ref) < 1e-12
