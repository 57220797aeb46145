"""The C ABI library loads and exports every function include/*.h declares (no device calls)."""

from __future__ import annotations

import ctypes
import glob
import os
import re
import types

import numpy as np
import pytest

from conftest import ROOT, pkg


def declared_functions() -> set[str]:
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(nzb_\w+)\s*\(", text))
    return names


@pytest.fixture(scope="module")
def lib():
    path = pkg("build").build()
    return ctypes.CDLL(path)


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_the_header():
    bound = {n for n, _, _ in pkg("capi").SIGNATURES}
    assert declared_functions() <= bound


def test_table_sizes_agree_with_the_packer():
    capi, layout, re_ = pkg("capi"), pkg("layout"), pkg("refelem")
    lib = capi.load()
    for kind, k in (("tri", 0), ("quad", 1)):
        for p in range(4):
            tab = layout.element_tables(re_.ref_tables(kind, p))
            assert lib.nzb_table_size(k, p) == tab.size
    assert lib.nzb_table_size(0, 4) == -1
    assert lib.nzb_version() == 1


def test_struct_layouts_match_the_header():
    capi = pkg("capi")
    # 4 x int32 + 2 x int64 + 10 pointers
    assert ctypes.sizeof(capi.Mesh) == 16 + 16 + 16 * 8
    assert ctypes.sizeof(capi.Physics) == 3 * 8 + 8 + 9 * 8 + 4 * 8 + 8 + 4 * 8 + 8
    assert ctypes.sizeof(capi.StageArgs) == 8 * 8 + 3 * 8 + 8
    assert ctypes.sizeof(capi.BatchMarch) == 8 + 12 * 8 + 2 * 8 + 2 * 4
    assert ctypes.sizeof(capi.AdjointArgs) == 8 + 11 * 8
    assert ctypes.sizeof(capi.AdjointBuffers) == 9 * 8
    assert ctypes.sizeof(capi.AdjointMarch) == 8 + 9 * 8 + 8 + 2 * 4
    assert ctypes.sizeof(capi.ObsArgs) == 8 + 2 * 4 + 3 * 8 + 2 * 8 + 8
    assert ctypes.sizeof(capi.GeometryArgs) == 3 * 8 + 16 * 8 + 4 * 8


def test_lebesgue_constant_bounds_probe_values():
    layout, re_ = pkg("layout"), pkg("refelem")
    for kind, p, expect in (("tri", 3, 2.031), ("quad", 3, 2.133), ("tri", 1, 1.0)):
        assert abs(layout.lebesgue_constant(re_.ref_tables(kind, p)) - expect) < 1e-3


def test_physics_struct_constants():
    layout, cfg, re_ = pkg("layout"), pkg("config"), pkg("refelem")
    flow = cfg.FlowConditions(flux="hllc", backflow=True)
    ph = layout.physics_struct(flow, cfg.SolverOptions(), re_.ref_tables("tri", 1))
    assert ph.flux == 1 and ph.limiter == 1
    assert ph.in_rho_t == pytest.approx(2.5) and ph.bf_rho_t == pytest.approx(2.5)
    assert ph.p_back == pytest.approx(0.15)
    assert list(ph.norm_w) == pytest.approx([1.0, 1 / 0.7483314773547883, 1 / 0.7483314773547883, 1 / 0.56])
    with pytest.raises(NotImplementedError):
        layout.physics_struct(types.SimpleNamespace(flux="slau2"), cfg.SolverOptions(), None)


def test_device_metric_arrays_from_lean_operators():
    """Lean operators (no inverse mass) give general-geometry arrays with a zero minv to fill on the device."""
    lay, opm = pkg("layout"), pkg("operators")
    from conftest import tiny_ops

    ops, _ = tiny_ops("quad", 2)
    lean = opm.build_operators(ops.topology, ops.node_coords, 2, lean=True)
    with pytest.raises(ValueError, match="inverse mass"):
        lay.host_arrays(lean)
    full, dev = lay.host_arrays(ops), lay.host_arrays(lean, device_metrics=True)
    assert dev["minv"].shape == full["minv"].shape and not dev["minv"].any()
    for k in ("geo", "area", "face_nbr", "face_code", "face_edge", "edge_geo", "edge_conn"):
        assert np.array_equal(dev[k], full[k]), k


def test_face_tangent_table_gives_the_edge_jacobians():
    """|sum_v T[f, v] X_v| is each face's |dX/dsigma| (straight faces), for both element kinds."""
    lay = pkg("layout")
    from conftest import tiny_ops

    for kind, p in (("tri", 1), ("quad", 1)):
        ops, _ = tiny_ops(kind, p)
        T = lay.face_tangent_table(ops.ref)
        nv = 3 if kind == "tri" else 4
        Xe = np.asarray(ops.node_coords)[np.asarray(ops.topology.elem_nodes)[:, :nv]]
        ed = ops.topology.edges
        own_e = np.concatenate([ed.iedge_elem[:, 0], ed.bedge_elem])
        own_f = np.concatenate([ed.iedge_face[:, 0], ed.bedge_face])
        t = np.einsum("kv,kvd->kd", T[own_f, :nv], Xe[own_e])
        assert np.allclose(np.hypot(t[:, 0], t[:, 1]), np.asarray(ops.edge_jac)[:, 0], rtol=1e-14, atol=0)
