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


STRUCTS = {"Mesh": "nzb_mesh", "Physics": "nzb_physics", "StageArgs": "nzb_stage_args", "Buffers": "nzb_buffers",
           "BatchMarch": "nzb_batch_march", "AdjointArgs": "nzb_adjoint_args", "AdjointBuffers": "nzb_adjoint_buffers",
           "AdjointMarch": "nzb_adjoint_march", "ObsArgs": "nzb_obs_args", "GeometryArgs": "nzb_geometry_args",
           "InitialArgs": "nzb_initial_args", "GenMesh": "nzb_gen_mesh", "GenUpdateArgs": "nzb_gen_update_args",
           "GenGeometryArgs": "nzb_gen_geometry_args", "GenInitialArgs": "nzb_gen_initial_args",
           "GenObsArgs": "nzb_gen_obs_args"}


def test_struct_layouts_match_the_header(tmp_path):
    """Every ctypes structure has the C compiler's size and field offsets for the header's struct."""
    import shutil
    import subprocess

    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    capi = pkg("capi")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "nozzle_b200.h"', "int main(void) {"]
    for py, c in STRUCTS.items():
        lines.append(f'  printf("{py} size %zu\\n", sizeof({c}));')
        for name, _ in getattr(capi, py)._fields_:
            lines.append(f'  printf("{py} {name} %zu\\n", offsetof({c}, {name}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {tuple(line.split()[:2]): int(line.split()[2]) for line in out if line}
    for py in STRUCTS:
        cls = getattr(capi, py)
        assert got[(py, "size")] == ctypes.sizeof(cls), py
        for name, _ in cls._fields_:
            assert got[(py, name)] == getattr(cls, name).offset, (py, name)


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
