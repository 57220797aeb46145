"""The Superbee TVB slope limiter (then positivity) on the device, against the reference's fixtures."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import golden, pkg, rel, tiny_ops
from oracle import dg_oracle as orc

pytestmark = pytest.mark.gpu
CASES = [("tri", 1), ("tri", 2), ("tri", 3), ("quad", 1), ("quad", 2), ("quad", 3)]


def backend(ops, **opt):
    cfg = pkg("config")
    return pkg("backend").B200Backend(ops, cfg.FlowConditions(), cfg.SolverOptions(limiter="superbee", **opt))


@pytest.mark.parametrize("kind,p", CASES)
def test_superbee_limit_matches_the_reference(cuda, kind, p):
    ops, _ = tiny_ops(kind, p)
    g = golden(f"superbee_{kind}_p{p}.npz")
    bk = backend(ops)
    out = bk.limit(g["U"])
    assert rel(out, g["superbee_positivity"]) < 1e-12
    ref, _ = orc.superbee(g["U"], ops, 50.0)
    assert rel(out, orc.positivity(ref, ops, pkg("config").FlowConditions())[0]) < 1e-12


@pytest.mark.parametrize("kind,p", CASES)
def test_superbee_ssprk3_steps_match_the_reference(cuda, kind, p):
    ops, _ = tiny_ops(kind, p)
    g = golden(f"superbee_{kind}_p{p}.npz")
    bk = backend(ops, scheme="ssprk3")
    V, res = bk.run(g["U"], 3, "ssprk3")
    assert rel(V, g["run3_ssprk3"]) < 1e-11
    assert abs(res - g["run3_ssprk3_res"]) <= 1e-11 * abs(g["run3_ssprk3_res"])


def test_superbee_is_refused_in_a_batch(cuda):
    cfg, nz = pkg("config"), pkg("nozzle")
    opts = cfg.SolverOptions(limiter="superbee")
    cs = nz.build_case(element="tri", order=1, refine=0, options=opts)
    inst = pkg("batch").Instance(cs.operators, cs.flow, opts, cs.initial_state(), cs.geometry.length)
    with pytest.raises(NotImplementedError):
        pkg("batch").BatchSolver([inst])
