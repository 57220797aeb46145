"""Orders above 3 and curved (Q = 2) elements on the device (csrc/generic.cuh, GenericB200Backend) against
the reference's fixtures: residual, rate and wave per flux and with backflow, the limiter, three SSP-RK3
steps; twenty steps against the oracle; the generic kernels on a p = 3 straight mesh against the
specialised ones."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import pkg, rel, tiny_ops
from oracle import dg_oracle as orc
from test_oracle_generic import CASES, generic_ops

pytestmark = pytest.mark.gpu


def backend(ops, flux="roe", **opt):
    cfg = pkg("config")
    flow = cfg.FlowConditions(flux=flux, **{k: v for k, v in opt.items() if k == "backflow"})
    opts = cfg.SolverOptions(scheme="ssprk3", **{k: v for k, v in opt.items() if k != "backflow"})
    return pkg("backend").B200Backend(ops, flow, opts)


@pytest.mark.parametrize("kind,p,q", CASES)
def test_generic_kernels_match_the_reference(cuda, kind, p, q):
    ops, g = generic_ops(kind, p, q)
    for flux in ("roe", "hllc", "ausmup"):
        bk = backend(ops, flux)
        assert type(bk).__name__ == "GenericB200Backend"
        R, wave = bk.residual(g["U"])
        F, _ = bk.rate(g["U"])
        assert rel(R, g[f"R_{flux}"]) < 1e-12 and rel(wave, g[f"wave_{flux}"]) < 1e-12
        assert rel(F, g[f"rate_{flux}"]) < 1e-12
        assert rel(bk.inverse_mass(R), -g[f"rate_{flux}"]) < 1e-12
    bb = backend(ops, "roe", backflow=True)
    assert rel(bb.residual(g["U"])[0], g["R_roe_backflow"]) < 1e-12
    bk = backend(ops)
    assert rel(bk.limit(g["U_bad"]), g["limited_bad"]) < 1e-12
    assert bk.n_limited > 0
    V, res = bk.run(g["U"], 3, "ssprk3")
    assert rel(V, g["run3_ssprk3"]) < 1e-11
    assert abs(res - g["run3_ssprk3_res"]) <= 1e-11 * g["run3_ssprk3_res"]


@pytest.mark.parametrize("kind,p,q", [("tri", 5, 1), ("quad", 2, 2)])
def test_generic_march_follows_the_oracle(cuda, kind, p, q):
    ops, g = generic_ops(kind, p, q)
    cfg = pkg("config")
    bk = backend(ops, "hllc", cfl=0.5)
    V, res = bk.run(g["U"], 20, "ssprk3")
    W, res_ref = orc.Stepper(ops, cfg.FlowConditions(flux="hllc"), cfg.SolverOptions(scheme="ssprk3", cfl=0.5)).run(
        g["U"].copy(), 20)
    assert rel(V, W) < 1e-10 and abs(res - res_ref) <= 1e-10 * res_ref


def test_generic_kernels_agree_with_the_specialised_ones(cuda):
    """On a straight p = 3 mesh, the generic path (forced) against the specialised kernels."""
    ops, g = tiny_ops("tri", 3)
    cfg = pkg("config")
    flow, opts = cfg.FlowConditions(flux="hllc"), cfg.SolverOptions(scheme="ssprk3")
    gen = pkg("generic").GenericB200Backend(ops, flow, opts)
    spec = pkg("backend").B200Backend(ops, flow, opts)
    for U in (g["U"], g["U_bad"]):
        assert rel(gen.residual(U)[0], spec.residual(U)[0]) < 1e-12
        assert rel(gen.limit(U), spec.limit(U)) < 1e-12
    assert rel(gen.run(g["U"], 3, "ssprk3")[0], spec.run(g["U"], 3, "ssprk3")[0]) < 1e-11
