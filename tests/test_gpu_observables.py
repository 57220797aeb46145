"""Device observables (nzb_observables) against the host sums and the reference's performance()."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import TINY, golden, pkg, rel, tiny_ops

pytestmark = pytest.mark.gpu


def backend(ops, **kw):
    cfg = pkg("config")
    return pkg("backend").B200Backend(ops, cfg.FlowConditions(), cfg.SolverOptions(), **kw)


@pytest.mark.parametrize("kind,p", TINY)
def test_device_sums_match_the_host(cuda, kind, p):
    ops, g = tiny_ops(kind, p)
    obs = pkg("observables")
    host = obs.sums(g["U"], ops, pkg("config").FlowConditions())
    for general in ((False, True) if kind == "tri" else (False,)):
        bk = backend(ops, force_general=general)
        dev = obs.DeviceObservables(bk.mesh, bk.phys, [(ops, 0, 0)], [bk.flow]).sums(bk.mesh.pack(g["U"]))
        assert dev.shape == (1, host.size)
        for k in range(host.size):
            assert rel(dev[0, k], host[k]) < 1e-13, (k, dev[0, k], host[k])


@pytest.mark.parametrize("kind,p", TINY)
def test_backend_performance_matches_the_reference(cuda, kind, p):
    ops, g = tiny_ops(kind, p)
    perf = backend(ops).performance(g["U"], pkg("nozzle").Geometry())
    ref = golden("observables.npz")
    for f in ("thrust", "thrust_wall", "mass_flow_in", "mass_flow_out", "entropy_error", "exit_mach_area_averaged",
              "exit_pressure_ratio", "exit_temperature_ratio", "thrust_coefficient", "discharge_coefficient",
              "thrust_efficiency"):
        assert rel(perf[f], ref[f"{kind}{p}_{f}"]) < 1e-12, f


def test_repeated_launches_give_the_same_bits(cuda):
    ops, g = tiny_ops("quad", 3)
    bk = backend(ops)
    ob = pkg("observables").DeviceObservables(bk.mesh, bk.phys, [(ops, 0, 0)], [bk.flow])
    U = bk.mesh.pack(g["U"])
    a = ob.sums(U)
    b = ob.sums(U)
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


def test_batch_observables_match_each_instance(cuda):
    """One launch per bucket gives each instance's metrics, as the host does from its state."""
    from test_gpu_batch import cases

    insts = cases()
    solver = pkg("batch").BatchSolver(insts)
    solver.run()
    dev = solver.observables()
    res = solver.results(with_state=True)
    obs = pkg("observables")
    for inst, r, d in zip(insts, res, dev):
        if not r.converged:
            continue
        host = obs.performance(r.U, inst.ops, inst.flow, inst.geometry)
        for f in ("thrust", "thrust_wall", "mass_flow_in", "mass_flow_out", "exit_mach", "entropy_error",
                  "thrust_coefficient", "thrust_efficiency"):
            assert rel(d[f], host[f]) < 1e-12, f
