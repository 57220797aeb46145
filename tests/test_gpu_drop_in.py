"""The B200 backend answers the reference's own march, call for call.

``tests/golden/drop_in_traces.*`` hold what the reference's ``solve_nozzle``
(src/api.py:247-402 -> src/timestepping/march.py:125-300) asked of its backend
on two small cases -- ``asarray``, the ``run`` chunks with their step counts and
scheme, ``scheme`` and counter reads, ``limiter_activity``, ``to_numpy`` -- and
what the reference's NumPy backend answered (tests/golden/make_golden.py,
``drop_in_traces``).  Each recorded call is replayed here on ``B200Backend``
with the recorded arguments, and its answer compared with the reference's: the
states within 1e-11 normwise, residuals within 1e-10, the counters and scheme
exactly.
"""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, pkg, rel

pytestmark = pytest.mark.gpu

TRACES = json.load(open(os.path.join(GOLDEN, "drop_in_traces.json")))


def _case(meta):
    cfg, nz = pkg("config"), pkg("nozzle")
    c = meta["case"]
    flow = cfg.FlowConditions(flux=c["flux"], back_pressure_ratio=c["back_pressure_ratio"])
    opts = cfg.SolverOptions(cfl=c["cfl"], tolerance=c["tolerance"], limiter=c["limiter"], scheme=c["scheme"],
                             max_iterations=c["max_iterations"], print_interval=0)
    cs = nz.build_case(element=c["element"], order=c["order"], refine=c["refine"], area_ratio=c["area_ratio"],
                       contour=c["contour"], flow=flow, options=opts)
    return cs, flow, opts


def _resolve(v, arrays, name):
    if isinstance(v, dict) and "array" in v:
        return arrays[f"{name}/{v['array']}"]
    if isinstance(v, list):
        return [_resolve(x, arrays, name) for x in v]
    return v


def _agrees(got, want):
    if isinstance(want, np.ndarray):
        got = np.asarray(got)
        assert got.shape == want.shape
        return rel(got, want) < 1e-11
    if isinstance(want, list):
        return len(got) == len(want) and all(_agrees(g, w) for g, w in zip(got, want))
    if isinstance(want, float):
        return abs(got - want) <= 1e-10 * abs(want)
    return got == want


@pytest.mark.parametrize("name", sorted(TRACES))
def test_reference_march_calls_replayed(cuda, name):
    meta = TRACES[name]
    arrays = np.load(os.path.join(GOLDEN, "drop_in_traces.npz"))
    cs, flow, opts = _case(meta)
    U0 = _resolve(meta["log"][0]["args"][0], arrays, name)
    # the host case builder gives the reference's initial state
    assert rel(cs.initial_state(), U0) < 1e-14
    bk = pkg("backend").B200Backend(cs.operators, flow, opts)
    runs = 0
    for k, entry in enumerate(meta["log"]):
        if "read" in entry:
            got = getattr(bk, entry["read"])
            assert _agrees(got, _resolve(entry["value"], arrays, name)), (k, entry["read"], got)
            continue
        args = _resolve(entry["args"], arrays, name)
        kw = {key: _resolve(v, arrays, name) for key, v in entry["kw"].items()}
        out = getattr(bk, entry["call"])(*args, **kw)
        want = _resolve(entry["out"], arrays, name)
        if entry["call"] == "run":
            runs += 1
            U_new, res = out
            assert U_new is not args[0] and not np.shares_memory(np.asarray(U_new), np.asarray(args[0]))
            out = [U_new, res]
        assert _agrees(out, want), (k, entry["call"])
    # the whole march: one single step, then chunks of check_interval up to the cap
    assert runs == 1 + -(-(meta["iterations"] - 1) // opts.check_interval)
