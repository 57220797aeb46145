"""Per-iteration cost of the reference's own Numba backend against the C port (cpu_step.c), one thread each.

Run in a container where the reference is importable (it does not travel with this repository):

    PYTHONPATH=/root/reference python oracle/calibrate_numba.py

For one member of each (element, order, refine) class of the design sweep it
builds the case with the reference's ``build_case`` (for its ``NumbaBackend``)
and with this repository's host restatement (for the C port), checks that both
start from the same state, warms each up, and times fused SSP-RK3 iterations on
one thread (``numba.set_num_threads(1)``; the reference's sweep runs one
single-threaded solve per worker).  Prints one JSON object: per class the
seconds per iteration of each and their ratio.
"""

from __future__ import annotations

import importlib
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _time(fn, seconds=1.5):
    fn()
    t0, n = time.perf_counter(), 0
    while n < 3 or time.perf_counter() - t0 < seconds:
        fn()
        n += 1
    return (time.perf_counter() - t0) / n


def main():
    import numba
    from src.api import build_case
    from src.backends.numba_backend import NumbaBackend
    from src.config import SolverOptions as RefOptions

    from oracle import cpu_port

    nz = importlib.import_module("2d_nozzle_b200.nozzle")
    cfg = importlib.import_module("2d_nozzle_b200.config")
    numba.set_num_threads(1)
    cpu_port.set_threads(1)
    out = {"threads": 1, "numba": numba.__version__, "classes": {}}
    steps = 10
    for element in ("tri", "quad"):
        for order in (1, 2, 3):
            for refine in (1, 2, 3):
                kw = dict(contour="bell", area_ratio=2.5, element=element, order=order, refine=refine, flux="hllc",
                          back_pressure_ratio=0.15)
                rc = build_case(**kw)
                ropts = RefOptions(cfl=None, limiter="positivity", scheme="ssprk3")
                nb = NumbaBackend(rc.operators, rc.flow, ropts)
                from src.timestepping import initialize as ini

                U0 = np.asarray(ini.initial_state(rc.operators, rc.flow, rc.geometry, "quasi1d"))
                flow = cfg.FlowConditions(flux="hllc", back_pressure_ratio=0.15)
                opts = cfg.SolverOptions(limiter="positivity", scheme="ssprk3")
                cs = nz.build_case(element=element, order=order, refine=refine, area_ratio=2.5, contour="bell",
                                   flow=flow, options=opts)
                assert np.abs(cs.initial_state() - U0).max() <= 1e-14 * np.abs(U0).max()
                st = cpu_port.CpuStepper(cs.operators, flow, opts)
                Vn, _ = nb.run(U0, steps, "ssprk3")
                Vc, _ = st.run(U0, steps, "ssprk3")
                agree = float(np.abs(Vn - Vc).max() / np.abs(Vn).max())
                t_n = _time(lambda: nb.run(U0, steps, "ssprk3")) / steps
                t_c = _time(lambda: st.run(U0, steps, "ssprk3")) / steps
                out["classes"][f"{element}:p{order}:r{refine}"] = {
                    "elements": int(rc.operators.n_elem), "numba_s_per_iteration": t_n, "c_port_s_per_iteration": t_c,
                    "c_port_over_numba_time": t_c / t_n, "state_agreement_after_10_steps": agree}
                print(element, order, refine, rc.operators.n_elem, f"{t_n * 1e3:.3f} ms", f"{t_c * 1e3:.3f} ms",
                      f"{t_c / t_n:.2f}", f"{agree:.1e}", file=sys.stderr)
    r = [v["c_port_over_numba_time"] for v in out["classes"].values()]
    out["geometric_mean_c_port_over_numba_time"] = float(np.exp(np.mean(np.log(r))))
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    main()
