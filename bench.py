"""Benchmark: steady solves/s on one B200, plus the residual-kernel HBM roofline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one steady solve of the reference nozzle case (smooth contour,
area ratio 2.5, p = 1 triangles, refine 1 = 560 elements, Roe, cfl 0.5,
positivity limiter, SSP-RK3, from its quasi-1D initial state to a scaled
residual of 1e-10: 11,751 iterations).  ``value`` times it with the state
resident in HBM (one 8-byte residual read back per 50-step convergence check);
``e2e`` times it through the public backend API the reference's march calls,
``run(U_host, n)``, which copies the state in and out every chunk.

``roofline`` is measured on the residual-kernel microbenchmark: 1,000,000
straight-sided cubic triangles (Np = 10) on the unit rectangle, states drawn
per node (density lognormal(0, 0.3), Mach U[0.2, 3] in a random direction,
pressure lognormal(0, 0.5)), one residual per flux and one SSP-RK3 step with
the positivity limiter; the state (320 MB) is larger than L2.

Multi-GPU: design points are independent, so N GPUs run N replicas
(weak scaling); ``value`` = all ranks' solves / the slowest rank's time.
"""

from __future__ import annotations

import argparse
import importlib
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pkg(name=""):
    return importlib.import_module("2d_nozzle_b200" + (f".{name}" if name else ""))


# ------------------------------------------------------------------ workloads
def config1_case():
    g = np.load(os.path.join(GOLDEN, "config1.npz"))
    cfg = pkg("config")
    topo, _, _ = pkg("mesh").channel_topology("tri", refine=1)
    ops = pkg("operators").build_operators(topo, g["node_coords"], 1)
    flow = cfg.FlowConditions(flux="roe", back_pressure_ratio=0.15)
    opts = cfg.SolverOptions(cfl=0.5, tolerance=1e-10, limiter="positivity", scheme="ssprk3", print_interval=0)
    return ops, flow, opts, g


def microbench_state(n_elem, nbf, gamma=1.4, seed=0):
    rng = np.random.default_rng(seed)
    shape = (n_elem, nbf)
    rho = rng.lognormal(0.0, 0.3, shape)
    mach = rng.uniform(0.2, 3.0, shape)
    ang = rng.uniform(0.0, 2.0 * np.pi, shape)
    p = rng.lognormal(0.0, 0.5, shape)
    a = np.sqrt(gamma * p / rho)
    vx, vy = mach * a * np.cos(ang), mach * a * np.sin(ang)
    E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)
    return np.ascontiguousarray(np.stack([rho, rho * vx, rho * vy, E], -1))


def microbench_case(nx=1000, nr=500):
    topo, xf, rf = pkg("mesh").channel_topology("tri", nx=nx, nr=nr)
    coords = pkg("mesh").rectangle_coords(xf, rf)
    ops = pkg("operators").build_operators(topo, coords, 3, lean=True)
    return ops, microbench_state(ops.n_elem, ops.ref.n_basis)


# ------------------------------------------------------------------ helpers
class Clocks:
    """nvidia-smi sampler over the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index=0):
        self.idx = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [line.split(", ") for line in out.strip().splitlines() if line.strip()]

    def summary(self):
        rows = [r for r in self.lines if len(r) >= 9]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def flush_l2(torch, buf):
    buf.add_(1.0)  # writes 256 MB, twice the 126 MB L2


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------ our arm
def solve_device(bk, U0_dev_soa, opts, scale, torch):
    """The reference march's bookkeeping on a device-resident state (one 8-byte read per check)."""
    S0 = bk._S[0]
    S0.copy_(U0_dev_soa)
    bk.run_device(1)
    res0 = float(bk._res.item())
    done, launches = 1, 4
    res = res0
    window = []
    converged = res0 <= opts.tolerance * scale
    while not converged and done < opts.max_iterations:
        n = min(opts.check_interval, opts.max_iterations - done)
        bk.run_device(n)
        done += n
        launches += 3 * n + 1
        res = float(bk._res.item())
        if not np.isfinite(res) or res > opts.divergence_factor * res0:
            break
        if res <= opts.tolerance * scale:
            converged = True
            break
        window.append(res)
        if len(window) > opts.stall_window:
            window.pop(0)
        if len(window) == opts.stall_window and max(window) > 0 and min(window) / max(window) > opts.stall_ratio:
            break
    return converged, done, res, launches


def microbench(torch, lib_capi, B, cfg, peak_gbs, peak_kind, nx=1000, nr=500):
    ops, U = microbench_case(nx, nr)
    E = ops.n_elem
    out = {"workload": f"residual microbench: {E} straight-sided cubic triangles (Np=10), unit rectangle {nx}x{nr} cells",
           "l2": f"state {U.nbytes / 1e6:.0f} MB vs 126 MB L2", "kernels": {}}
    results = {}
    for flux in ("roe", "hllc", "ausmup"):
        bk = B(ops, cfg.FlowConditions(flux=flux), cfg.SolverOptions(cfl=0.5))
        bk.mesh.pack(U, bk._S[0])
        st = torch.cuda.current_stream()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

        def residual():
            lib_capi.check(bk.lib.nzb_residual(bk.mesh.c_ref, bk._phys_ref, 0, bk._S[0].data_ptr(), bk._S[1].data_ptr(),
                                               bk._wave.data_ptr(), st.cuda_stream), "nzb_residual")

        for _ in range(3):
            residual()
        torch.cuda.synchronize()
        times = []
        for _ in range(5):
            ev[0].record(st)
            residual()
            ev[1].record(st)
            torch.cuda.synchronize()
            times.append(ev[0].elapsed_time(ev[1]) * 1e-3)
        results[f"residual_{flux}"] = float(np.mean(times))
        if flux == "hllc":
            # one SSP-RK3 step with the limiter, stage by stage
            stimes = {1: [], 2: [], 3: []}
            for rep in range(4):
                bk.mesh.pack(U, bk._S[0])
                torch.cuda.synchronize()
                S0, S1, S2 = bk._S
                factor = cfg.step_coefficient(3, 0.5, "ssprk3")
                for V, U0_, o, stage, a, b in ((S0, None, S2, 1, 0.0, 1.0), (S2, S0, S1, 2, 0.75, 0.25),
                                              (S1, S0, S0, 3, 1 / 3, 2 / 3)):
                    args = lib_capi.StageArgs()
                    args.V, args.out, args.dt = V.data_ptr(), o.data_ptr(), bk._dt.data_ptr()
                    args.U0 = U0_.data_ptr() if U0_ is not None else None
                    args.norm_partial = bk._partial.data_ptr() if stage == 1 else None
                    args.counters = bk._counters.data_ptr()
                    args.dt_factor, args.a, args.b, args.stage = factor, a, b, stage
                    ev[0].record(st)
                    lib_capi.check(bk.lib.nzb_stage(bk.mesh.c_ref, bk._phys_ref, lib_capi.C.byref(args), st.cuda_stream), "nzb_stage")
                    ev[1].record(st)
                    torch.cuda.synchronize()
                    if rep > 0:
                        stimes[stage].append(ev[0].elapsed_time(ev[1]) * 1e-3)
            cnt = bk._counters.cpu().numpy()
            out["limited_fraction_per_stage"] = float(cnt[0]) / (4 * 3 * E)
            for k in (1, 2, 3):
                results[f"stage{k}_hllc"] = float(np.mean(stimes[k]))
        del bk
        torch.cuda.empty_cache()
    # algorithmic bytes per element: state in/out, geometry, connectivity, edges once
    S = 10 * 4 * 8
    n_edge = ops.n_edges_total
    base = 40 + 36 + 32.0 * n_edge / E
    alg = {"residual": 2 * S + base + 8, "stage1": 2 * S + base + 8 + 8, "stage23": 3 * S + base + 8 + 8}
    for name, t in results.items():
        b = alg["residual"] if name.startswith("residual") else (alg["stage1"] if name.startswith("stage1") else alg["stage23"])
        out["kernels"][name] = {"ms": t * 1e3, "alg_bytes_per_elem": b, "gbs": b * E / t / 1e9}
    dom = max(results, key=results.get)
    k = out["kernels"][dom]
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": k["gbs"], "peak": peak_gbs, "unit": "GB/s",
                       "frac": k["gbs"] / peak_gbs, "peak_source": peak_kind, "traffic": None,
                       "workload": out["workload"]}
    return out


def cpu_baseline_oracle(seconds=15.0):
    """The oracle (NumPy restatement) marching config 1 for a bounded number of iterations."""
    from oracle import dg_oracle as orc

    ops, flow, opts, g = config1_case()
    st = orc.Stepper(ops, flow, opts)
    U = g["U0"].copy()
    st.run(U, 2)
    t0 = time.perf_counter()
    n = 0
    while time.perf_counter() - t0 < seconds:
        U, _ = st.run(U, 5)
        n += 5
    dt = (time.perf_counter() - t0) / n
    iters = int(g["iterations"])
    return {"value": 1.0 / (dt * iters), "unit": "solves/s", "cores": 1, "kind": "port",
            "sample": f"{n} SSP-RK3 iterations of the config-1 march ({dt * 1e3:.2f} ms each), scaled to the "
                      f"reference's {iters} iterations per solve; NumPy oracle, single thread"}


def run_ours(args, rank, world, torch, dist):
    capi = pkg("capi")
    cfg = pkg("config")
    B = pkg("backend").B200Backend
    march = pkg("march")
    peak, peak_kind = load_peaks()
    ops, flow, opts, g = config1_case()
    bk = B(ops, flow, opts)
    scale = cfg.residual_scale(flow, float(g["length"]))
    U0 = bk.mesh.pack(g["U0"]).clone()
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    for _ in range(max(3, args.warmup)):
        conv, its, res, _ = solve_device(bk, U0, opts, scale, torch)
    if not conv or its != int(g["iterations"]):
        raise RuntimeError(f"warm-up solve did not reproduce the reference: converged={conv}, iterations={its}")

    times, launches = [], 0
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        for _ in range(args.steps):
            flush_l2(torch, flush)
            ev[0].record(st)
            conv, its, res, nl = solve_device(bk, U0, opts, scale, torch)
            ev[1].record(st)
            torch.cuda.synchronize()
            times.append(ev[0].elapsed_time(ev[1]) * 1e-3)
            launches += nl
            assert conv and its == int(g["iterations"])
    if dist is not None:
        dist.barrier()
    t_rank = float(np.sum(times))
    t_max = t_rank
    if dist is not None:
        tt = torch.tensor([t_rank], dtype=torch.float64, device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    value = world * args.steps / t_max

    # end to end through the public API: host state in and out every chunk
    pin = torch.from_numpy(g["U0"].copy()).pin_memory()
    e2e_times = []
    state_bytes = g["U0"].nbytes
    chunks = None
    for k in range(args.steps + 1):
        bk2 = bk
        bk2.n_limited = bk2.n_limit_calls = bk2.n_mean_repaired = 0
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        U0h = pin.numpy()
        r = march.solve(bk2, U0h, length=float(g["length"]))
        torch.cuda.synchronize()
        if k > 0:
            e2e_times.append(time.perf_counter() - t0)
        chunks = len(r.history_iterations)
        assert r.converged and r.iterations == int(g["iterations"])
    e2e_value = world / float(np.mean(e2e_times))

    line = {
        "metric": "steady solves/s at 1e-10 residual (plain, one solve at a time; batched sweep not yet built)",
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": max(3, args.warmup),
        "ms_per_step": 1e3 * t_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: the reference's own mesh and quasi-1D initial state for config 1 (fixtures in tests/golden)",
        "config": {"workload": "config1: smooth AR 2.5, tri p=1, refine 1 (560 elements), Roe, cfl 0.5, tol 1e-10",
                   "iterations_per_solve": int(g["iterations"]), "l2": "flushed (256 MB write) between solves",
                   "parallelism": f"replicas x{world}"},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(state_bytes * chunks),
                "d2h_bytes_per_step": int((state_bytes + 8) * chunks), "path": "march -> B200Backend.run(host U, 50)"},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and not args.no_micro:
        mb = microbench(torch, capi, B, cfg, peak, peak_kind)
        line["roofline"] = mb.pop("roofline")
        line["microbench"] = mb
    if rank == 0:
        line["cpu_baseline"] = cpu_baseline_oracle(args.cpu_seconds)
    return line


def run_reference(args):
    """The reference's CPU path (the NumPy oracle restating it) on config 1."""
    from oracle import dg_oracle as orc

    ops, flow, opts, g = config1_case()
    st = orc.Stepper(ops, flow, opts)
    U = g["U0"].copy()
    sample = 25
    for _ in range(args.warmup):
        U, _ = st.run(U, sample)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        U, _ = st.run(U, sample)
        ts.append(time.perf_counter() - t0)
    per_it = float(np.sum(ts)) / (sample * args.steps)
    iters = int(g["iterations"])
    value = 1.0 / (per_it * iters)
    return {
        "impl": "reference", "metric": "steady solves/s at 1e-10 residual (plain, one solve at a time; batched sweep not yet built)",
        "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(ts)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "the reference's config-1 mesh and initial state",
        "config": {"workload": "config1: smooth AR 2.5, tri p=1, refine 1 (560 elements), Roe, cfl 0.5, tol 1e-10"},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": 1, "kind": "port",
                         "sample": f"each step = {sample} SSP-RK3 iterations of the NumPy oracle, scaled to {iters} per solve"},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-micro", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--micro-only", action="store_true", help="run only the residual microbench (profiling)")
    ap.add_argument("--micro-nx", type=int, default=1000, help="microbench cells along x (two triangles per cell)")
    ap.add_argument("--micro-nr", type=int, default=500, help="microbench cells across")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)))
        return
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    pkg("build").build()
    if args.micro_only:
        peak, kind = load_peaks()
        print(json.dumps(microbench(torch, pkg("capi"), pkg("backend").B200Backend, pkg("config"), peak, kind,
                                    args.micro_nx, args.micro_nr)))
        return
    line = run_ours(args, rank, world, torch, dist)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
