"""Benchmark: batched steady design-sweep solves/s on one B200, with the plain
(one solve at a time) rate on the same points, the residual-kernel roofline and
the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one batched sweep: 256 operating points sampled with seed 0 (area
ratio U[1.5, 4], back-pressure ratio U[0.1, 0.9], p in {1, 2, 3}, refine in
{1, 2, 3}, triangles / quadrilaterals 50/50, bell contour, HLLC, positivity
limiter, SSP-RK3, tolerance 1e-10).  Points that stand a normal shock in the
nozzle are refused on the host, as the reference's sweep records them; every
other point is marched from its quasi-1D initial state, all together, each to
its own retirement (converged, stalled, diverged, non-finite or the iteration
cap).  ``value`` counts converged solves per second with every state resident
in HBM; ``e2e`` times the public path -- BatchSolver set-up from host arrays
(states, geometry, connectivity copied in), the march, every status and each
point's performance() metrics (thrust, mass flows, exit averages, entropy
error: integrated on the device, only the sums copied back).  ``plain`` marches a subset one instance at a time through
the single-solve backend and the same subset as a batch: their ratio is the
batched speed-up over the same attempted set.

``adjoint`` times thrust gradients w.r.t. eight Bezier wall offsets for 64
perturbed members (AR 2.5, p = 2 triangles, refine 2, AUSM+-up, forward and
adjoint to 1e-10): all members as one batch (forward batch, one adjoint march
object in which each member starts as soon as its own forward solve converges,
one coordinate-VJP launch) against every 8th member one at a time; the same
batch with the forward and adjoint phases run one after the other is timed
beside it.

``roofline`` is measured on the residual-kernel microbenchmark: 1,000,000
straight-sided cubic triangles (Np = 10) on the unit rectangle, states drawn
per node (density lognormal(0, 0.3), Mach U[0.2, 3] in a random direction,
pressure lognormal(0, 0.5)), one residual per flux and one SSP-RK3 step with
the positivity limiter; the state (320 MB) is larger than L2.

``cpu_baseline`` and ``--impl reference`` time the reference's compiled CPU
step -- its Numba backend, restated in C with OpenMP (oracle/cpu_step.c; the
reference's Python source does not travel with this repository): seconds per
fused SSP-RK3 iteration of one member of each (kind, order, mesh) class, times
every point's iteration count, the points spread over every host core one
single-threaded march each, as the reference's process-pool sweep runs them.

Multi-GPU: design points are independent, so N GPUs split one sweep of 256 N
points, 256 per GPU (weak scaling); ``value`` = all ranks' converged solves /
the slowest rank's time.
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
def microbench_state(n_elem, nbf, gamma=1.4, seed=0):
    """The microbenchmark's seeded per-node states (the package's generator, so tests draw the same ones)."""
    return pkg("autotune").random_states(n_elem, nbf, gamma, seed)


def microbench_case(nx=1000, nr=500, kind="tri", order=3):
    topo, xf, rf = pkg("mesh").channel_topology(kind, nx=nx, nr=nr)
    coords = pkg("mesh").rectangle_coords(xf, rf)
    ops = pkg("operators").build_operators(topo, coords, order, lean=True)
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


def microbench(torch, lib_capi, B, cfg, peak_gbs, peak_kind, nx=1000, nr=500, kind="tri", order=3):
    ops, U = microbench_case(nx, nr, kind, order)
    E, NP = ops.n_elem, int(ops.ref.n_basis)
    shape = {"tri": "triangles", "quad": "quadrilaterals"}[kind]
    out = {"workload": f"residual microbench: {E} straight-sided p={order} {shape} (Np={NP}), unit rectangle {nx}x{nr} "
                       f"cells", "l2": f"state {U.nbytes / 1e6:.0f} MB vs 126 MB L2", "kernels": {}}
    results = {}
    for flux in ("roe", "hllc", "ausmup"):
        bk = B(ops, cfg.FlowConditions(flux=flux), cfg.SolverOptions(cfl=0.5), device_metrics=kind != "tri")
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
                factor = cfg.step_coefficient(order, 0.5, "ssprk3")
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
    # algorithmic bytes per element: the state read and the result written (S = NP * 4 * 8 bytes each;
    # stages 2 and 3 also read the step's start state), the element geometry (affine: inverse Jacobian and
    # det, 40 B; general: the vertices, 64 B, and for rates and stages the inverse mass, NP^2 * 8 B), the
    # connectivity (neighbour, edge and face code per face: 12 B each), every edge's normal, |dX/dsigma| and
    # length once (32 B per edge), and the element's wave speed or local step (8 B; stage 1 also reads the area)
    S = NP * 4 * 8
    n_edge = ops.n_edges_total
    nf = 3 if kind == "tri" else 4
    geo = 40 if kind == "tri" else 2 * nf * 8  # the residual applies no inverse mass
    minv = 0 if kind == "tri" else NP * NP * 8  # general geometry: per-element inverse mass, read by rates and stages
    base = geo + 12 * nf + 32.0 * n_edge / E
    alg = {"residual": 2 * S + base + 8, "stage1": 2 * S + base + minv + 8 + 8,
           "stage23": 3 * S + base + minv + 8 + 8}
    for name, t in results.items():
        b = alg["residual"] if name.startswith("residual") else (alg["stage1"] if name.startswith("stage1") else alg["stage23"])
        out["kernels"][name] = {"ms": t * 1e3, "alg_bytes_per_elem": b, "gbs": b * E / t / 1e9}
    # FP64 operations per element (2 per DFMA, 1 per DADD or DMUL thread instruction; divisions and square
    # roots count as the instructions they compile to), counted by ncu on 490,000 cubic triangles and 245,000
    # cubic quadrilaterals of the same state distribution with the one-thread kernels (the stages' counts
    # depend on how many elements the limiter works on, 53 % / 66 % here)
    fp64 = {("tri", 3): {"residual_roe": 9067.1, "residual_hllc": 9323.5, "residual_ausmup": 8753.7,
                         "stage1_hllc": 12996.2, "stage2_hllc": 12945.0, "stage3_hllc": 12938.8},
            ("quad", 3): {"residual_roe": 13154.5, "residual_hllc": 13496.5, "residual_ausmup": 12721.2,
                          "stage1_hllc": 21072.5, "stage2_hllc": 20930.6, "stage3_hllc": 20979.5}}.get((kind, order), {})
    # nominal FP64 peak: 148 SMs x 64 FP64 lanes x 2 flops per FMA at 1965 MHz
    peak_fp64 = 148 * 64 * 2 * 1.965e9 / 1e12
    for name, t in results.items():
        if name in fp64:
            out["kernels"][name]["fp64_tflops"] = fp64[name] * E / t / 1e12
    dom = max(results, key=results.get)
    k = out["kernels"][dom]
    # DRAM bytes per element of each kernel from an ncu capture of 490,000 cubic triangles
    # (profiles/k_element_stage_tri_p3_490k.md), scaled to this launch by its element count
    traffic = ({"residual_roe": 1055.0, "stage1_hllc": 1139.0, "stage2_hllc": 1510.0, "stage3_hllc": 1446.0}
               if (kind, order) == ("tri", 3) else {})
    out["roofline"] = {"bound": "hbm", "kernel": dom, "achieved": k["gbs"], "peak": peak_gbs, "unit": "GB/s",
                       "frac": k["gbs"] / peak_gbs, "peak_source": peak_kind,
                       "traffic": traffic[dom] * E if dom in traffic else None,
                       "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum on 490,000 elements, "
                                         "scaled by element count", "workload": out["workload"]}
    if dom in fp64:
        f = fp64[dom]
        ach = f * E / results[dom] / 1e12
        # arithmetic intensity above the FP64 ridge caps the attainable HBM fraction below 1
        out["roofline"]["fp64"] = {
            "flops_per_elem": f, "achieved_tflops": ach, "peak_tflops": peak_fp64, "frac": ach / peak_fp64,
            "peak_source": "nominal (148 SMs x 64 FP64 lanes x 2 flops x 1965 MHz)",
            "intensity_flop_per_byte": f / k["alg_bytes_per_elem"],
            "ridge_flop_per_byte": peak_fp64 * 1e3 / peak_gbs,
            "hbm_frac_at_fp64_peak": min(1.0, peak_fp64 * 1e12 / f * k["alg_bytes_per_elem"] / (peak_gbs * 1e9))}
    return out


SWEEP_POINTS = 256
SWEEP_SEED = 0


def sweep_workload(max_iterations, n_points=SWEEP_POINTS, rank=0, world=1, lean=True):
    """This rank's share of one sweep of ``n_points * world`` design points (seed 0): points rank, rank + world, ...
    (with one rank, the whole ``n_points``-point sweep).  ``lean``: the cases as the GPU path builds them
    (metric terms and initial states left to the device); otherwise with the reference's full host
    operators and initial states (what the CPU legs run on)."""
    sweep = pkg("sweep")
    points = pkg("replicas").partition(sweep.sample_points(n_points * world, SWEEP_SEED), rank, world)
    insts, index, refused = sweep.build_instances(points, max_iterations=max_iterations, lean=lean)
    return points, insts, index, refused


def _classes(insts):
    classes = {}
    for i, inst in enumerate(insts):
        classes.setdefault((inst.ops.ref.kind, inst.ops.ref.order, inst.ops.n_elem), i)
    return classes


def _port_cost(inst, per, chunk=10):
    """Seconds per fused SSP-RK3 iteration of the C port on one instance, one thread, timed for about
    ``per`` seconds in chunks of ``chunk`` steps (each chunk copies the state in and out once, as the
    reference's run() does)."""
    from oracle import cpu_port

    cpu_port.set_threads(1)
    st = cpu_port.CpuStepper(inst.ops, inst.flow, inst.opts)
    U, _ = st.run(np.asarray(inst.U0, float), 1)
    t0, n = time.perf_counter(), 0
    while n < 2 * chunk or time.perf_counter() - t0 < per:
        U, _ = st.run(U, chunk)
        n += chunk
    return (time.perf_counter() - t0) / n


def port_costs(insts, seconds):
    """Seconds per iteration of the C port for each (kind, order, n_elem) class of the sweep, one member
    each, one after another on one thread, within a total of about ``seconds``."""
    classes = _classes(insts)
    per = seconds / max(1, len(classes))
    return {key: _port_cost(insts[i], per) for key, i in classes.items()}, len(classes)


def _class_cost(args):
    """Worker: the C port's seconds per iteration on one instance (one thread), timed for about ``per`` s."""
    inst, per = args
    return _port_cost(inst, per)


def port_costs_parallel(insts, seconds, workers):
    """port_costs with every host core busy: one class per worker process at a time (spawned), so each
    per-iteration cost is measured under the contention a parallel CPU sweep would see."""
    from concurrent.futures import ProcessPoolExecutor
    import multiprocessing as mp

    classes = _classes(insts)
    keys = list(classes)
    rounds = -(-len(keys) // workers)
    per = seconds / max(1, rounds)
    with ProcessPoolExecutor(workers, mp_context=mp.get_context("spawn")) as ex:
        costs = list(ex.map(_class_cost, [(insts[classes[k]], per) for k in keys]))
    return dict(zip(keys, costs)), len(keys)


def port_solve_seconds(inst, iterations, chunk=50):
    """Wall time of one whole march on the C port: ``iterations`` steps from the initial state in chunks of
    ``chunk`` (the march's check interval), one thread."""
    from oracle import cpu_port

    cpu_port.set_threads(1)
    st = cpu_port.CpuStepper(inst.ops, inst.flow, inst.opts)
    U = np.asarray(inst.U0, float)
    t0 = time.perf_counter()
    U, _ = st.run(U, 1)
    done = 1
    while done < iterations:
        n = min(chunk, iterations - done)
        U, _ = st.run(U, n)
        done += n
    return time.perf_counter() - t0


def parallel_makespan(insts, iterations, cost, workers):
    """Wall time of the sweep on ``workers`` cores: instances assigned longest first to the least
    loaded core (each instance is one serial march)."""
    times = sorted((it * cost[(inst.ops.ref.kind, inst.ops.ref.order, inst.ops.n_elem)]
                    for inst, it in zip(insts, iterations)), reverse=True)
    load = [0.0] * workers
    for t in times:
        k = load.index(min(load))
        load[k] += t
    return max(load)


def plain_solve(inst, torch, variants="single"):
    """One instance through the single-solve backend, state resident in HBM (a lean instance: metric terms
    and initial state built on the device, as the batch builds them).  ``variants``: the single-solve
    kernels (the variant table's latency choice) or the batch's."""
    cfg = pkg("config")
    lean = getattr(inst.ops, "inv_mass", None) is None
    bk = pkg("backend").B200Backend(inst.ops, inst.flow, inst.opts, device_metrics=lean, variants=variants)
    U0 = (bk.initial_state(inst.geometry, host=False) if inst.U0 is None else bk.mesh.pack(inst.U0)).clone()
    scale = cfg.residual_scale(inst.flow, inst.length)
    return bk, U0, scale


def bezier8_members(n, sigma=0.02, seed=0):
    """Eight radial wall offsets per member, Gaussian (sigma: a fraction of the throat half-height)."""
    rng = np.random.default_rng(seed)
    return [{f"offset_{k}": float(v) for k, v in enumerate(rng.normal(0.0, sigma, 8))} for _ in range(n)]


def adjoint_section(args, torch):
    """Batched vs one-at-a-time thrust gradients w.r.t. the 8 Bezier offsets (AR 2.5, p = 2 triangles,
    refine 2, AUSM+-up, p_b 0.15; forward and adjoint to 1e-10)."""
    ad = pkg("adjoint")
    dc = ad.differentiable_case(contour="bezier8", area_ratio=2.5, order=2, refine=2, flux="ausmup",
                                back_pressure_ratio=0.15, tolerance=1e-10, max_iterations=args.adjoint_cap)
    members = bezier8_members(args.adjoint_members)
    names = tuple(members[0])
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    # the members' host set-up (mesh, operators, initial state) is timed, as the plain path's is
    bg = ad.BatchGradient(dc, members, "thrust", names=names)
    out = bg.run(adjoint_tolerance=1e-10)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t0
    ok = [r for r in out if r.grad is not None]
    # the same batch with every forward solve finished before any adjoint starts (for comparison)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bg_p = ad.BatchGradient(dc, members, "thrust", names=names)
    out_p = bg_p.run(adjoint_tolerance=1e-10, overlap=False)
    torch.cuda.synchronize()
    t_phased = time.perf_counter() - t0
    same = max([abs(a.grad[k] - b.grad[k]) / max(abs(b.grad[k]), 1e-12) for a, b in zip(out, out_p)
                if a.grad is not None and b.grad is not None for k in names] or [0.0])
    sub = list(range(0, len(members), args.plain_stride))
    t0 = time.perf_counter()
    plain = {}
    for i in sub:
        try:
            plain[i] = dc.value_and_gradient("thrust", members[i], names=names, adjoint_tolerance=1e-10)[1]
        except RuntimeError:  # the member's forward or adjoint march failed, as in the batch
            plain[i] = None
    torch.cuda.synchronize()
    t_plain = time.perf_counter() - t0
    n_plain = sum(g is not None for g in plain.values())
    diff = max([abs(out[i].grad[k] - g[k]) / max(abs(g[k]), 1e-12) for i, g in plain.items() for k in names
                if g is not None and out[i].grad is not None] or [0.0])

    # every member one at a time, estimated: a plain member costs its forward iterations times the plain
    # forward march's cost per iteration, its adjoint iterations times the plain adjoint march's, plus a
    # fixed set-up (case build, seeds, coordinate products) taken from the measured subset; the iteration
    # counts are the batch's own, which equal the plain ones
    batch = pkg("batch")
    cs0 = dc.case_at(members[0])
    inst0 = batch.Instance(cs0.operators, cs0.flow, dc.options, cs0.initial_state(), float(cs0.geometry.length))
    ci = dc.options.check_interval

    def per_iteration(variants):
        """Seconds per plain forward iteration and per plain adjoint RK4 step of member 0."""
        bk, U0, _ = plain_solve(inst0, torch, variants=variants)
        bk._S[0].copy_(U0)
        bk.run_device(1)
        bk.run_device(ci)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(10):
            bk.run_device(ci)
            float(bk._res.item())
        t_f = (time.perf_counter() - t0) / (10 * ci)
        model = ad.AdjointModel(cs0.operators, cs0.flow, dc.options, variants=variants)
        U_soa = ad.to_soa(torch.as_tensor(np.asarray(cs0.initial_state()), device="cuda"))
        gen = torch.Generator(device="cuda")
        gen.manual_seed(0)
        am = ad.AdjointMarch(model, U_soa, torch.randn(U_soa.shape, generator=gen, dtype=torch.float64,
                                                       device="cuda"), dc.options.cfl)
        am._create(1e-300, 10**9)
        am.run(0)
        am.run(100)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(5):
            am.run(100)
        t_a = (time.perf_counter() - t0) / 500
        del am, bk
        return t_f, t_a

    t_fwd, t_adj = per_iteration("single")
    t_fwd_b, t_adj_b = per_iteration("batch")
    cost = lambda r: r.forward_iterations * t_fwd + r.adjoint_iterations * t_adj  # noqa: E731
    fixed = max(0.0, (t_plain - sum(cost(out[i]) for i in sub)) / len(sub))
    est_all = sum(cost(r) for r in out) + fixed * len(out)
    est_same = sum(r.forward_iterations * t_fwd_b + r.adjoint_iterations * t_adj_b for r in out) + fixed * len(out)
    return {"workload": f"{len(members)} bezier8 members (8 offsets, sigma 2% of the throat half-height, seed 0) "
                        f"around AR 2.5, tri p=2 refine 2 (2240 elements), AUSM+-up, forward and adjoint to 1e-10",
            "metric": "thrust gradients/s (8 design variables each)", "batched_gradients": len(ok),
            "batched_seconds": t_batch, "batched_gradients_per_s": len(ok) / t_batch,
            "plain_attempted": len(sub), "plain_gradients": n_plain, "plain_seconds": t_plain,
            "plain_gradients_per_s": n_plain / t_plain, "speedup": (len(ok) / t_batch) / max(n_plain / t_plain, 1e-300),
            "adjoint_iterations_max": max(r.adjoint_iterations for r in out),
            "forward_iterations_max": max(r.forward_iterations for r in out),
            "max_rel_diff_batched_vs_plain": diff, "batched_phases_s": bg.timings,
            "phased_seconds": t_phased, "phased_phases_s": bg_p.timings, "max_rel_diff_overlapped_vs_phased": same,
            "tail_switch": {"overlapped": bg.tail_switched, "phased": bg_p.tail_switched},
            "compactions": {"overlapped": bg.compactions, "phased": bg_p.compactions},
            "forward_status": {st: sum(r.forward_status == st for r in out) for st in {r.forward_status for r in out}},
            "forward_iteration_cap": args.adjoint_cap,
            "all_members_estimated_plain_seconds": est_all,
            "speedup_all_members": (len(ok) / t_batch) / max(len(ok) / est_all, 1e-300),
            "plain_cost_model": {"forward_s_per_iteration": t_fwd, "adjoint_s_per_iteration": t_adj,
                                 "fixed_s_per_member": fixed},
            "same_kernels": {"note": "every member one at a time with the batch's kernel variants instead of the "
                                     "single-solve (latency) ones, estimated the same way",
                             "forward_s_per_iteration": t_fwd_b, "adjoint_s_per_iteration": t_adj_b,
                             "all_members_estimated_plain_seconds": est_same,
                             "speedup_all_members": (len(ok) / t_batch) / max(len(ok) / est_same, 1e-300)}}


def vjp_micro(torch, n_members=64):
    """Adjoint-kernel microbenchmark (profiling): the batched-gradient bucket -- n_members bezier8 members,
    tri p = 2, refine 2, AUSM+-up, 2240 elements each -- after 50 batched forward steps; k_vjp per launch
    in product and RK4-stage modes beside the residual kernel, with a random adjoint state."""
    import ctypes as C

    ad, capi = pkg("adjoint"), pkg("capi")
    dc = ad.differentiable_case(contour="bezier8", area_ratio=2.5, order=2, refine=2, flux="ausmup",
                                back_pressure_ratio=0.15, tolerance=1e-10)
    members = bezier8_members(n_members)
    bg = ad.BatchGradient(dc, members, "thrust", names=tuple(members[0]))
    sv = pkg("batch").BatchSolver(bg.instances)
    sv.step_chunk(1, True)
    sv.step_chunk(50, False)
    dm, S0, ph = sv.meshes[0], sv.buffers[0][1][0], sv.phys[0]
    lib, st = capi.load(), torch.cuda.current_stream()
    gen = torch.Generator(device="cuda")
    gen.manual_seed(0)
    rnd = lambda: torch.randn(S0.shape, generator=gen, dtype=torch.float64, device="cuda")  # noqa: E731
    lam, seed, out = rnd(), rnd(), torch.empty_like(S0)
    lam0, f0, f1, f2 = lam.clone(), torch.zeros_like(S0), torch.zeros_like(S0), torch.zeros_like(S0)
    dt = torch.full((dm.E,), 1e-4, dtype=torch.float64, device="cuda")
    wave = torch.empty(dm.E, dtype=torch.float64, device="cuda")
    status = torch.zeros(n_members, dtype=torch.int32, device="cuda")
    mesh = capi.Mesh()
    C.memmove(C.byref(mesh), C.byref(dm.c), C.sizeof(capi.Mesh))
    mesh.inst_status = status.data_ptr()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timeit(fn, n=20):
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(n):
            ev[0].record(st)
            fn()
            ev[1].record(st)
            torch.cuda.synchronize()
            ts.append(ev[0].elapsed_time(ev[1]) * 1e3)
        return float(np.median(ts))

    res = {"workload": f"batched-gradient bucket: {n_members} bezier8 members, tri p=2 refine 2, {dm.E} elements, AUSM+-up",
           "unit": "us per launch"}
    a = capi.AdjointArgs()
    a.mode, a.U, a.lam, a.seed, a.out = capi.ADJ_VJP, S0.data_ptr(), lam.data_ptr(), seed.data_ptr(), out.data_ptr()
    res["k_vjp_product"] = timeit(lambda: capi.check(lib.nzb_vjp(C.byref(mesh), C.byref(ph), C.byref(a), st.cuda_stream), "nzb_vjp"))
    r = capi.AdjointArgs()
    r.mode, r.stage = capi.ADJ_RK4, 1
    r.U, r.lam, r.seed, r.out, r.lam0, r.dt = (t.data_ptr() for t in (S0, lam, seed, out, lam0, dt))
    r.f0, r.f1, r.f2 = f0.data_ptr(), f1.data_ptr(), f2.data_ptr()
    res["k_vjp_rk4_stage"] = timeit(lambda: capi.check(lib.nzb_vjp(C.byref(mesh), C.byref(ph), C.byref(r), st.cuda_stream), "nzb_vjp"))
    res["k_element_residual"] = timeit(lambda: capi.check(lib.nzb_residual(C.byref(mesh), C.byref(ph), 0, S0.data_ptr(), out.data_ptr(),
                                                                           wave.data_ptr(), st.cuda_stream), "nzb_residual"))
    return res


def run_ours(args, rank, world, torch, dist):
    capi = pkg("capi")
    BatchSolver = pkg("batch").BatchSolver
    peak, peak_kind = load_peaks()
    points, insts, index, refused = sweep_workload(args.max_iterations, args.points, rank, world)
    solver = BatchSolver(insts)
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    W = max(3, args.warmup)
    for _ in range(W):
        solver.reset()
        solver.run()
    ref_out = [(r.status, r.iterations) for r in solver.results(with_state=False)]

    times, launches = [], 0
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(torch.cuda.current_device()) as clk:
        for _ in range(args.steps):
            solver.reset()
            flush_l2(torch, flush)
            torch.cuda.synchronize()
            ev[0].record(st)
            solver.run()
            ev[1].record(st)
            torch.cuda.synchronize()
            times.append(ev[0].elapsed_time(ev[1]) * 1e-3)
            launches += solver.launches
    res = solver.results(with_state=False)
    if [(r.status, r.iterations) for r in res] != ref_out:
        raise RuntimeError("the batched sweep is not deterministic across repeats")
    if dist is not None:
        dist.barrier()
    n_conv = sum(r.converged for r in res)
    t_rank = float(np.sum(times))
    replicas = pkg("replicas")
    t_max = replicas.max_over_ranks(t_rank, dist, "cuda")
    # host-side gather of the ranks' tallies (no data-path collective)
    statuses = ("converged", "max_iterations", "stalled", "diverged", "non-finite", "running")
    tally = [n_conv, len(insts), len(refused), int(solver.n_elem)] + [sum(r.status == s for r in res) for s in statuses]
    tally = [int(round(v)) for v in replicas.sum_over_ranks(tally, dist, "cuda")]
    n_conv_all, n_built_all, n_refused_all, n_elem_all = tally[:4]
    value = replicas.whole_job_rate(n_conv_all * args.steps, t_max)
    outcomes = {s: n for s, n in zip(statuses, tally[4:]) if n}
    other = n_built_all - sum(tally[4:])
    if other:
        outcomes["other"] = other
    outcomes["refused"] = n_refused_all

    # end to end: set-up from host arrays, march, every state and status back
    # end to end from the design points: the host builds each case's topology, node coordinates and
    # quasi-1D solution (refusing the shocked points), the device its metric terms and initial state,
    # then the march, every status and each point's performance() metrics
    e2e_t, h2d, d2h = [], 0, 0
    for k in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        insts_k, _, _ = pkg("sweep").build_instances(points, max_iterations=args.max_iterations)
        sv = BatchSolver(insts_k)
        sv.run()
        out = sv.results(with_state=False)
        perf = sv.observables()
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if k > 0:
            e2e_t.append(t1 - t0)
        h2d = sv.h2d_bytes
        # statuses, iterations, residuals, the observable sums, and one 4-byte read per chunk
        d2h = (4 * 2 + 8 * 2) * len(out) + 8 * pkg("capi").NOBS * len(perf) + 4 * sv.chunks
        del sv
    e2e_value = replicas.whole_job_rate(n_conv_all, replicas.max_over_ranks(float(np.mean(e2e_t)), dist, "cuda"))

    # plain (one solve at a time) vs batched on the same subset
    sub = insts[:: args.plain_stride]
    p_times, p_conv, p_its = [], 0, []
    for inst in sub:
        bk, U0, scale = plain_solve(inst, torch)
        bk._S[0].copy_(U0)
        bk.run_device(1)  # warm: capture the 1-step and check-interval graphs
        bk.run_device(inst.opts.check_interval)
        torch.cuda.synchronize()
        ev[0].record(st)
        conv, its, _, _ = solve_device(bk, U0, inst.opts, scale, torch)
        ev[1].record(st)
        torch.cuda.synchronize()
        p_times.append(ev[0].elapsed_time(ev[1]) * 1e-3)
        p_conv += conv
        p_its.append(its)
        del bk
    sb = BatchSolver(sub)
    sb.run()
    sb.reset()
    torch.cuda.synchronize()
    ev[0].record(st)
    sb.run()
    ev[1].record(st)
    torch.cuda.synchronize()
    b_time = ev[0].elapsed_time(ev[1]) * 1e-3
    b_res = sb.results(with_state=False)
    b_conv = sum(r.converged for r in b_res)
    plain = {"instances": len(sub), "converged": int(p_conv), "plain_seconds": float(np.sum(p_times)),
             "batched_seconds": b_time, "plain_solves_per_s": p_conv / float(np.sum(p_times)),
             "batched_solves_per_s": b_conv / b_time, "speedup": float(np.sum(p_times)) / b_time,
             "subset": f"every {args.plain_stride}th built point",
             "iterations_match": [r.iterations for r in b_res] == p_its}

    # the whole sweep one solve at a time: a plain march's time is linear in its iterations, so each
    # (kind, order, mesh) class's cost per iteration (500 iterations of one member, with the march's
    # per-check read-back) times every instance's iteration count (the same in both paths)
    key = lambda inst: (inst.ops.ref.kind, inst.ops.ref.order, inst.ops.n_elem)  # noqa: E731
    first = {}
    for inst in insts:
        first.setdefault(key(inst), inst)
    def class_costs(variants):
        t_it = {}
        for k, inst in first.items():
            bk, U0, scale = plain_solve(inst, torch, variants)
            bk._S[0].copy_(U0)
            bk.run_device(1)
            bk.run_device(inst.opts.check_interval)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for _ in range(10):
                bk.run_device(inst.opts.check_interval)
                float(bk._res.item())
            torch.cuda.synchronize()
            t_it[k] = (time.perf_counter() - t0) / (10 * inst.opts.check_interval)
            del bk
        return t_it

    t_it = class_costs("single")
    t_same = class_costs("batch")
    est_all = float(sum(r.iterations * t_it[key(inst)] for inst, r in zip(insts, res)))
    est_same = float(sum(r.iterations * t_same[key(inst)] for inst, r in zip(insts, res)))
    est_sub = float(sum(it * t_it[key(inst)] for inst, it in zip(sub, p_its)))
    plain.update({"all_instances_estimated_plain_seconds": est_all,
                  "all_instances_batched_seconds": t_rank / args.steps,
                  "speedup_all_instances": est_all / (t_rank / args.steps),
                  "estimate_check": {"subset_estimated_seconds": est_sub, "subset_measured_seconds": float(np.sum(p_times))},
                  "same_kernels": {"note": "the plain path run with the batch's kernel variants instead of the "
                                           "single-solve (latency) ones",
                                   "all_instances_estimated_plain_seconds": est_same,
                                   "speedup_all_instances": est_same / (t_rank / args.steps)}})

    line = {
        "metric": "batched steady design-sweep solves/s at 1e-10 scaled residual (converged solves)",
        "value": value,
        "unit": "solves/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": W,
        "ms_per_step": 1e3 * t_max / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic: sampled operating points (seed 0) on the reference's own mesh generator and quasi-1D "
                "initial states, built on the host",
        "config": {"workload": sweep_workload_name(args.points * world, n_built_all, n_refused_all, args.max_iterations),
                   "elements": n_elem_all, "buckets_rank0": len(solver.meshes), "outcomes": outcomes,
                   "converged_per_step": n_conv_all, "l2": "flushed (256 MB write) before each sweep",
                   "tail_switch_iteration_rank0": solver.tail_switched_at,
                   "block_list_compactions_rank0": solver.compactions,
                   "parallelism": (f"sweep of {args.points * world} points partitioned over {world} GPUs "
                                   f"({args.points} each, points r::{world})" if world > 1 else "1 GPU")},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "path": "design points -> build_instances (host: topology, coordinates, quasi-1D) -> BatchSolver "
                        "(device: metric terms, initial states) -> run() -> results() + observables()"},
        "plain": plain,
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if rank == 0 and args.adjoint_members > 0:
        line["adjoint"] = adjoint_section(args, torch)
    if rank == 0 and not args.no_micro:
        mb = microbench(torch, capi, pkg("backend").B200Backend, pkg("config"), peak, peak_kind)
        line["roofline"] = mb.pop("roofline")
        line["microbench"] = mb
    if rank == 0:
        # the C port runs on the reference's full operators: one full case per (kind, order, mesh) class
        reps = {}
        for j, inst in enumerate(insts):
            reps.setdefault((inst.ops.ref.kind, inst.ops.ref.order, inst.ops.n_elem), j)
        full, _, _ = pkg("sweep").build_instances([points[index[j]] for j in reps.values()],
                                                  max_iterations=args.max_iterations, lean=False)
        cost, ncls = port_costs(full, args.cpu_seconds)
        cores = max(1, os.cpu_count() or 1)
        t_cpu = parallel_makespan(insts, [r.iterations for r in res], cost, cores)
        line["cpu_baseline"] = {
            "value": n_conv / t_cpu, "unit": "solves/s", "cores": cores, "kind": "port",
            "sample": f"the reference's compiled CPU step (its Numba backend restated in C, oracle/cpu_step.c): "
                      f"fused SSP-RK3 iterations timed on one member of each of the sweep's {ncls} (kind, order, "
                      f"mesh) classes (~{args.cpu_seconds:.0f} s in all, one thread), times every point's iteration "
                      f"count on the GPU, the points spread over {cores} cores one single-threaded march each "
                      f"(makespan)"}
    del solver
    return line


def sweep_workload_name(n_points, n_built, n_refused, max_iterations):
    """The workload string both arms report, so the driver sees one configuration."""
    return (f"design sweep: {n_points} points, {n_built} built, {n_refused} refused (shock in nozzle); tri/quad p 1-3 "
            f"refine 1-3, bell contour, HLLC, positivity limiter, tol 1e-10, cap {max_iterations} iterations")


def run_reference(args):
    """The reference's CPU path on the same sweep: its compiled step (the Numba backend restated in C,
    oracle/cpu_step.c), timed per mesh class with every host core busy, times the iteration count the
    reference solver itself took on each point (tests/golden/sweep_reference.json), the points spread over
    the cores one single-threaded march each; then two whole marches timed end to end to check that model."""
    path = os.path.join(GOLDEN, "sweep_reference.json")
    base = {"impl": "reference", "metric": "batched steady design-sweep solves/s at 1e-10 scaled residual (converged solves)"}
    if not os.path.exists(path):
        return {**base, "unavailable": "tests/golden/sweep_reference.json (the reference's sweep outcomes) is missing"}
    with open(path) as f:
        ref = json.load(f)
    points, insts, index, refused = sweep_workload(ref["max_iterations"], ref["n"], lean=False)
    rows = {r["point"]: r for r in ref["rows"]}
    its = [rows[k]["iterations"] for k in index]
    n_conv = sum(1 for k in index if rows[k].get("converged"))
    workers = max(1, os.cpu_count() or 1)
    ts = []
    for _ in range(args.warmup):
        port_costs_parallel(insts, 0.5, workers)
    for _ in range(args.steps):
        t0 = time.perf_counter()
        cost, ncls = port_costs_parallel(insts, args.cpu_seconds / max(1, args.steps), workers)
        ts.append(time.perf_counter() - t0)
    t_cpu = parallel_makespan(insts, its, cost, workers)
    value = n_conv / t_cpu
    # the model's check: the two cheapest converged points marched whole on the C port
    key = lambda inst: (inst.ops.ref.kind, inst.ops.ref.order, inst.ops.n_elem)  # noqa: E731
    conv = sorted((its[j] * cost[key(insts[j])], j) for j, k in enumerate(index) if rows[k].get("converged"))[:2]
    check = [{"point": int(index[j]), "iterations": int(its[j]), "modeled_s": float(m),
              "measured_s": port_solve_seconds(insts[j], its[j])} for m, j in conv]
    sample = (f"each step times the C port of the reference's compiled step (oracle/cpu_step.c; 1.11x the time of the "
              f"reference's own Numba backend per iteration, geometric mean over the sweep's classes, "
              f"oracle/numba_calibration.json) on one member of each of {ncls} mesh classes, {workers} at a time on "
              f"{workers} cores, one thread each; the sweep's CPU time is the makespan of every point's march (that "
              f"cost times the reference solver's own iteration count) spread over the {workers} cores")
    return {
        **base, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * float(np.mean(ts)), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic: sampled operating points (seed 0) on the reference's own mesh generator "
                                "and quasi-1D initial states, built on the host",
        "config": {"workload": sweep_workload_name(len(points), len(insts), len(refused), ref["max_iterations"]),
                   "reference_converged": n_conv, "sweep_cpu_seconds": t_cpu},
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": workers, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "model_check": check,
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--points", type=int, default=SWEEP_POINTS, help="operating points sampled for the sweep")
    ap.add_argument("--max-iterations", type=int, default=20000, help="iteration cap of every instance")
    ap.add_argument("--plain-stride", type=int, default=8, help="plain-vs-batched subset: every n-th built point")
    ap.add_argument("--no-micro", action="store_true")
    ap.add_argument("--adjoint-members", type=int, default=64, help="batched-gradient members (0: skip)")
    ap.add_argument("--adjoint-cap", type=int, default=100000, help="forward iteration cap of the gradient members")
    ap.add_argument("--cpu-seconds", type=float, default=18.0, help="seconds of CPU-baseline class timing")
    ap.add_argument("--micro-only", action="store_true", help="run only the residual microbench (profiling)")
    ap.add_argument("--micro-nx", type=int, default=1000, help="microbench cells along x (two triangles per cell)")
    ap.add_argument("--micro-nr", type=int, default=500, help="microbench cells across")
    ap.add_argument("--micro-kind", choices=("tri", "quad"), default="tri", help="microbench element kind (profiling)")
    ap.add_argument("--micro-order", type=int, default=3, help="microbench order (profiling)")
    ap.add_argument("--vjp-only", action="store_true", help="run only the adjoint-kernel microbench (profiling)")
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
    if args.vjp_only:
        print(json.dumps(vjp_micro(torch)))
        return
    if args.micro_only:
        peak, kind = load_peaks()
        print(json.dumps(microbench(torch, pkg("capi"), pkg("backend").B200Backend, pkg("config"), peak, kind,
                                    args.micro_nx, args.micro_nr, args.micro_kind, args.micro_order)))
        return
    line = run_ours(args, rank, world, torch, dist)
    if rank == 0:
        print(json.dumps(line))
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
