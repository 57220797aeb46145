"""Launch variant per (element kind, order), measured and written to a table.

The forward kernels come in three variants:

* ``t1``       -- one thread per element, each interior flux evaluated from
                  both sides inside the element kernel;
* ``t1_edge``  -- one thread per element, the fluxes from a separate edge
                  pass (one thread per edge, each flux once);
* ``split4``   -- four threads per element (a block of four warps owns 32
                  elements: faces and volume points split over the warps, the
                  projection by component, the limiter's probe scan split).

They evaluate the same formulas and agree to round-off on a step (the
compiler contracts multiply-adds differently in different kernels, and
``split4`` associates a few sums differently).  The adjoint state kernel has
``t1`` and ``split4`` too.

Which is fastest depends on the context, so the table has two: ``single``
(one solve on its own mesh of a few thousand elements -- latency-bound, where
four threads per element shorten an element's path) and ``batch`` (a bucket
of a batch marching beside the other buckets -- throughput-bound, where one
thread per element wastes fewer instructions).  Within a context the variant
is fixed per (kind, order), never per mesh; a batch built with
``variants="single"`` runs the plain solve's kernels and gives its bits.

The table is ``variants.json`` beside this module, written by
``python -m 2d_nozzle_b200.autotune --write`` on a B200 (see :func:`tune`).
Without it the built-in defaults apply; ``NZB_VARIANTS_FILE`` names another
table.  ``NZB_VARIANT`` / ``NZB_VJP_VARIANT`` in the environment force one
forward / adjoint variant everywhere.
"""

from __future__ import annotations

import ctypes as C
import json
import os

from . import capi

VARIANTS = {
    "t1": {"split": 1, "edge_pass": False},
    "t1_edge": {"split": 1, "edge_pass": True},
    "split4": {"split": 4, "edge_pass": False},
}
ORDERS = (0, 1, 2, 3)
KINDS = ("tri", "quad")
TABLE_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "variants.json")

# used when variants.json is absent
DEFAULT = {("tri", 0): "t1", ("tri", 1): "t1_edge", ("tri", 2): "split4", ("tri", 3): "split4",
           ("quad", 0): "t1", ("quad", 1): "t1_edge", ("quad", 2): "split4", ("quad", 3): "split4"}


CONTEXTS = ("single", "batch")
# table keys per context: forward and adjoint variants
_KEYS = {("single", "fwd"): "choice", ("batch", "fwd"): "batch_choice",
         ("single", "vjp"): "vjp_choice", ("batch", "vjp"): "batch_vjp_choice"}


def table_path() -> str:
    """The variant table in use: ``NZB_VARIANTS_FILE`` when set (another measured table), else the one
    beside this module."""
    return os.environ.get("NZB_VARIANTS_FILE") or TABLE_PATH


def load_table(path: str | None = None, context: str = "single", which: str = "fwd") -> dict:
    """(kind, order) -> variant name for a context, from the measured table (or the defaults).  A table
    without the batch entries uses its single-solve ones for batches too."""
    if context not in CONTEXTS:
        raise ValueError(f"context {context!r}: use one of {CONTEXTS}")
    path = path or table_path()
    names = VARIANTS if which == "fwd" else VJP_VARIANTS
    table = dict(DEFAULT if which == "fwd" else VJP_DEFAULT)
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
        entries = data.get(_KEYS[(context, which)]) or data.get(_KEYS[("single", which)], {})
        for key, name in entries.items():
            kind, order = key.split(":")
            if name not in names:
                raise ValueError(f"{path}: unknown variant {name!r} for {key}")
            table[(kind, int(order))] = name
    return table


_TABLES: dict = {}


def _lookup(kind: str, order: int, context: str, which: str) -> str:
    key = (table_path(), context, which)
    if key not in _TABLES:
        _TABLES[key] = load_table(key[0], context, which)
    return _TABLES[key].get((kind, int(order)), "t1")


def variant_for(kind: str, order: int, context: str = "single") -> str:
    """The forward variant of (kind, order) in a context: ``single`` (one solve on its own mesh: latency)
    or ``batch`` (a bucket of a batch, its buckets side by side: throughput)."""
    forced = (os.environ.get("NZB_VARIANT") or "").strip()
    if forced:
        if forced not in VARIANTS:
            raise ValueError(f"NZB_VARIANT={forced!r}: use one of {sorted(VARIANTS)}")
        return forced
    name = _lookup(kind, order, context, "fwd")
    # four threads per element apply from p = 1 up
    return "t1" if (name == "split4" and int(order) == 0) else name


def apply_variant(mesh, name: str) -> None:
    v = VARIANTS[name]
    mesh.split = v["split"] if mesh.order > 0 else 1
    mesh.edge_pass = v["edge_pass"]


# The adjoint state kernel: one thread per element (``t1``) or four (``split4``),
# chosen per (kind, order) and context from the same table; NZB_VJP_VARIANT
# forces one.
VJP_VARIANTS = {"t1": 1, "split4": 4}
VJP_DEFAULT = {(k, p): "t1" for k in KINDS for p in ORDERS}


def vjp_variant_for(kind: str, order: int, context: str = "single") -> str:
    forced = (os.environ.get("NZB_VJP_VARIANT") or "").strip()
    if forced:
        if forced not in VJP_VARIANTS:
            raise ValueError(f"NZB_VJP_VARIANT={forced!r}: use one of {sorted(VJP_VARIANTS)}")
        name = forced
    else:
        name = _lookup(kind, order, context, "vjp")
    return "t1" if int(order) == 0 else name


def set_struct_variant(mc, kind: str, order: int, context: str) -> None:
    """The variant fields of a copied ``capi.Mesh`` struct (``split``, ``edge_pass``, ``vjp_split``) set for
    a context, as ``choose_variant`` sets a mesh's."""
    v = VARIANTS[variant_for(kind, order, context)]
    mc.split = v["split"] if order > 0 else 1
    mc.edge_pass = 1 if v["edge_pass"] else 0
    mc.vjp_split = VJP_VARIANTS[vjp_variant_for(kind, order, context)] if order > 0 else 1


def tail_elements() -> int:
    """Active elements below which a batch switches to the single-solve variants: with fewer, one thread
    (or four) per active element no longer fills a B200 (148 SMs x 8 resident warps of 32 threads at the
    one-thread kernels' 255 registers is 37 888), so latency, not throughput, decides.
    ``NZB_TAIL_ELEMENTS`` overrides; 0 turns the switch off."""
    return int(os.environ.get("NZB_TAIL_ELEMENTS", "32768"))


def context_for(n_elem: int, variants: str = "auto") -> str:
    """The variant context of one solve on a mesh of ``n_elem`` elements: ``auto`` takes the single-solve
    (latency) choice for a mesh too small to fill the GPU and the batch (throughput) choice for a larger
    one, with the same threshold as a batch's tail switch; ``single`` or ``batch`` forces one."""
    if variants == "auto":
        return "batch" if tail_elements() and n_elem > tail_elements() else "single"
    if variants not in CONTEXTS:
        raise ValueError(f"variants {variants!r}: use 'auto' or one of {CONTEXTS}")
    return variants


def choose_variant(mesh, context: str = "single") -> str:
    """Set ``mesh.split`` / ``mesh.edge_pass`` / ``mesh.vjp_split`` for its element type in a context
    (``single`` or ``batch``); returns the forward variant's name."""
    name = variant_for(mesh.kind, mesh.order, context)
    apply_variant(mesh, name)
    mesh.vjp_split = VJP_VARIANTS[vjp_variant_for(mesh.kind, mesh.order, context)]
    return name


def measure_vjp(mesh, phys, state, reps: int = 5) -> dict:
    """Microseconds of one adjoint RK4 stage (the march's unit of work: the transposed product, the rate
    and the stage update) on ``mesh`` for each adjoint variant (best of ``reps``); the mesh's own variant
    is restored afterwards."""
    import torch

    lib = capi.load()
    n = state.numel()
    lam, seed, out, f0, f1, f2 = (torch.zeros(n, dtype=torch.float64, device=mesh.device) for _ in range(6))
    seed.normal_(generator=torch.Generator(device=mesh.device).manual_seed(0))
    dt = torch.full((mesh.E,), 1e-3, dtype=torch.float64, device=mesh.device)
    a = capi.AdjointArgs()
    a.mode, a.stage = capi.ADJ_RK4, 1
    a.U, a.lam, a.seed, a.out = state.data_ptr(), seed.data_ptr(), seed.data_ptr(), out.data_ptr()
    a.lam0, a.dt, a.f0, a.f1, a.f2 = lam.data_ptr(), dt.data_ptr(), f0.data_ptr(), f1.data_ptr(), f2.data_ptr()
    stream = torch.cuda.current_stream(mesh.device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    keep = mesh.vjp_split
    res = {}
    for name, threads in VJP_VARIANTS.items():
        mesh.vjp_split = threads

        def run():
            capi.check(lib.nzb_vjp(C.byref(mesh.c), C.byref(phys), C.byref(a), stream.cuda_stream), "nzb_vjp")

        run()
        t = []
        for _ in range(reps):
            ev[0].record(stream)
            run()
            ev[1].record(stream)
            ev[1].synchronize()
            t.append(1e3 * ev[0].elapsed_time(ev[1]))
        res[name] = {"rk4_stage_us": min(t)}
    mesh.vjp_split = keep
    return res


def measure(mesh, phys, state, reps: int = 5, variants=None) -> dict:
    """Microseconds of one SSP-RK3 first and second stage on ``mesh`` for each variant.

    ``state`` is an admissible (4, NP, E) device state of the mesh.  The mesh's
    own variant is restored afterwards.  Returns {variant: {"stage1_us",
    "stage2_us", "total_us"}} (best of ``reps``).
    """
    import torch

    lib = capi.load()
    out = torch.empty_like(state)
    out2 = torch.empty_like(state)
    dt = torch.empty(mesh.E, dtype=torch.float64, device=mesh.device)
    stream = torch.cuda.current_stream(mesh.device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    a1, a2 = capi.StageArgs(), capi.StageArgs()
    a1.V, a1.out, a1.dt = state.data_ptr(), out.data_ptr(), dt.data_ptr()
    a1.dt_factor, a1.a, a1.b, a1.stage = 0.1, 0.0, 1.0, 1
    a2.V, a2.U0, a2.out, a2.dt = out.data_ptr(), state.data_ptr(), out2.data_ptr(), dt.data_ptr()
    a2.dt_factor, a2.a, a2.b, a2.stage = 0.1, 0.75, 0.25, 2
    keep = (mesh.split, mesh.edge_pass)
    names = [n for n in (variants or VARIANTS) if not (n == "split4" and mesh.order == 0)]
    res = {}
    for name in names:
        apply_variant(mesh, name)

        def stage(args):
            capi.check(lib.nzb_stage(C.byref(mesh.c), C.byref(phys), C.byref(args), stream.cuda_stream), "nzb_stage")

        stage(a1)
        stage(a2)
        best = {}
        for key, args in (("stage1_us", a1), ("stage2_us", a2)):
            t = []
            for _ in range(reps):
                if key == "stage2_us":
                    stage(a1)
                ev[0].record(stream)
                stage(args)
                ev[1].record(stream)
                ev[1].synchronize()
                t.append(1e3 * ev[0].elapsed_time(ev[1]))
            best[key] = min(t)
        best["total_us"] = best["stage1_us"] + best["stage2_us"]
        res[name] = best
    mesh.split, mesh.edge_pass = keep
    return res


def _sweep_buckets(device, max_points: int = 256):
    """The sampled design sweep's buckets: {(kind, order): (mesh, physics, state)}."""
    from .batch import BatchSolver
    from .sweep import build_instances, sample_points

    insts, _, _ = build_instances(sample_points(max_points, 0), max_iterations=10)
    bs = BatchSolver(insts, device=device)
    out = {}
    for dm, ph, U0 in zip(bs.meshes, bs.phys, bs.U0_soa):
        out[(dm.kind, dm.order)] = (dm, ph, U0)
    return bs, out


def random_states(n_elem: int, n_basis: int, gamma: float = 1.4, seed: int = 0):
    """(E, NP, 4) admissible states of the residual microbenchmark's distribution: per node density
    lognormal(0, 0.3), Mach U[0.2, 3] in a direction U[0, 2 pi), pressure lognormal(0, 0.5)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    shape = (n_elem, n_basis)
    rho = rng.lognormal(0.0, 0.3, shape)
    mach = rng.uniform(0.2, 3.0, shape)
    ang = rng.uniform(0.0, 2.0 * np.pi, shape)
    p = rng.lognormal(0.0, 0.5, shape)
    a = np.sqrt(gamma * p / rho)
    vx, vy = mach * a * np.cos(ang), mach * a * np.sin(ang)
    E = p / (gamma - 1.0) + 0.5 * rho * (vx * vx + vy * vy)
    return np.ascontiguousarray(np.stack([rho, rho * vx, rho * vy, E], -1))


def _rectangle(kind, order, n_elem_target, device):
    """A unit-rectangle mesh of about ``n_elem_target`` elements with random admissible states."""
    from .backend import B200Backend
    from .config import FlowConditions, SolverOptions
    from .mesh import channel_topology, rectangle_coords
    from .operators import build_operators

    per_cell = 2 if kind == "tri" else 1
    nr = max(2, int(round((n_elem_target / per_cell / 2) ** 0.5)))
    topo, xf, rf = channel_topology(kind, nx=2 * nr, nr=nr)
    ops = build_operators(topo, rectangle_coords(xf, rf), order, lean=True)
    bk = B200Backend(ops, FlowConditions(flux="hllc"), SolverOptions(cfl=0.5), device=device, device_metrics=True)
    state = bk.mesh.state()
    bk.mesh.pack(random_states(ops.n_elem, ops.ref.n_basis), state)
    return bk, state


def _single_meshes(device, max_points: int = 256):
    """One design-sweep instance per (kind, order, refine) on its own mesh, as a single solve runs it:
    {(kind, order): [(backend, state), ...]} (metric terms and initial state built on the device)."""
    from .backend import B200Backend
    from .sweep import build_instances, sample_points

    insts, _, _ = build_instances(sample_points(max_points, 0), max_iterations=10)
    seen, out = set(), {}
    for inst in insts:
        key = (inst.ops.ref.kind, inst.ops.ref.order, inst.ops.n_elem)
        if key in seen:
            continue
        seen.add(key)
        bk = B200Backend(inst.ops, inst.flow, inst.opts, device=device, device_metrics=True)
        out.setdefault(key[:2], []).append((bk, bk.initial_state(inst.geometry, host=False)))
    return out


def _batch_step_seconds(insts, table: dict, device, chunks: int = 3) -> float:
    """Seconds per step of the whole batch (every bucket marching side by side) with the forward variants
    of ``table`` ((kind, order) -> name): one warm chunk, then ``chunks`` timed chunks of the march's
    check interval."""
    import tempfile

    import torch

    from .batch import BatchSolver

    with tempfile.NamedTemporaryFile("w", suffix=".json", delete=False) as fh:
        json.dump({"batch_choice": {f"{k}:{o}": v for (k, o), v in table.items()}}, fh)
        path = fh.name
    old = os.environ.get("NZB_VARIANTS_FILE")
    os.environ["NZB_VARIANTS_FILE"] = path
    try:
        bs = BatchSolver(insts, device=device, variants="batch")
        n = bs.opts.check_interval
        bs.step_chunk(1, True)
        bs.step_chunk(n, False)
        st = torch.cuda.current_stream(device)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(st)
        for _ in range(chunks):
            bs.launch_chunk(n, False)
        ev[1].record(st)
        ev[1].synchronize()
        t = ev[0].elapsed_time(ev[1]) * 1e-3 / (chunks * n)
        del bs
        return t
    finally:
        if old is None:
            os.environ.pop("NZB_VARIANTS_FILE", None)
        else:
            os.environ["NZB_VARIANTS_FILE"] = old
        os.unlink(path)


def tune(device="cuda:0", reps: int = 5, grad_elements: int = 143_360) -> dict:
    """Measure the variants per (kind, order) in both contexts; returns the table document.

    * single solve (``choice``, ``vjp_choice``): one SSP-RK3 first and second stage and one adjoint RK4
      stage of every variant on one design-sweep instance per mesh size, each on its own mesh (a plain
      solve's latency);
    * batch (``batch_choice``): coordinate descent over the buckets' forward variants, each candidate
      timed as whole steps of the sampled 256-point sweep's batch (every bucket marching side by side:
      throughput); a change is kept when it saves more than 1 %;
    * batch adjoint (``batch_vjp_choice``): the adjoint RK4 stage on the sweep's bucket of that element
      type and on a unit rectangle of ``grad_elements`` elements (the batched gradients' bucket size).
    """
    import torch

    from .sweep import build_instances, sample_points

    doc = {"device": torch.cuda.get_device_name(device), "reps": reps, "measured": {}, "choice": {},
           "vjp_measured": {}, "vjp_choice": {}, "batch_measured": {}, "batch_choice": {},
           "batch_vjp_measured": {}, "batch_vjp_choice": {}}
    singles = _single_meshes(device)
    for (kind, order), meshes in sorted(singles.items()):
        if order == 0:
            continue
        key = f"{kind}:{order}"
        rows, vrows, tot, vtot = [], [], {}, {}
        for bk, st in meshes:
            m = measure(bk.mesh, bk.phys, st, reps)
            v = measure_vjp(bk.mesh, bk.phys, st, reps)
            rows.append({"elements": bk.mesh.E, "us": m})
            vrows.append({"elements": bk.mesh.E, "us": v})
            for name, t in m.items():
                tot[name] = tot.get(name, 0.0) + t["total_us"]
            for name, t in v.items():
                vtot[name] = vtot.get(name, 0.0) + t["rk4_stage_us"]
        doc["measured"][key], doc["choice"][key] = rows, min(tot, key=tot.get)
        doc["vjp_measured"][key], doc["vjp_choice"][key] = vrows, min(vtot, key=vtot.get)
    del singles
    torch.cuda.empty_cache()

    insts, _, _ = build_instances(sample_points(256, 0), max_iterations=20000)
    keys = sorted({(i.ops.ref.kind, i.ops.ref.order) for i in insts if i.ops.ref.order > 0})
    table = {(k, o): "t1" for k in KINDS for o in ORDERS}
    best = _batch_step_seconds(insts, table, device)
    trials = [{"table": {f"{k}:{o}": table[(k, o)] for k, o in keys}, "us_per_step": 1e6 * best}]
    for _ in range(2):
        changed = False
        for key in keys:
            for name in VARIANTS:
                if name == table[key]:
                    continue
                cand = dict(table)
                cand[key] = name
                t = _batch_step_seconds(insts, cand, device)
                trials.append({"table": {f"{k}:{o}": cand[(k, o)] for k, o in keys}, "us_per_step": 1e6 * t})
                if t < 0.99 * best:
                    best, table, changed = t, cand, True
        if not changed:
            break
    doc["batch_measured"] = {"workload": f"sampled 256-point sweep, {len(insts)} instances, whole-batch steps",
                             "trials": trials, "best_us_per_step": 1e6 * best}
    doc["batch_choice"] = {f"{k}:{o}": v for (k, o), v in sorted(table.items())}
    del insts
    torch.cuda.empty_cache()

    bs, buckets = _sweep_buckets(device)
    for (kind, order), (dm, ph, U0) in sorted(buckets.items()):
        if order == 0:
            continue
        key = f"{kind}:{order}"
        rows = {"sweep_bucket": {"elements": dm.E, "us": measure_vjp(dm, ph, U0, reps)}}
        bk, state = _rectangle(kind, order, grad_elements, device)
        rows["rectangle"] = {"elements": bk.mesh.E, "us": measure_vjp(bk.mesh, bk.phys, state, reps)}
        del bk, state
        vtot = {}
        for row in rows.values():
            for name, t in row["us"].items():
                vtot[name] = vtot.get(name, 0.0) + t["rk4_stage_us"]
        doc["batch_vjp_measured"][key], doc["batch_vjp_choice"][key] = rows, min(vtot, key=vtot.get)
    del bs
    for k in KINDS:
        for c in ("choice", "batch_choice"):
            doc[c][f"{k}:0"] = "t1"
    return doc


if __name__ == "__main__":
    import sys

    doc = tune()
    print(json.dumps(doc, indent=1))
    if "--write" in sys.argv:
        with open(TABLE_PATH, "w") as fh:
            json.dump(doc, fh, indent=1)
        print(f"wrote {TABLE_PATH}")
