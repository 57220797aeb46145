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
``split4`` associates a few sums differently).  Over a
long march round-off differences grow, so the variant is fixed per (kind,
order), never per mesh: a single solve and a batch of the same element type
run the same kernels and give the same bits.

The table is ``variants.json`` beside this module, written by
``python -m 2d_nozzle_b200.autotune --write`` on a B200: for every (kind,
order) it times an SSP-RK3 first and second stage (the march's unit of work:
rate, local step, update, limiter) of every variant on the sampled design
sweep's buckets of that element type and on a large unit-rectangle mesh with
random admissible states (the residual microbenchmark's distribution), and
keeps the variant with the least total time over those meshes.  Without the
file the built-in :data:`DEFAULT` applies; ``NZB_VARIANTS_FILE`` names another
table.  ``NZB_VARIANT`` in the environment (``t1``, ``t1_edge`` or ``split4``)
forces a variant.
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


def table_path() -> str:
    """The variant table in use: ``NZB_VARIANTS_FILE`` when set (another measured table), else the one
    beside this module."""
    return os.environ.get("NZB_VARIANTS_FILE") or TABLE_PATH


def load_table(path: str | None = None) -> dict:
    """(kind, order) -> variant name, from the measured table (or the default)."""
    path = path or table_path()
    table = dict(DEFAULT)
    if os.path.exists(path):
        with open(path) as fh:
            data = json.load(fh)
        for key, name in data.get("choice", {}).items():
            kind, order = key.split(":")
            if name not in VARIANTS:
                raise ValueError(f"{path}: unknown variant {name!r} for {key}")
            table[(kind, int(order))] = name
    return table


_TABLE = None


def variant_for(kind: str, order: int) -> str:
    forced = (os.environ.get("NZB_VARIANT") or "").strip()
    if forced:
        if forced not in VARIANTS:
            raise ValueError(f"NZB_VARIANT={forced!r}: use one of {sorted(VARIANTS)}")
        return forced
    global _TABLE
    if _TABLE is None:
        _TABLE = load_table()
    name = _TABLE.get((kind, int(order)), "t1")
    # four threads per element apply from p = 1 up
    return "t1" if (name == "split4" and int(order) == 0) else name


def apply_variant(mesh, name: str) -> None:
    v = VARIANTS[name]
    mesh.split = v["split"] if mesh.order > 0 else 1
    mesh.edge_pass = v["edge_pass"]


# The adjoint state kernel: one thread per element (``t1``) or four (``split4``),
# chosen per (kind, order) from the same table ("vjp_choice"; NZB_VJP_VARIANT
# forces one).
VJP_VARIANTS = {"t1": 1, "split4": 4}
VJP_DEFAULT = {(k, p): "t1" for k in KINDS for p in ORDERS}
_VJP_TABLE = None


def vjp_variant_for(kind: str, order: int) -> str:
    forced = (os.environ.get("NZB_VJP_VARIANT") or "").strip()
    if forced:
        if forced not in VJP_VARIANTS:
            raise ValueError(f"NZB_VJP_VARIANT={forced!r}: use one of {sorted(VJP_VARIANTS)}")
        name = forced
    else:
        global _VJP_TABLE
        if _VJP_TABLE is None:
            table = dict(VJP_DEFAULT)
            path = table_path()
            if os.path.exists(path):
                with open(path) as fh:
                    for key, nm in json.load(fh).get("vjp_choice", {}).items():
                        k, o = key.split(":")
                        if nm not in VJP_VARIANTS:
                            raise ValueError(f"{path}: unknown adjoint variant {nm!r} for {key}")
                        table[(k, int(o))] = nm
            _VJP_TABLE = table
        name = _VJP_TABLE.get((kind, int(order)), "t1")
    return "t1" if int(order) == 0 else name


def choose_variant(mesh) -> str:
    """Set ``mesh.split`` / ``mesh.edge_pass`` / ``mesh.vjp_split`` for its element type; returns the forward
    variant's name."""
    name = variant_for(mesh.kind, mesh.order)
    apply_variant(mesh, name)
    mesh.vjp_split = VJP_VARIANTS[vjp_variant_for(mesh.kind, mesh.order)]
    return name


def measure_vjp(mesh, phys, state, reps: int = 5) -> dict:
    """Microseconds of one adjoint RK4 stage (the march's unit of work: the transposed product, the rate
    and the stage update) on ``mesh`` for each adjoint variant (best of ``reps``); the mesh's own variant
    is restored afterwards."""
    import torch

    lib = capi.load()
    n = state.numel()
    bufs = [torch.zeros(n, dtype=torch.float64, device=mesh.device) for _ in range(6)]
    lam, seed, out, f0, f1, f2 = bufs
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


def tune(device="cuda:0", rect_elements: int = 200_000, reps: int = 5) -> dict:
    """Measure every variant per (kind, order); returns the table document."""
    import torch

    bs, buckets = _sweep_buckets(device)
    doc = {"device": torch.cuda.get_device_name(device), "rect_elements": rect_elements, "reps": reps,
           "measured": {}, "choice": {}}
    for kind in KINDS:
        for order in (1, 2, 3):
            key = f"{kind}:{order}"
            rows = {}
            if (kind, order) in buckets:
                dm, ph, U0 = buckets[(kind, order)]
                rows["sweep_bucket"] = {"elements": dm.E, "us": measure(dm, ph, U0, reps)}
            bk, state = _rectangle(kind, order, rect_elements, device)
            rows["rectangle"] = {"elements": bk.mesh.E, "us": measure(bk.mesh, bk.phys, state, reps)}
            del bk, state
            torch.cuda.empty_cache()
            total = {}
            for row in rows.values():
                for name, t in row["us"].items():
                    total[name] = total.get(name, 0.0) + t["total_us"]
            doc["measured"][key] = rows
            doc["choice"][key] = min(total, key=total.get)
            # the adjoint kernel on the same sweep bucket and on the gradient members' bucket shape
            vrows = {}
            if (kind, order) in buckets:
                dm, ph, U0 = buckets[(kind, order)]
                vrows["sweep_bucket"] = {"elements": dm.E, "us": measure_vjp(dm, ph, U0, reps)}
            vtotal = {}
            for row in vrows.values():
                for name, t in row["us"].items():
                    vtotal[name] = vtotal.get(name, 0.0) + t["rk4_stage_us"]
            doc.setdefault("vjp_measured", {})[key] = vrows
            if vtotal:
                doc.setdefault("vjp_choice", {})[key] = min(vtotal, key=vtotal.get)
    doc["choice"]["tri:0"] = "t1"
    doc["choice"]["quad:0"] = "t1"
    del bs
    return doc


if __name__ == "__main__":
    import sys

    doc = tune()
    print(json.dumps(doc, indent=1))
    if "--write" in sys.argv:
        with open(TABLE_PATH, "w") as fh:
            json.dump(doc, fh, indent=1)
        print(f"wrote {TABLE_PATH}")
