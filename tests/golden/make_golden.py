"""Generate the golden fixtures in this directory from the reference solver.

Run from the repository root with the reference importable as ``src``::

    PYTHONPATH=<reference checkout> python tests/golden/make_golden.py

Every array here comes from the reference's own code path (its NumPy backend
for per-stage values, its Numba backend for the long converged solve); nothing
is computed by this repository.  The fixtures pin both the CPU oracle and the
host-side mesh/operator builder, and the GPU tests compare against them.
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _save(name, **arrays):
    path = os.path.join(HERE, name)
    np.savez_compressed(path, **arrays)
    print(f"wrote {name}: {os.path.getsize(path) / 1024:.0f} KiB")


def ref_violates(U, ops, flow, fraction=1e-8):
    """The set of elements the reference's positivity limiter scales.

    Evaluated with the reference's own limiter helpers, in the order
    ``positivity_limiter`` uses them (src/spatial/limiter.py:216-228).  The
    limiter's output cannot be used for this: it rebuilds every element as
    ``ubar + theta (U - ubar)``, which moves unlimited ones by round-off.
    """
    from src.spatial import limiter as lim

    g = flow.gamma
    rho_floor, p_floor = lim.reference_floors(flow, fraction)
    U = lim.floor_cell_means(U, ops, flow, fraction=fraction)
    ubar = lim.cell_means(U, ops)
    probes = lim.probe_values(U, ops)
    p_bar = (g - 1.0) * (ubar[..., 3] - 0.5 * (ubar[..., 1] ** 2 + ubar[..., 2] ** 2) / ubar[..., 0])
    eps_rho = np.maximum(fraction * ubar[..., 0], 0.5 * rho_floor)
    eps_p = np.maximum(fraction * p_bar, 0.5 * p_floor)
    return (probes[..., 0].min(axis=1) < eps_rho) | (lim._pressure_at(probes, g, np).min(axis=1) < eps_p)


def _stage_record(bk, U, scheme):
    """One step of the reference base-class stepper, recording each stage."""
    F0, wave = bk.rate(U)
    dt = bk.time_step(wave)
    res = bk.norm(F0)
    stages = []

    def lim(V):
        stages.append(ref_violates(V, bk.ops, bk.flow))
        return bk.limit(V)

    if scheme == "euler":
        return lim(U + dt * F0), res, stages, wave, F0
    U1 = lim(U + dt * F0)
    F1, _ = bk.rate(U1)
    U2 = lim(0.75 * U + 0.25 * (U1 + dt * F1))
    F2, _ = bk.rate(U2)
    U3 = lim((1.0 / 3.0) * U + (2.0 / 3.0) * (U2 + dt * F2))
    return U3, res, stages, wave, F0


def random_state(n_elem, nbf, seed=0):
    rng = np.random.default_rng(seed)
    base = np.array([2.0, 0.6, 0.02, 5.0])
    return np.ascontiguousarray(base * (1.0 + 0.03 * rng.standard_normal((n_elem, nbf, 4))))


def microbench_state(n_elem, nbf, gamma=1.4, seed=0):
    """Per-node density lognormal(0,0.3), Mach U[0.2,3], random angle, p lognormal(0,0.5)."""
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


def operator_arrays(cs):
    ops = cs.operators
    ed = cs.topology.edges
    return dict(
        node_coords=np.asarray(cs.node_coords),
        elem_nodes=cs.topology.elem_nodes,
        face_edge=ed.face_edge,
        face_side=ed.face_side,
        iedge_elem=ed.iedge_elem,
        bedge_tag=ed.bedge_tag,
        grad_x_m=np.asarray(ops.grad_x_m),
        grad_y_m=np.asarray(ops.grad_y_m),
        face_basis_m=np.asarray(ops.face_basis_m),
        inv_mass=np.asarray(ops.inv_mass),
        edge_normal=np.asarray(ops.edge_normal),
        edge_jac=np.asarray(ops.edge_jac),
        edge_length=np.asarray(ops.edge_length),
        elem_area=np.asarray(ops.elem_area),
        mean_weights=np.asarray(ops.mean_weights),
    )


def per_flux(cs, U, fluxes=("roe", "hllc", "ausmup"), **flow_kw):
    from src.backends import get_backend
    from src.config import SolverOptions

    out = {}
    for name in fluxes:
        flow = cs.flow.replace(flux=name, **flow_kw)
        bk = get_backend("numpy", cs.operators, flow, SolverOptions(limiter="positivity"))
        R, wave = bk.residual(U)
        out[f"R_{name}"] = np.asarray(R)
        out[f"wave_{name}"] = np.asarray(wave)
        out[f"rate_{name}"] = -np.asarray(bk.inverse_mass(R))
    return out


def small_cases():
    from src.api import build_case
    from src.backends import get_backend
    from src.config import SolverOptions
    from src.spatial import limiter as lim

    for kind, orders in (("tri", (0, 1, 2, 3)), ("quad", (1, 2, 3))):
        for p in orders:
            cs = build_case(contour="smooth", element=kind, order=p, refine=0)
            ops = cs.operators
            U = random_state(ops.n_elem, ops.ref.n_basis)
            arrays = operator_arrays(cs)
            arrays["U"] = U
            arrays.update(per_flux(cs, U))
            arrays.update({k + "_backflow": v for k, v in per_flux(cs, U, ("roe",), backflow=True).items()})
            # a state with violations, for the limiter
            Ubad = U.copy()
            if p > 0:
                Ubad[3, 0, 0] = -0.5
                Ubad[7, 1, 3] = -1.0
                Ubad[11, :, 0] = -5.0
            arrays["U_bad"] = Ubad
            arrays["limited_bad"] = lim.positivity_limiter(Ubad, ops, cs.flow)
            # three steps of each scheme from the random state
            for scheme in ("euler", "ssprk3"):
                bk = get_backend("numpy", ops, cs.flow, SolverOptions(limiter="positivity", scheme=scheme))
                V, res = bk.run(U.copy(), 3, scheme)
                arrays[f"run3_{scheme}"] = np.asarray(V)
                arrays[f"run3_{scheme}_res"] = np.float64(res)
            _save(f"tiny_{kind}_p{p}.npz", **arrays)


GENERIC_CASES = (("tri", 4, 1), ("tri", 5, 1), ("quad", 4, 1), ("tri", 2, 2), ("tri", 3, 2), ("quad", 2, 2))


def generic_cases():
    """The tiny-mesh fixtures for orders above 3 and curved (Q = 2) elements, as small_cases makes them."""
    from src.api import build_case
    from src.backends import get_backend
    from src.config import SolverOptions
    from src.spatial import limiter as lim

    for kind, p, q in GENERIC_CASES:
        cs = build_case(contour="smooth", element=kind, order=p, refine=0, geometry_order=q)
        ops = cs.operators
        U = random_state(ops.n_elem, ops.ref.n_basis)
        # the operators' smaller arrays (the folded per-element ones follow from these)
        arrays = {k: v for k, v in operator_arrays(cs).items() if k not in ("grad_x_m", "grad_y_m", "face_basis_m")}
        arrays["U"] = U
        arrays.update(per_flux(cs, U))
        arrays.update({k + "_backflow": v for k, v in per_flux(cs, U, ("roe",), backflow=True).items()})
        Ubad = U.copy()
        Ubad[3, 0, 0] = -0.5
        Ubad[7, 1, 3] = -1.0
        Ubad[11, :, 0] = -5.0
        arrays["U_bad"] = Ubad
        arrays["limited_bad"] = lim.positivity_limiter(Ubad, ops, cs.flow)
        bk = get_backend("numpy", ops, cs.flow, SolverOptions(limiter="positivity", scheme="ssprk3"))
        V, res = bk.run(U.copy(), 3, "ssprk3")
        arrays["run3_ssprk3"] = np.asarray(V)
        arrays["run3_ssprk3_res"] = np.float64(res)
        _save(f"tiny_{kind}_p{p}_q{q}.npz", **arrays)


def generic_superbee_cases():
    """The Superbee slope limiter (then positivity) on the generic meshes: the fixture state with per-node
    jumps of up to 30 % (seed 7) and the TVB constant 0.5, so that most elements are limited; and three
    SSP-RK3 steps with it."""
    from src.api import build_case
    from src.backends import get_backend
    from src.config import SolverOptions
    from src.spatial import limiter as lim

    for kind, p, q in GENERIC_CASES:
        cs = build_case(contour="smooth", element=kind, order=p, refine=0, geometry_order=q)
        ops = cs.operators
        U = random_state(ops.n_elem, ops.ref.n_basis)
        rng = np.random.default_rng(7)
        U = U * (1.0 + 0.3 * rng.uniform(-1.0, 1.0, size=U.shape[:2])[..., None])
        arrays = {"U": U,
                  "superbee": lim.superbee_limiter(U, ops, cs.flow, tvb_constant=0.5),
                  "superbee_positivity": lim.apply_limiter(U, ops, cs.flow, "superbee", tvb_constant=0.5)}
        bk = get_backend("numpy", ops, cs.flow, SolverOptions(limiter="superbee", scheme="ssprk3", tvb_constant=0.5))
        V, res = bk.run(U.copy(), 3, "ssprk3")
        arrays["run3_ssprk3"] = np.asarray(V)
        arrays["run3_ssprk3_res"] = np.float64(res)
        _save(f"tiny_{kind}_p{p}_q{q}_superbee.npz", **arrays)


def superbee_cases():
    """The Superbee TVB slope limiter on a rough state of every tiny mesh, and three SSP-RK3 steps with it."""
    from src.api import build_case
    from src.backends import get_backend
    from src.config import SolverOptions
    from src.spatial import limiter as lim

    for kind, orders in (("tri", (1, 2, 3)), ("quad", (1, 2, 3))):
        for p in orders:
            cs = build_case(contour="smooth", element=kind, order=p, refine=0)
            ops = cs.operators
            rng = np.random.default_rng(3)
            base = np.array([2.0, 0.6, 0.02, 5.0])
            U = np.ascontiguousarray(base * (1.0 + 0.15 * rng.standard_normal((ops.n_elem, ops.ref.n_basis, 4))))
            arrays = {"U": U,
                      "superbee": lim.superbee_limiter(U, ops, cs.flow, tvb_constant=50.0),
                      "superbee_tvb0": lim.superbee_limiter(U, ops, cs.flow, tvb_constant=0.0),
                      "superbee_positivity": lim.apply_limiter(U, ops, cs.flow, "superbee", tvb_constant=50.0)}
            bk = get_backend("numpy", ops, cs.flow, SolverOptions(limiter="superbee", scheme="ssprk3"))
            V, res = bk.run(U.copy(), 3, "ssprk3")
            arrays["run3_ssprk3"] = np.asarray(V)
            arrays["run3_ssprk3_res"] = np.float64(res)
            _save(f"superbee_{kind}_p{p}.npz", **arrays)


def rectangle_microbench():
    """Config-2 distribution at 20x10 cells, cubic triangles, unit rectangle."""
    from src.backends import get_backend
    from src.config import FlowConditions, SolverOptions
    from src.geometry.mesh import structured_nozzle_topology
    from src.spatial.operators import build_operators

    topo, xf, rf = structured_nozzle_topology("tri", nx=20, nr=10)
    X, Y = np.meshgrid(xf, rf)
    coords = np.column_stack([X.ravel(), Y.ravel()])
    ops = build_operators(topo, coords, 3)
    U = microbench_state(ops.n_elem, ops.ref.n_basis)
    arrays = {"node_coords": coords, "U": U}
    for name in ("roe", "hllc", "ausmup"):
        flow = FlowConditions(flux=name)
        bk = get_backend("numpy", ops, flow, SolverOptions(limiter="positivity", cfl=0.5))
        R, wave = bk.residual(U)
        arrays[f"R_{name}"] = np.asarray(R)
        arrays[f"wave_{name}"] = np.asarray(wave)
        U3, res, stages, _, _ = _stage_record(bk, U.copy(), "ssprk3")
        arrays[f"step_{name}"] = U3
        arrays[f"step_{name}_res"] = np.float64(res)
        arrays[f"step_{name}_limited"] = np.stack(stages)
    _save("rect_tri_p3.npz", **arrays)


def config1():
    """Smooth contour, AR 2.5, p=1 triangles, refine 1, Roe, cfl 0.5, tol 1e-10."""
    from src.api import build_case, solve_nozzle
    from src.post.postprocess import performance
    from src.timestepping import initialize as ini

    kw = dict(contour="smooth", area_ratio=2.5, element="tri", order=1, refine=1, flux="roe", back_pressure_ratio=0.15)
    cs = build_case(**kw)
    U0 = ini.initial_state(cs.operators, cs.flow, cs.geometry, "quasi1d")
    res = solve_nozzle(case=cs, cfl=0.5, tolerance=1e-10, limiter="positivity", scheme="ssprk3", backend="numba", verbose=False)
    perf = performance(res)
    it, hist = res.history.as_arrays()
    _save(
        "config1.npz",
        node_coords=np.asarray(cs.node_coords),
        U0=np.asarray(U0),
        U_final=np.asarray(res.U),
        converged=np.bool_(res.converged),
        iterations=np.int64(res.iterations),
        residual=np.float64(res.residual),
        residual_scale=np.float64(res.residual_scale),
        history_iterations=it,
        history_residual=hist,
        thrust=np.float64(perf.thrust),
        mass_flow_in=np.float64(perf.mass_flow_in),
        exit_mach=np.float64(perf.exit_mach_area_averaged),
        throat_height=np.float64(cs.geometry.throat_height()),
        length=np.float64(cs.geometry.length),
    )


PERF_FIELDS = ("thrust", "thrust_wall", "thrust_imbalance", "thrust_coefficient", "mass_flow_in", "mass_flow_out",
               "mass_imbalance", "entropy_error", "exit_mach_area_averaged", "exit_pressure_ratio",
               "exit_temperature_ratio", "specific_thrust", "specific_thrust_ratio", "discharge_coefficient",
               "ideal_thrust", "thrust_efficiency")


def config1_q2():
    """Config 1 on curved (Q = 2) triangles: the same solve with quadratic geometry (refine 0)."""
    from src.api import build_case, solve_nozzle
    from src.post.postprocess import performance
    from src.timestepping import initialize as ini

    kw = dict(contour="smooth", area_ratio=2.5, element="tri", order=1, refine=0, geometry_order=2, flux="roe",
              back_pressure_ratio=0.15)
    cs = build_case(**kw)
    U0 = ini.initial_state(cs.operators, cs.flow, cs.geometry, "quasi1d")
    res = solve_nozzle(case=cs, cfl=0.5, tolerance=1e-10, limiter="positivity", scheme="ssprk3", backend="numba",
                       verbose=False)
    perf = performance(res)
    _save(
        "config1_q2.npz",
        node_coords=np.asarray(cs.node_coords),
        elem_nodes=np.asarray(cs.topology.elem_nodes),
        U0=np.asarray(U0),
        U_final=np.asarray(res.U),
        converged=np.bool_(res.converged),
        iterations=np.int64(res.iterations),
        residual=np.float64(res.residual),
        thrust=np.float64(perf.thrust),
        mass_flow_in=np.float64(perf.mass_flow_in),
        exit_mach=np.float64(perf.exit_mach_area_averaged),
    )


def observables():
    """The reference's performance() of the tiny cases' states and of config 1's converged state."""
    from types import SimpleNamespace

    from src.api import build_case
    from src.post.postprocess import performance

    def perf(cs, U):
        res = SimpleNamespace(operators=cs.operators, flow=cs.flow, U=U, geometry=cs.geometry)
        pf = performance(res)
        return {f: np.float64(getattr(pf, f)) for f in PERF_FIELDS}

    arrays = {}
    for kind, orders in (("tri", (0, 1, 2, 3)), ("quad", (1, 2, 3))):
        for p in orders:
            cs = build_case(contour="smooth", element=kind, order=p, refine=0)
            U = np.load(os.path.join(HERE, f"tiny_{kind}_p{p}.npz"))["U"]
            arrays.update({f"{kind}{p}_{k}": v for k, v in perf(cs, U).items()})
    cs = build_case(contour="smooth", area_ratio=2.5, element="tri", order=1, refine=1, flux="roe",
                    back_pressure_ratio=0.15)
    U = np.load(os.path.join(HERE, "config1.npz"))["U_final"]
    arrays.update({f"config1_{k}": v for k, v in perf(cs, U).items()})
    _save("observables.npz", **arrays)


def config3(n_steps=5):
    """Conical AR 3.0, p=3 quads, refine 3, HLLC, pb 0.6: fixed-step record."""
    from src.api import build_case
    from src.backends import get_backend
    from src.config import SolverOptions
    from src.timestepping import initialize as ini

    cs = build_case(contour="conical", area_ratio=3.0, element="quad", order=3, refine=3, flux="hllc",
                    back_pressure_ratio=0.6, allow_shock_in_nozzle=True)
    U0 = np.asarray(ini.initial_state(cs.operators, cs.flow, cs.geometry, "quasi1d"))
    bk = get_backend("numpy", cs.operators, cs.flow, SolverOptions(limiter="positivity", scheme="ssprk3"))
    U = U0.copy()
    ress, masks = [], []
    for _ in range(n_steps):
        U, res, stages, _, _ = _stage_record(bk, U, "ssprk3")
        ress.append(res)
        masks.extend(stages)
    _save("config3.npz", node_coords=np.asarray(cs.node_coords), U0=U0, U_final=U, res=np.asarray(ress),
          limited=np.stack(masks), n_steps=np.int64(n_steps))


BATCH_CASES = [  # element, order, refine, area ratio, back pressure, contour
    ("tri", 1, 0, 2.5, 0.15, "smooth"),
    ("quad", 1, 0, 3.0, 0.995, "bell"),
    ("tri", 2, 0, 1.8, 0.30, "conical"),
    ("tri", 1, 1, 2.2, 0.10, "bell"),
    ("quad", 2, 0, 2.5, 0.15, "bell"),
]


def batch_cases():
    """Outcomes of a few HLLC solves at tolerance 1e-8 (Numba backend)."""
    import json

    from src.api import solve_nozzle
    from src.post.postprocess import performance

    out = []
    for el, p, r, ar, pb, contour in BATCH_CASES:
        res = solve_nozzle(element=el, order=p, refine=r, area_ratio=ar, back_pressure_ratio=pb, contour=contour,
                           flux="hllc", tolerance=1e-8, max_iterations=6000, backend="numba", verbose=False)
        row = {"case": [el, p, r, ar, pb, contour], "converged": bool(res.converged), "iterations": int(res.iterations),
               "residual": float(res.residual), "message": res.message}
        if res.converged:
            perf = performance(res)
            row.update(thrust=perf.thrust, mass_flow_in=perf.mass_flow_in, exit_mach=perf.exit_mach_area_averaged)
        out.append(row)
    with open(os.path.join(HERE, "batch_cases.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote batch_cases.json")


CONTINUATION_CASES = [  # element, order, refine, area ratio, back pressure, contour, flux
    ("tri", 2, 0, 2.5, 0.15, "smooth", "roe"),
    ("tri", 3, 0, 2.0, 0.20, "bell", "hllc"),
    ("quad", 1, 0, 2.5, 0.15, "smooth", "hllc"),
]


def continuation_cases():
    """Solves with p-continuation (orders 0..p) at tolerance 1e-8, and the change_order projections."""
    import json

    from src.api import build_case, solve_nozzle
    from src.post.postprocess import performance
    from src.timestepping import initialize as ini

    out = []
    for el, p, r, ar, pb, contour, flux in CONTINUATION_CASES:
        res = solve_nozzle(element=el, order=p, refine=r, area_ratio=ar, back_pressure_ratio=pb, contour=contour,
                           flux=flux, tolerance=1e-8, max_iterations=30000, p_continuation=True, backend="numba",
                           verbose=False)
        row = {"case": [el, p, r, ar, pb, contour, flux], "converged": bool(res.converged),
               "iterations": int(res.iterations), "residual": float(res.residual), "message": res.message}
        if res.converged:
            perf = performance(res)
            row.update(thrust=perf.thrust, mass_flow_in=perf.mass_flow_in, exit_mach=perf.exit_mach_area_averaged)
        out.append(row)
    with open(os.path.join(HERE, "continuation_cases.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("wrote continuation_cases.json")
    # change_order of a quasi-1D state between every pair of orders (up and down)
    arrays = {}
    for kind in ("tri", "quad"):
        cs = {q: build_case(contour="smooth", element=kind, order=q, refine=0) for q in (0, 1, 2, 3)}
        for a in (0, 1, 2, 3):
            U = np.asarray(ini.initial_state(cs[a].operators, cs[a].flow, cs[a].geometry, "quasi1d"))
            arrays[f"{kind}_U{a}"] = U
            for b in (0, 1, 2, 3):
                if a != b:
                    arrays[f"{kind}_{a}to{b}"] = np.asarray(ini.change_order(U, cs[a].operators, cs[b].operators))
    _save("change_order.npz", **arrays)


def _sweep_point(args):
    """One design point through the reference's own solve (one Numba thread per worker)."""
    k, el, p, r, ar, pb, max_it = args
    import numba

    numba.set_num_threads(1)
    from src.api import solve_nozzle
    from src.post.postprocess import performance

    try:
        res = solve_nozzle(element=el, order=p, refine=r, area_ratio=ar, back_pressure_ratio=pb, flux="hllc",
                           tolerance=1e-10, max_iterations=max_it, limiter="positivity", backend="numba", verbose=False)
    except ValueError as exc:
        return {"point": k, "refused": True, "message": str(exc)[:80]}
    row = {"point": k, "refused": False, "converged": bool(res.converged), "iterations": int(res.iterations),
           "residual": float(res.residual), "message": res.message[:120]}
    if res.converged:
        perf = performance(res)
        row.update(thrust=perf.thrust, mass_flow_in=perf.mass_flow_in, exit_mach=perf.exit_mach_area_averaged)
    return row


def sweep_outcomes(n=256, seed=0, max_it=20000, workers=6):
    """The reference's outcome for every point of the sampled design sweep.

    The points come from the same sampler as the batched sweep (area ratio
    U[1.5, 4], back pressure U[0.1, 0.9], p in {1, 2, 3}, refine in {1, 2, 3},
    tri/quad 50/50, seed 0), each solved by the reference's solve_nozzle with
    HLLC, the positivity limiter, tolerance 1e-10 and an iteration cap.
    """
    import importlib
    import json
    from concurrent.futures import ProcessPoolExecutor

    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    pts = importlib.import_module("2d_nozzle_b200.sweep").sample_points(n, seed)
    jobs = [(k, pt.element, pt.order, pt.refine, pt.area_ratio, pt.back_pressure_ratio, max_it) for k, pt in enumerate(pts)]
    # the heaviest first, so the pool drains evenly
    jobs.sort(key=lambda j: -(4 ** j[3]) * (j[2] + 1) ** 2)
    with ProcessPoolExecutor(workers) as ex:
        rows = sorted(ex.map(_sweep_point, jobs), key=lambda r: r["point"])
    with open(os.path.join(HERE, "sweep_reference.json"), "w") as f:
        json.dump({"n": n, "seed": seed, "max_iterations": max_it, "rows": rows}, f, indent=0)
    print("wrote sweep_reference.json")



# the config-4 member whose gradient the GPU test checks: eight radial offsets,
# Gaussian with sigma = 2 % of the throat half-height (numpy default_rng(4))
CONFIG4 = dict(area_ratio=2.5, element="tri", order=2, refine=2, flux="ausmup", back_pressure_ratio=0.15)


def config4_offsets(sigma=0.02, seed=4):
    return np.random.default_rng(seed).normal(0.0, sigma, 8)


def config4_fd(h=1e-6, tol=1e-12):
    """Central differences of thrust w.r.t. the eight Bezier offsets of config 4, from the reference's solver.

    The reference has no eight-offset wall.  In this generator process only,
    its wall function is wrapped: for the smooth contour it returns the
    reference's own smooth wall plus y_throat * sum_k B_{9,k+1}(s) offset_k
    (degree-9 Bernstein polynomials of the diverging coordinate s, zero at both
    ends), which is the eight-offset family the repository builds.  Every
    forward solve is the reference's solve_nozzle (Numba backend) from its own
    quasi-1D initial state, to a scaled residual of ``tol``; thrust is the
    reference's objective (src/sensitivity.py:107-114): twice the outflow plus
    inflow axial momentum flux through its own boundary_trace.
    """
    import json
    import math

    import src.geometry.contour as contour_mod
    import src.geometry.mesh as mesh_mod
    from src.api import solve_nozzle
    from src.geometry.mesh import BoundaryTag
    from src.post.postprocess import axial_momentum_flux, boundary_trace

    orig = contour_mod.wall_half_height
    current = {"off": np.zeros(8)}

    def wall_bezier8(x, params, contour="bell", xp=np):
        y = orig(x, params, contour, xp=xp)
        if contour != "smooth":
            return y
        xi = xp.asarray(x) / params.get("length", 1.0)
        x_th = params["throat_x"]
        s = xp.clip((xi - x_th) / (1.0 - x_th), 0.0, 1.0)
        bump = sum(math.comb(9, k + 1) * s ** (k + 1) * (1.0 - s) ** (8 - k) * current["off"][k] for k in range(8))
        return y + params["throat_half_height"] * bump

    contour_mod.wall_half_height = wall_bezier8
    mesh_mod.wall_half_height = wall_bezier8

    def thrust(off):
        current["off"] = np.asarray(off, float)
        res = solve_nozzle(contour="smooth", tolerance=tol, max_iterations=400_000, backend="numba", verbose=False,
                           **CONFIG4)
        if not res.converged:
            raise RuntimeError(f"reference forward solve did not converge: {res.message}")
        gam = res.flow.gamma
        out = boundary_trace(res.U, res.operators, BoundaryTag.OUTFLOW)
        inl = boundary_trace(res.U, res.operators, BoundaryTag.INFLOW)
        return float(2.0 * (axial_momentum_flux(out, gam) + axial_momentum_flux(inl, gam))), int(res.iterations)

    base = config4_offsets()
    value, it0 = thrust(base)
    grad, iters = [], [it0]
    for k in range(8):
        up, dn = base.copy(), base.copy()
        up[k] += h
        dn[k] -= h
        tu, iu = thrust(up)
        td, idn = thrust(dn)
        grad.append((tu - td) / (2.0 * h))
        iters += [iu, idn]
        print(f"offset_{k}: {grad[-1]:.10e}")
    contour_mod.wall_half_height = orig
    mesh_mod.wall_half_height = orig
    doc = {"case": CONFIG4, "offsets": base.tolist(), "step": h, "tolerance": tol, "thrust": value,
           "gradient": grad, "iterations": iters}
    with open(os.path.join(HERE, "config4_fd.json"), "w") as f:
        json.dump(doc, f, indent=1)
    print("wrote config4_fd.json")

class _Recorder:
    """A reference backend behind a recording proxy: every attribute its caller reads and every method it
    calls, with the arguments and the results (arrays stored once, by identity or equality)."""

    def __init__(self, inner, log, arrays):
        self.__dict__.update(_inner=inner, _log=log, _arrays=arrays, _ids={})

    def _ref(self, v):
        if isinstance(v, np.ndarray):
            key = id(v)
            if key in self._ids and np.array_equal(self._arrays[self._ids[key]], v):
                return {"array": self._ids[key]}
            for name, a in self._arrays.items():
                if a.shape == v.shape and np.array_equal(a, v, equal_nan=True):
                    self._ids[key] = name
                    return {"array": name}
            name = f"a{len(self._arrays)}"
            self._arrays[name] = np.array(v, copy=True)
            self._ids[key] = name
            return {"array": name}
        if isinstance(v, (tuple, list)):
            return [self._ref(x) for x in v]
        if isinstance(v, (np.floating, np.integer, np.bool_)):
            return v.item()
        return v

    def __getattr__(self, name):
        val = getattr(self._inner, name)
        if callable(val):
            def call(*args, **kw):
                out = val(*args, **kw)
                self._log.append({"call": name, "args": self._ref(list(args)), "kw": {k: self._ref(v) for k, v in kw.items()},
                                  "out": self._ref(out)})
                return out
            return call
        self._log.append({"read": name, "value": self._ref(val)})
        return val


def drop_in_traces():
    """The reference's own solve_nozzle driving a recorded NumPy backend: the sequence of Backend calls
    its march makes (asarray, run chunks, limiter_activity, to_numpy, the counters), with every argument
    and result.  The GPU tests replay each call on the B200 backend and compare the answers."""
    import json

    import src.backends as backends
    from src.api import build_case, solve_nozzle
    from src.backends.numpy_backend import NumpyBackend

    cases = {
        "smooth_tri_p1_roe": dict(contour="smooth", area_ratio=2.5, element="tri", order=1, refine=0, flux="roe",
                                  back_pressure_ratio=0.15, max_iterations=400),
        "bell_quad_p2_hllc": dict(contour="bell", area_ratio=2.0, element="quad", order=2, refine=0, flux="hllc",
                                  back_pressure_ratio=0.1, max_iterations=250),
    }
    meta, arrays = {}, {}
    original = backends.get_backend
    try:
        for name, kw in cases.items():
            log, arr = [], {}

            def recorded(bname, ops, flow, opts, _log=log, _arr=arr):
                return _Recorder(NumpyBackend(ops, flow, opts), _log, _arr)

            backends.get_backend = recorded
            kw = dict(kw)
            max_it = kw.pop("max_iterations")
            cs = build_case(**kw)
            res = solve_nozzle(case=cs, cfl=0.5, tolerance=1e-10, limiter="positivity", scheme="ssprk3",
                               max_iterations=max_it, backend="numpy", verbose=False)
            meta[name] = {"case": {**kw, "max_iterations": max_it, "cfl": 0.5, "tolerance": 1e-10,
                                   "limiter": "positivity", "scheme": "ssprk3"},
                          "log": log, "iterations": int(res.iterations), "converged": bool(res.converged),
                          "residual": float(res.residual), "message": res.message}
            arrays.update({f"{name}/{k}": v for k, v in arr.items()})
    finally:
        backends.get_backend = original
    with open(os.path.join(HERE, "drop_in_traces.json"), "w") as fh:
        json.dump(meta, fh, indent=1)
    _save("drop_in_traces.npz", **arrays)


if __name__ == "__main__":
    import src  # noqa: F401  -- fails loudly when the reference is not on PYTHONPATH

    which = sys.argv[1:] or ["small", "rect", "config1", "config3", "batch"]
    if "small" in which:
        small_cases()
    if "rect" in which:
        rectangle_microbench()
    if "config1" in which:
        config1()
    if "config1_q2" in which:
        config1_q2()
    if "config3" in which:
        config3()
    if "batch" in which:
        batch_cases()
    if "sweep" in which:
        sweep_outcomes()
    if "superbee" in which:
        superbee_cases()
    if "observables" in which:
        observables()
    if "continuation" in which:
        continuation_cases()
    if "config4" in which:
        config4_fd()
    if "dropin" in which:
        drop_in_traces()
    if "generic" in which:
        generic_cases()
    if "generic_superbee" in which:
        generic_superbee_cases()
