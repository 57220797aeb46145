"""Launch variant per (element kind, order): fused face fluxes or a separate edge pass.

The element kernel can evaluate the face fluxes itself (each interior flux
from both sides, one thread per element) or take them from an edge pass (each
flux once, one thread per edge, then a lighter element kernel).  The two
evaluate the same formulas in the same order, but they are different kernels
and the compiler may contract multiply-adds differently in each, so their
results agree to round-off rather than bit for bit over a long march.  The
variant is therefore fixed per (kind, order) -- a single solve and a batch of
the same element type run the same kernels and give the same bits -- from the
table below, which :func:`measure` produces: one SSP-RK3 first stage (rate,
local step, update, limiter: the march's unit of work) timed both ways on a
mesh.  The table was measured on a B200 on the sampled design sweep's buckets
(19 000 - 68 000 elements): the edge pass wins for p = 1 (11 % for triangles,
9 % for quadrilaterals), the fused kernel for p = 2 and 3.
``NZB_EDGE_PASS=0/1`` in the environment forces a variant.
"""

from __future__ import annotations

import ctypes as C
import os

from . import capi

# (kind, order) -> edge pass on
EDGE_PASS = {
    ("tri", 0): False, ("tri", 1): True, ("tri", 2): False, ("tri", 3): False,
    ("quad", 0): False, ("quad", 1): True, ("quad", 2): False, ("quad", 3): False,
}


def choose_variant(mesh) -> bool:
    """Set ``mesh.edge_pass`` for its element type (the table, or ``NZB_EDGE_PASS``); returns it."""
    forced = (os.environ.get("NZB_EDGE_PASS") or "").strip()
    mesh.edge_pass = (forced == "1") if forced in ("0", "1") else EDGE_PASS.get((mesh.kind, mesh.order), False)
    return mesh.edge_pass


def measure(mesh, phys, state, reps: int = 5) -> dict:
    """Microseconds of one SSP-RK3 first stage on ``mesh`` with and without the edge pass.

    ``state`` is an admissible (4, NP, E) device state of the mesh.  The mesh's
    own setting is restored afterwards.
    """
    import torch

    lib = capi.load()
    out = torch.empty_like(state)
    dt = torch.empty(mesh.E, dtype=torch.float64, device=mesh.device)
    stream = torch.cuda.current_stream(mesh.device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    a = capi.StageArgs()
    a.V, a.out, a.dt = state.data_ptr(), out.data_ptr(), dt.data_ptr()
    a.dt_factor, a.a, a.b, a.stage = 0.1, 0.0, 1.0, 1
    keep = mesh.edge_pass
    best = {}
    for ep in (False, True):
        mesh.edge_pass = ep

        def once():
            capi.check(lib.nzb_stage(C.byref(mesh.c), C.byref(phys), C.byref(a), stream.cuda_stream), "nzb_stage")

        once()
        t = []
        for _ in range(reps):
            ev[0].record(stream)
            once()
            ev[1].record(stream)
            ev[1].synchronize()
            t.append(1e3 * ev[0].elapsed_time(ev[1]))
        best[ep] = min(t)
    mesh.edge_pass = keep
    return {"fused_us": best[False], "edge_pass_us": best[True]}
