"""Launch-variant autotuning: fused face fluxes or a separate edge pass, per mesh.

The element kernel can evaluate the face fluxes itself (each interior flux
from both sides, one thread per element) or take them from an edge pass (each
flux once, one thread per edge, then a lighter element kernel).  Both give
bit-identical results; which is faster depends on the element kind and order
(register pressure of the fused kernel) and on the mesh size (how well either
launch fills the GPU).  :func:`tune_edge_pass` times one rate evaluation each
way on the mesh it is given and keeps the faster, caching the answer per
(device, kind, order, geometry layout, element count).  ``NZB_EDGE_PASS=0/1``
in the environment forces a variant.
"""

from __future__ import annotations

import ctypes as C
import os

from . import capi

_cache: dict = {}


def tune_edge_pass(mesh, phys, state, reps: int = 3) -> bool:
    """Set ``mesh.edge_pass`` to the faster variant for this mesh; returns the choice.

    ``state`` is a (4, NP, E) device state the timing runs on (any admissible
    state of the mesh: the work does not depend on it beyond the limiter).
    """
    import torch

    forced = os.environ.get("NZB_EDGE_PASS")
    if forced in ("0", "1"):
        mesh.edge_pass = forced == "1"
        return mesh.edge_pass
    dev = mesh.device.index if mesh.device.index is not None else torch.cuda.current_device()
    key = (dev, mesh.kind, mesh.order, mesh.affine, mesh.E)
    if key not in _cache:
        lib = capi.load()
        out = torch.empty_like(state)
        wave = torch.empty(mesh.E, dtype=torch.float64, device=mesh.device)
        stream = torch.cuda.current_stream(mesh.device)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        best = {}
        for ep in (False, True):
            mesh.edge_pass = ep

            def once():
                capi.check(lib.nzb_residual(C.byref(mesh.c), C.byref(phys), 1, state.data_ptr(), out.data_ptr(),
                                            wave.data_ptr(), stream.cuda_stream), "nzb_residual")

            once()
            t = []
            for _ in range(reps):
                ev[0].record(stream)
                once()
                ev[1].record(stream)
                ev[1].synchronize()
                t.append(ev[0].elapsed_time(ev[1]))
            best[ep] = min(t)
        _cache[key] = best[True] < best[False]
    mesh.edge_pass = _cache[key]
    return mesh.edge_pass


def choices() -> dict:
    """The cached choices: (device, kind, order, affine, n_elem) -> edge pass on."""
    return dict(_cache)
