"""Block lists: launches that span only the blocks holding running elements.

A batch late in its march lists the blocks that still hold elements of running
instances (``fwd_blocks`` / ``vjp_blocks`` of the mesh descriptor), so a launch
no longer walks every retired block.  The listed blocks run the same kernels on
the same elements, so every result is the same, bit for bit; an unlisted block
is left untouched.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import pkg

pytestmark = pytest.mark.gpu


def _case(element="tri", order=2, refine=1, pb=0.15):
    nz, cfg = pkg("nozzle"), pkg("config")
    opts = cfg.SolverOptions(tolerance=1e-8, max_iterations=6000, limiter="positivity", print_interval=0)
    flow = cfg.FlowConditions(flux="hllc", back_pressure_ratio=pb)
    return nz.build_case(element=element, order=order, refine=refine, area_ratio=2.5, contour="bell", flow=flow,
                         options=opts)


@pytest.mark.parametrize("variant", ["t1", "split4"])
@pytest.mark.parametrize("op", [0, 1])
def test_listed_blocks_match_and_others_are_untouched(cuda, variant, op, monkeypatch):
    import torch

    monkeypatch.setenv("NZB_VARIANT", variant)
    capi = pkg("capi")
    cs = _case()
    bk = pkg("backend").B200Backend(cs.operators, cs.flow, cs.options)
    lib, E, NP = bk.lib, bk.mesh.E, bk.mesh.np_
    src = bk.mesh.pack(cs.initial_state(), torch.empty(4 * NP * E, dtype=torch.float64, device="cuda"))
    stream = torch.cuda.current_stream().cuda_stream
    full = torch.zeros_like(src)
    wave_full = torch.zeros(E, dtype=torch.float64, device="cuda")
    capi.check(lib.nzb_residual(bk.mesh.c_ref, bk._phys_ref, op, src.data_ptr(), full.data_ptr(),
                                wave_full.data_ptr(), stream), "nzb_residual")
    W = int(lib.nzb_block_width(bk.mesh.c_ref, 0))
    n_blocks = (E + W - 1) // W
    listed = np.asarray(sorted({0, 2, n_blocks // 2, n_blocks - 1}), np.int32)
    blocks = torch.as_tensor(listed, device="cuda")
    mc = capi.Mesh()
    C.memmove(C.byref(mc), bk.mesh.c_ref, C.sizeof(capi.Mesh))
    mc.fwd_blocks, mc.n_fwd_blocks = blocks.data_ptr(), int(listed.size)
    out = torch.full_like(src, 12345.0)
    wave = torch.full((E,), -7.0, dtype=torch.float64, device="cuda")
    capi.check(lib.nzb_residual(C.byref(mc), bk._phys_ref, op, src.data_ptr(), out.data_ptr(), wave.data_ptr(),
                                stream), "nzb_residual (listed blocks)")
    torch.cuda.synchronize()
    on = np.zeros(E, bool)
    for b in listed:
        on[b * W:min((b + 1) * W, E)] = True
    got, ref = out.view(4, NP, E).cpu().numpy(), full.view(4, NP, E).cpu().numpy()
    assert np.array_equal(got[:, :, on], ref[:, :, on])
    assert np.all(got[:, :, ~on] == 12345.0)
    w, wf = wave.cpu().numpy(), wave_full.cpu().numpy()
    assert np.array_equal(w[on], wf[on])
    assert np.all(w[~on] == -7.0)


def test_block_list_bounds_are_checked(cuda):
    import torch

    capi = pkg("capi")
    cs = _case(order=1, refine=0)
    bk = pkg("backend").B200Backend(cs.operators, cs.flow, cs.options)
    lib, E, NP = bk.lib, bk.mesh.E, bk.mesh.np_
    n_blocks = int(lib.nzb_element_blocks(bk.mesh.c_ref))
    blocks = torch.arange(n_blocks + 1, dtype=torch.int32, device="cuda")
    mc = capi.Mesh()
    C.memmove(C.byref(mc), bk.mesh.c_ref, C.sizeof(capi.Mesh))
    mc.fwd_blocks, mc.n_fwd_blocks = blocks.data_ptr(), n_blocks + 1
    src = torch.zeros(4 * NP * E, dtype=torch.float64, device="cuda")
    out = torch.zeros_like(src)
    wave = torch.zeros(E, dtype=torch.float64, device="cuda")
    rc = lib.nzb_residual(C.byref(mc), bk._phys_ref, 0, src.data_ptr(), out.data_ptr(), wave.data_ptr(),
                          torch.cuda.current_stream().cuda_stream)
    assert rc != 0
    assert b"block count" in lib.nzb_last_error()


def _sweep_like():
    """Instances of uneven sizes and speeds in shared buckets: several retire well before the others."""
    batch = pkg("batch")
    out = []
    for el, p, r, pb in [("tri", 1, 1, 0.10), ("tri", 1, 0, 0.15), ("tri", 1, 0, 0.30), ("tri", 2, 0, 0.15),
                         ("tri", 2, 1, 0.20), ("quad", 1, 0, 0.15), ("quad", 1, 1, 0.12)]:
        cs = _case(el, p, r, pb)
        out.append(batch.Instance(cs.operators, cs.flow, cs.options, cs.initial_state(), cs.geometry.length,
                                  cs.geometry))
    return out


@pytest.mark.parametrize("variants", ["single", "batch"])
def test_compacted_batch_gives_the_same_bits(cuda, variants):
    batch = pkg("batch")
    insts = _sweep_like()
    runs = []
    for compact in (False, True):
        solver = batch.BatchSolver(insts, variants=variants, compact=compact)
        solver.run()
        runs.append((solver, solver.results()))
    (plain, a), (packed, b) = runs
    assert packed.compactions >= 1
    assert plain.compactions == (1 if plain.tail_switched_at is not None else 0)
    assert packed.tail_switched_at == plain.tail_switched_at
    for x, y in zip(a, b):
        assert (x.status, x.iterations) == (y.status, y.iterations)
        assert np.array_equal(x.U, y.U)
        assert x.residual == y.residual or (np.isnan(x.residual) and np.isnan(y.residual))


def test_compacted_batch_gradients_are_the_same(cuda):
    ad = pkg("adjoint")
    dc = ad.differentiable_case(contour="smooth", order=1, refine=0, back_pressure_ratio=0.15, tolerance=1e-11,
                                max_iterations=9000)
    members = [{"area_ratio": a, "throat_x": 0.1388} for a in (1.6, 2.0, 2.5, 3.2, 3.9)]
    got = []
    for compact in (False, True):
        bg = ad.BatchGradient(dc, members, "thrust", variants="single", compact=compact)
        got.append(bg.run(overlap=True))
        if compact:
            assert bg.compactions["adjoint"] + bg.compactions["forward"] >= 1
    for x, y in zip(*got):
        assert (x.forward_status, x.forward_iterations) == (y.forward_status, y.forward_iterations)
        assert (x.adjoint_converged, x.adjoint_iterations) == (y.adjoint_converged, y.adjoint_iterations)
        assert x.value == y.value or (np.isnan(x.value) and np.isnan(y.value))
        assert x.grad == y.grad


@pytest.mark.parametrize("variant", ["t1", "split4"])
def test_an_empty_block_list_launches_nothing(cuda, variant, monkeypatch):
    """A bucket whose instances have all retired lists no block: the residual leaves every output as it was."""
    import torch

    monkeypatch.setenv("NZB_VARIANT", variant)
    capi = pkg("capi")
    cs = _case(order=3, refine=0)
    bk = pkg("backend").B200Backend(cs.operators, cs.flow, cs.options)
    lib, E, NP = bk.lib, bk.mesh.E, bk.mesh.np_
    src = bk.mesh.pack(cs.initial_state(), torch.empty(4 * NP * E, dtype=torch.float64, device="cuda"))
    blocks = torch.zeros(1, dtype=torch.int32, device="cuda")
    mc = capi.Mesh()
    C.memmove(C.byref(mc), bk.mesh.c_ref, C.sizeof(capi.Mesh))
    mc.fwd_blocks, mc.n_fwd_blocks = blocks.data_ptr(), 0
    out = torch.full_like(src, 3.5)
    wave = torch.full((E,), -1.0, dtype=torch.float64, device="cuda")
    for op in (0, 1):
        capi.check(lib.nzb_residual(C.byref(mc), bk._phys_ref, op, src.data_ptr(), out.data_ptr(), wave.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream), "nzb_residual (empty list)")
    torch.cuda.synchronize()
    assert bool((out == 3.5).all()) and bool((wave == -1.0).all())
