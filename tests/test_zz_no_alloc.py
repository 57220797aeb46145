"""nzb_norm_noalloc -- the residual norm for callers that cannot allocate device memory.

A host application that hands this library only buffers from a fixed pool it
manages itself, or a loop that must never enter the CUDA allocator, cannot give
nzb_norm the scratch buffer it takes; nzb_norm_noalloc keeps its partial sums
in a fixed array inside the library instead.  These tests call both entry
points through the C ABI on the same device arrays and require the same
answer, twice in a row and across a change of size, and check that a size
beyond the fixed array is refused before anything is launched.

This file sorts last so that a run stopping at its first failure has already
run every other test.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import pkg

pytestmark = pytest.mark.gpu


def _norm_both(torch, lib, capi, E, np_, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    A = torch.randn(4 * np_ * E, generator=g, dtype=torch.float64).cuda()
    w = np.array([1.0, 1.336, 1.336, 1.786])
    stream = torch.cuda.current_stream().cuda_stream
    scratch = torch.zeros(int(lib.nzb_norm_blocks(E)) + 1, dtype=torch.float64, device="cuda")
    ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    capi.check(lib.nzb_norm(A.data_ptr(), E, np_, w.ctypes.data, scratch.data_ptr(), ref.data_ptr(), stream), "nzb_norm")
    got = torch.zeros(1, dtype=torch.float64, device="cuda")
    capi.check(lib.nzb_norm_noalloc(A.data_ptr(), E, np_, w.ctypes.data, got.data_ptr(), stream), "nzb_norm_noalloc")
    torch.cuda.synchronize()
    expect = float(np.sqrt(np.mean((A.cpu().numpy().reshape(4, np_ * E) * w[:, None]) ** 2)))
    return float(ref.item()), float(got.item()), expect


def test_noalloc_norm_matches_the_allocating_one(cuda):
    capi = pkg("capi")
    lib = capi.load()
    # a large call leaves many partial sums behind; the smaller calls after it
    # must not see them
    for E, np_, seed in ((200_000, 10, 1), (1000, 3, 2), (1000, 3, 2), (77, 16, 3)):
        ref, got, expect = _norm_both(cuda, lib, capi, E, np_, seed)
        assert got == ref, (E, got, ref)
        assert abs(got - expect) <= 1e-13 * expect


def test_noalloc_norm_at_its_largest_size(cuda):
    """n_elem = 8,388,608 fills every slot of the fixed array (np = 1: a 256 MB input)."""
    capi = pkg("capi")
    lib = capi.load()
    for _ in range(2):
        ref, got, expect = _norm_both(cuda, lib, capi, 8_388_608, 1, 4)
        assert got == ref, (got, ref)
        assert abs(got - expect) <= 1e-12 * expect
    cuda.cuda.empty_cache()


def test_noalloc_norm_refuses_an_oversized_mesh(cuda):
    capi = pkg("capi")
    lib = capi.load()
    out = cuda.zeros(1, dtype=cuda.float64, device="cuda")
    w = np.ones(4)
    # n_elem is checked before the array is touched, so a one-element array suffices
    A = cuda.zeros(4, dtype=cuda.float64, device="cuda")
    rc = lib.nzb_norm_noalloc(A.data_ptr(), 8_388_609, 1, w.ctypes.data, out.data_ptr(), ctypes.c_void_p(0))
    assert rc != 0
    assert b"exceeds its fixed scratch" in lib.nzb_last_error()


def test_noalloc_norm_inside_a_captured_graph(cuda):
    """After one call outside capture (which looks the fixed array's address up), the call can be
    captured into a CUDA graph: each replay takes the norm of the array's contents at that time."""
    torch = cuda
    capi = pkg("capi")
    lib = capi.load()
    E, np_ = 50_000, 6
    g = torch.Generator(device="cpu").manual_seed(5)
    A = torch.randn(4 * np_ * E, generator=g, dtype=torch.float64).cuda()
    w = np.array([1.0, 0.9, 0.9, 0.8])
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    capi.check(lib.nzb_norm_noalloc(A.data_ptr(), E, np_, w.ctypes.data, out.data_ptr(),
                                    torch.cuda.current_stream().cuda_stream), "nzb_norm_noalloc (warm-up)")
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.graph(graph, stream=side):
        capi.check(lib.nzb_norm_noalloc(A.data_ptr(), E, np_, w.ctypes.data, out.data_ptr(), side.cuda_stream),
                   "nzb_norm_noalloc (captured)")
    scratch = torch.zeros(int(lib.nzb_norm_blocks(E)) + 1, dtype=torch.float64, device="cuda")
    ref = torch.zeros(1, dtype=torch.float64, device="cuda")
    seen = set()
    for k in range(3):
        A.mul_(1.5)
        graph.replay()
        capi.check(lib.nzb_norm(A.data_ptr(), E, np_, w.ctypes.data, scratch.data_ptr(), ref.data_ptr(),
                                torch.cuda.current_stream().cuda_stream), "nzb_norm")
        torch.cuda.synchronize()
        assert float(out.item()) == float(ref.item()), k
        seen.add(float(out.item()))
    assert len(seen) == 3
    del graph
