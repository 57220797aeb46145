"""Host side of the block lists: the block widths the library reports and the lists a batch builds."""

from __future__ import annotations

import ctypes as C

import numpy as np

from conftest import pkg


def _mesh(kind, order, split=1, vjp_split=1, n_elem=1000):
    m = pkg("capi").Mesh()
    m.kind, m.order, m.n_elem, m.split, m.vjp_split = kind, order, n_elem, split, vjp_split
    return m


def test_block_widths_follow_the_variant():
    lib = pkg("capi").load()
    for kind in (0, 1):
        for order in (1, 2, 3):
            one = _mesh(kind, order)
            split = _mesh(kind, order, split=4, vjp_split=4)
            bt = int(lib.nzb_block_width(C.byref(one), 0))
            assert bt in (64, 128)
            assert int(lib.nzb_block_width(C.byref(one), 1)) == bt
            assert int(lib.nzb_block_width(C.byref(split), 0)) == 32
            assert int(lib.nzb_block_width(C.byref(split), 1)) == 32
            assert int(lib.nzb_element_blocks(C.byref(one))) == (1000 + bt - 1) // bt
            assert int(lib.nzb_element_blocks(C.byref(split))) == (1000 + 31) // 32
    # order 0 has no four-thread kernel: the width stays one element per thread
    assert int(lib.nzb_block_width(C.byref(_mesh(0, 0, split=4)), 0)) == 128
    assert int(lib.nzb_block_width(None, 0)) == -1
    assert int(lib.nzb_block_width(C.byref(_mesh(0, 1)), 2)) == -1


def test_blocks_of_covers_exactly_the_running_ranges():
    blocks_of = pkg("batch").blocks_of
    assert blocks_of([], 32).size == 0
    assert blocks_of([(5, 5)], 32).size == 0
    got = blocks_of([(0, 40), (100, 129), (64, 65)], 32)
    assert got.dtype == np.int32
    assert got.tolist() == [0, 1, 2, 3, 4]
    got = blocks_of([(300, 301), (33, 64)], 32)
    assert got.tolist() == [1, 9]
    rng = np.random.default_rng(0)
    for _ in range(50):
        W = int(rng.choice([32, 64, 128]))
        edges = np.sort(rng.choice(5000, 12, replace=False))
        ranges = [(int(a), int(b)) for a, b in zip(edges[::2], edges[1::2]) if rng.random() < 0.6]
        got = set(blocks_of(ranges, W).tolist())
        want = {e // W for a, b in ranges for e in range(a, b)}
        assert got == want
