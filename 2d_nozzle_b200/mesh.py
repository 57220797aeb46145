"""Mesh connectivity: structured channel topology and generic edge matching.

The kernels take connectivity as plain integer arrays, so any conforming
single-kind mesh works.  The structured channel builder here exists so that a
run on a machine without the reference solver can still build the nozzle
channel and the unit-rectangle benchmark mesh *with the reference's numbering*
-- element order, node order, the owner rule and the boundary-edge order all
match src/geometry/mesh.py, which is what lets per-element results be compared
index for index:

* nodes ``j * n_ix + i`` (src/geometry/mesh.py:398-399);
* cells ``ci * ncy + cj``; for triangles every cell's lower-left triangle
  first, then every upper-right one (src/geometry/mesh.py:401-409,330-336);
* interior edges in order of their sorted (lo, hi) corner-node key, the lower
  element index owning the edge (src/geometry/mesh.py:121-151);
* boundary edges stably sorted by tag INFLOW=1, OUTFLOW=2, WALL=3, AXIS=4
  (src/geometry/mesh.py:34-40,163-176).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import refelem as re

INFLOW, OUTFLOW, WALL, AXIS = 1, 2, 3, 4
TAGS = (INFLOW, OUTFLOW, WALL, AXIS)


@dataclass(frozen=True)
class Edges:
    iedge_elem: np.ndarray
    iedge_face: np.ndarray
    bedge_elem: np.ndarray
    bedge_face: np.ndarray
    bedge_tag: np.ndarray
    face_edge: np.ndarray
    face_side: np.ndarray
    face_neighbour: np.ndarray
    tag_slices: dict = field(default_factory=dict)

    @property
    def n_interior(self) -> int:
        return int(self.iedge_elem.shape[0])

    @property
    def n_boundary(self) -> int:
        return int(self.bedge_elem.shape[0])


@dataclass(frozen=True)
class Topology:
    kind: str
    geometry_order: int
    elem_nodes: np.ndarray
    n_nodes: int
    edges: Edges
    logical: dict = field(default_factory=dict)

    @property
    def n_elem(self) -> int:
        return int(self.elem_nodes.shape[0])

    @property
    def n_faces(self) -> int:
        return re.n_faces(self.kind)

    def tag_slice(self, tag: int) -> slice:
        return self.edges.tag_slices.get(int(tag), slice(0, 0))


def match_edges(kind, elem_nodes, geometry_order, tagger, node_coords) -> Edges:
    """Pair element faces on their corner nodes and build the gather maps."""
    nface = re.n_faces(kind)
    corners = elem_nodes[:, list(re.vertex_node_ids(kind, geometry_order))]
    ne = corners.shape[0]
    va = np.empty((ne, nface), np.int64)
    vb = np.empty((ne, nface), np.int64)
    for f in range(nface):
        a, b = re.edge_vertices(kind, f)
        va[:, f], vb[:, f] = corners[:, a], corners[:, b]
    a_all, b_all = va.reshape(-1), vb.reshape(-1)
    owner_elem = np.repeat(np.arange(ne, dtype=np.int64), nface)
    owner_face = np.tile(np.arange(nface, dtype=np.int64), ne)
    lo, hi = np.minimum(a_all, b_all), np.maximum(a_all, b_all)
    perm = np.lexsort((hi, lo))
    slo, shi = lo[perm], hi[perm]
    dup = np.zeros(slo.size, bool)
    dup[:-1] = (slo[:-1] == slo[1:]) & (shi[:-1] == shi[1:])
    if np.any(dup[:-1] & dup[1:]):
        raise ValueError("non-conforming mesh: a face is shared by more than two elements")
    first = np.flatnonzero(dup)
    taken = np.zeros(slo.size, bool)
    taken[first] = True
    taken[first + 1] = True
    s0, s1 = perm[first], perm[first + 1]
    a_left = owner_elem[s0] <= owner_elem[s1]
    left = np.where(a_left, s0, s1)
    right = np.where(a_left, s1, s0)
    iedge_elem = np.stack([owner_elem[left], owner_elem[right]], axis=1)
    iedge_face = np.stack([owner_face[left], owner_face[right]], axis=1)

    bslot = perm[np.flatnonzero(~taken)]
    mid = 0.5 * (node_coords[a_all[bslot]] + node_coords[b_all[bslot]])
    tag = np.asarray(tagger(np.asarray(mid, float)), np.int64)
    order = np.argsort(tag, kind="stable")
    bslot, tag = bslot[order], tag[order]
    bedge_elem, bedge_face = owner_elem[bslot], owner_face[bslot]
    slices = {}
    for t in np.unique(tag):
        idx = np.flatnonzero(tag == t)
        slices[int(t)] = slice(int(idx[0]), int(idx[-1]) + 1)

    ni = iedge_elem.shape[0]
    face_edge = np.full((ne, nface), -1, np.int64)
    face_side = np.zeros((ne, nface), np.int64)
    face_edge[owner_elem[left], owner_face[left]] = np.arange(ni)
    face_edge[owner_elem[right], owner_face[right]] = np.arange(ni)
    face_side[owner_elem[right], owner_face[right]] = 1
    face_edge[bedge_elem, bedge_face] = ni + np.arange(bedge_elem.size)
    if np.any(face_edge < 0):
        raise ValueError("some element face matched no edge")
    nbr = np.repeat(np.arange(ne, dtype=np.int64)[:, None], nface, axis=1)
    nbr[iedge_elem[:, 0], iedge_face[:, 0]] = iedge_elem[:, 1]
    nbr[iedge_elem[:, 1], iedge_face[:, 1]] = iedge_elem[:, 0]
    return Edges(iedge_elem, iedge_face, bedge_elem, bedge_face, tag, face_edge, face_side, nbr, slices)


def channel_tagger(length: float, tol: float):
    """x=0 inflow, x=length outflow, y=0 axis, anything else wall."""

    def tag(mid):
        x, y = mid[:, 0], mid[:, 1]
        t = np.full(x.shape, WALL, np.int64)
        t[np.abs(y) < tol] = AXIS
        t[x < tol] = INFLOW
        t[x > length - tol] = OUTFLOW
        return t

    return tag


def _cell_offsets(kind: str, q: int) -> list[np.ndarray]:
    ref = re.lagrange_nodes(kind, q)
    if kind == "quad":
        return [np.rint(ref * q).astype(np.int64)]
    out = []
    for a, b, c in (((0, 0), (q, 0), (0, q)), ((q, 0), (q, q), (0, q))):
        a, b, c = (np.asarray(v, float) for v in (a, b, c))
        out.append(np.rint(a + ref[:, :1] * (b - a) + ref[:, 1:2] * (c - a)).astype(np.int64))
    return out


def channel_topology(kind="tri", *, nx=14, nr=5, refine=0, geometry_order=1):
    """Structured channel topology plus its logical grids ``(topo, x_frac, r_frac)``.

    Mirrors ``structured_nozzle_topology`` (src/geometry/mesh.py:361-439).
    """
    if kind not in re.KINDS:
        raise ValueError(f"unknown element kind {kind!r}")
    if refine < 0 or geometry_order < 1 or nx < 1 or nr < 1:
        raise ValueError("refine >= 0, geometry_order >= 1, nx, nr >= 1 required")
    q = geometry_order
    ncx, ncy = nx * 2**refine, nr * 2**refine
    n_ix, n_iy = q * ncx + 1, q * ncy + 1
    ci, cj = np.meshgrid(np.arange(ncx), np.arange(ncy), indexing="ij")
    bi, bj = (ci * q).reshape(-1), (cj * q).reshape(-1)
    elem_nodes = np.concatenate(
        [(bj[:, None] + off[None, :, 1]) * n_ix + (bi[:, None] + off[None, :, 0]) for off in _cell_offsets(kind, q)],
        axis=0,
    )
    x_frac = np.linspace(0.0, 1.0, n_ix)
    r_frac = np.linspace(0.0, 1.0, n_iy)
    probe = np.column_stack([np.tile(x_frac, n_iy), np.repeat(r_frac, n_ix)])
    tol = 0.25 / max(n_ix, n_iy)
    edges = match_edges(kind, elem_nodes, q, channel_tagger(1.0, tol), probe)
    logical = {"nx_cells": ncx, "nr_cells": ncy, "nx_nodes": n_ix, "nr_nodes": n_iy, "refine": refine}
    topo = Topology(kind, q, elem_nodes, n_ix * n_iy, edges, logical)
    return topo, x_frac, r_frac


def rectangle_coords(x_frac, r_frac, length=1.0, height=1.0) -> np.ndarray:
    """Node coordinates of the straight channel ``[0, length] x [0, height]``."""
    X = np.broadcast_to(np.asarray(x_frac)[None, :] * length, (len(r_frac), len(x_frac)))
    Y = np.broadcast_to(np.asarray(r_frac)[:, None] * height, (len(r_frac), len(x_frac)))
    return np.stack([X.reshape(-1), Y.reshape(-1)], axis=-1)


def channel_coords(x_frac, r_frac, wall_height, length=1.0) -> np.ndarray:
    """Node coordinates ``(x, r * y_wall(x))`` for a wall-height callable."""
    x = np.asarray(x_frac) * length
    yw = np.asarray(wall_height(x), float)
    X = np.broadcast_to(x[None, :], (len(r_frac), len(x_frac)))
    Y = np.asarray(r_frac)[:, None] * yw[None, :]
    return np.stack([X.reshape(-1), Y.reshape(-1)], axis=-1)
