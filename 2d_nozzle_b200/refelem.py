"""Reference-element tables for the quadrature-based nodal DG discretisation.

The kernels never evaluate a basis function: every basis value, derivative and
quadrature weight they use is tabulated here once per (element kind, order) and
uploaded to constant memory.  The tables follow the reference solver's element
definitions exactly, because parity with it depends on evaluating the same
polynomials at the same points:

* equispaced Lagrange nodes, ``for iy: for ix`` row order, a centroid node at
  ``p = 0`` (src/reference/elements.py:56-75);
* triangle vertices (0,0),(1,0),(0,1) with local edge ``f`` opposite vertex
  ``f``; square vertices CCW with edge ``f`` from vertex ``f`` to ``f+1``
  (src/reference/elements.py:170-221);
* volume rules of degree ``2p+1+2(Q-1)`` and edge rules of degree ``2p+Q``,
  both at least ``2p+1`` on squares (src/reference/elements.py:224-241);
* positive-weight rules: Gauss-Legendre on [0,1], its tensor square, the
  one- and three-point symmetric triangle rules for degree <= 2, and the
  Duffy-collapsed Gauss-Jacobi(1,0) x Gauss-Legendre rule above that
  (src/reference/quadrature.py:48-144).

The attribute names of :class:`RefTables` match the reference's
``ReferenceData`` (src/spatial/operators.py:46-81) so that either object can be
handed to the device packer.
"""

from __future__ import annotations

from dataclasses import dataclass
from functools import lru_cache

import numpy as np

KINDS = ("tri", "quad")


def n_faces(kind: str) -> int:
    if kind == "tri":
        return 3
    if kind == "quad":
        return 4
    raise ValueError(f"unknown element kind {kind!r}; use one of {KINDS}")


def n_basis(kind: str, order: int) -> int:
    if order < 0:
        raise ValueError(f"order must be non-negative, got {order}")
    if kind == "tri":
        return (order + 1) * (order + 2) // 2
    if kind == "quad":
        return (order + 1) ** 2
    raise ValueError(f"unknown element kind {kind!r}; use one of {KINDS}")


def lagrange_nodes(kind: str, order: int) -> np.ndarray:
    """Node coordinates ``(n_basis, 2)`` in reference ordering."""
    if order == 0:
        return np.array([[1.0 / 3.0, 1.0 / 3.0]] if kind == "tri" else [[0.5, 0.5]])
    h = 1.0 / order
    rows = []
    for iy in range(order + 1):
        top = order - iy if kind == "tri" else order
        rows.extend((ix * h, iy * h) for ix in range(top + 1))
    return np.asarray(rows, dtype=float)


def _exponents(kind: str, order: int) -> list[tuple[int, int]]:
    if kind == "tri":
        return [(a, b) for b in range(order + 1) for a in range(order + 1 - b)]
    return [(a, b) for b in range(order + 1) for a in range(order + 1)]


@lru_cache(maxsize=32)
def _coeff(kind: str, order: int) -> np.ndarray:
    """Monomial coefficients ``C`` with ``phi_j(x) = sum_k C[k, j] m_k(x)``."""
    nodes = lagrange_nodes(kind, order)
    ex = _exponents(kind, order)
    V = np.array([[x**a * y**b for (a, b) in ex] for (x, y) in nodes])
    return np.linalg.solve(V, np.eye(len(ex)))


def basis(kind: str, order: int, pts: np.ndarray):
    """``(phi, dphi/dxi, dphi/deta)``, each ``(n_basis, npts)``, at reference points."""
    pts = np.atleast_2d(np.asarray(pts, dtype=float))
    npts = pts.shape[0]
    if order == 0:
        return np.ones((1, npts)), np.zeros((1, npts)), np.zeros((1, npts))
    C = _coeff(kind, order)
    ex = _exponents(kind, order)
    xi, eta = pts[:, 0], pts[:, 1]
    nb = len(ex)
    phi = np.zeros((nb, npts))
    dxi = np.zeros((nb, npts))
    deta = np.zeros((nb, npts))
    for k, (a, b) in enumerate(ex):
        c = C[k, :][:, None]
        phi += c * (xi**a * eta**b)[None, :]
        if a:
            dxi += (c * a) * (xi ** (a - 1) * eta**b)[None, :]
        if b:
            deta += (c * b) * (xi**a * eta ** (b - 1))[None, :]
    return phi, dxi, deta


# ---- edges ---------------------------------------------------------------
_TRI_EDGE = {0: ((1.0, 0.0), (-1.0, 1.0)), 1: ((0.0, 1.0), (0.0, -1.0)), 2: ((0.0, 0.0), (1.0, 0.0))}
_QUAD_EDGE = {
    0: ((0.0, 0.0), (1.0, 0.0)),
    1: ((1.0, 0.0), (0.0, 1.0)),
    2: ((1.0, 1.0), (-1.0, 0.0)),
    3: ((0.0, 1.0), (0.0, -1.0)),
}


def edge_start_and_direction(kind: str, f: int):
    """``(start vertex, d(xi,eta)/dsigma)`` of local edge ``f``."""
    table = _TRI_EDGE if kind == "tri" else _QUAD_EDGE
    return table[f]


def edge_points(kind: str, f: int, sigma: np.ndarray) -> np.ndarray:
    (x0, y0), (dx, dy) = edge_start_and_direction(kind, f)
    s = np.asarray(sigma, dtype=float).ravel()
    # written as the reference's (1 - s) style expressions so values coincide
    if kind == "tri":
        cols = {0: (1.0 - s, s), 1: (np.zeros_like(s), 1.0 - s), 2: (s, np.zeros_like(s))}[f]
    else:
        one, zero = np.ones_like(s), np.zeros_like(s)
        cols = {0: (s, zero), 1: (one, s), 2: (1.0 - s, one), 3: (zero, 1.0 - s)}[f]
    return np.column_stack(cols)


def edge_vertices(kind: str, f: int) -> tuple[int, int]:
    """Local vertex ids (CCW) at the start and end of edge ``f``."""
    if kind == "tri":
        return ((f + 1) % 3, (f + 2) % 3)
    return (f, (f + 1) % 4)


def vertex_node_ids(kind: str, order: int) -> tuple[int, ...]:
    """Positions of the element vertices within the order-``order`` node list."""
    if kind == "tri":
        return (0, order, n_basis("tri", order) - 1)
    q = order
    return (0, q, (q + 1) * q + q, (q + 1) * q)


def edge_node_ids(kind: str, order: int, f: int) -> list[int]:
    """Nodes lying on edge ``f``, ordered from its start vertex to its end vertex.

    A Lagrange basis restricted to an edge depends only on these ``p + 1``
    nodes; the kernels use that to form traces from a quarter of the
    coefficients.
    """
    if order == 0:
        return [0]
    nodes = lagrange_nodes(kind, order)
    (x0, y0), (dx, dy) = edge_start_and_direction(kind, f)
    out = []
    for j in range(order + 1):
        t = j / order
        target = np.array([x0 + t * dx, y0 + t * dy])
        out.append(int(np.argmin(np.abs(nodes - target).sum(axis=1))))
    return out


# ---- quadrature ------------------------------------------------------------
def _n_gauss(degree: int) -> int:
    return max(1, (degree + 2) // 2)


@lru_cache(maxsize=64)
def gauss_legendre(degree: int) -> tuple[np.ndarray, np.ndarray]:
    """Points and weights on [0, 1], exact to ``degree``."""
    x, w = np.polynomial.legendre.leggauss(_n_gauss(degree))
    return 0.5 * (x + 1.0), 0.5 * w


def square_rule(degree: int):
    x, w = gauss_legendre(degree)
    X, Y = np.meshgrid(x, x, indexing="ij")
    return np.column_stack([X.ravel(), Y.ravel()]), np.outer(w, w).ravel()


def triangle_rule(degree: int):
    if degree <= 1:
        return np.array([[1.0 / 3.0, 1.0 / 3.0]]), np.array([0.5])
    if degree == 2:
        a, b = 1.0 / 6.0, 2.0 / 3.0
        return np.array([[a, a], [b, a], [a, b]]), np.full(3, 1.0 / 6.0)
    from scipy.special import roots_jacobi

    n = _n_gauss(degree)
    t, wj = roots_jacobi(n, 1.0, 0.0)
    x = 0.5 * (t + 1.0)
    wx = wj / 4.0
    y, wy = gauss_legendre(degree)
    X, Y = np.meshgrid(x, y, indexing="ij")
    pts = np.column_stack([X.ravel(), ((1.0 - X) * Y).ravel()])
    return pts, np.outer(wx, wy).ravel()


def quadrature_degrees(kind: str, order: int, geometry_order: int = 1) -> tuple[int, int]:
    vol = 2 * order + 1 + 2 * (geometry_order - 1)
    edge = 2 * order + geometry_order
    if kind == "quad":
        vol = max(vol, 2 * order + 1)
        edge = max(edge, 2 * order + 1)
    return vol, edge


@dataclass(frozen=True)
class RefTables:
    """Mesh-independent tables for one (kind, order, geometry order)."""

    kind: str
    order: int
    geometry_order: int
    n_basis: int
    n_basis_geom: int
    points_vol: np.ndarray
    w_vol: np.ndarray
    phi_vol: np.ndarray
    dphi_dxi_vol: np.ndarray
    dphi_deta_vol: np.ndarray
    dgeom_dxi_vol: np.ndarray
    dgeom_deta_vol: np.ndarray
    geom_vol: np.ndarray
    w_face: np.ndarray
    phi_face: np.ndarray  # (2, nface, nbf, nqf): side 0 walks sigma, side 1 walks 1 - sigma
    geom_face: np.ndarray
    dgeom_dsigma_face: np.ndarray

    @property
    def n_qvol(self) -> int:
        return int(self.w_vol.size)

    @property
    def n_qface(self) -> int:
        return int(self.w_face.size)

    @property
    def n_faces(self) -> int:
        return n_faces(self.kind)


@lru_cache(maxsize=32)
def ref_tables(kind: str, order: int, geometry_order: int = 1) -> RefTables:
    dv, df = quadrature_degrees(kind, order, geometry_order)
    pts, wv = (triangle_rule if kind == "tri" else square_rule)(dv)
    sig, wf = gauss_legendre(df)
    nf = n_faces(kind)
    phi, dxi, deta = basis(kind, order, pts)
    g, gdxi, gdeta = basis(kind, geometry_order, pts)
    nbf, nbq, nq = n_basis(kind, order), n_basis(kind, geometry_order), sig.size
    phi_face = np.zeros((2, nf, nbf, nq))
    geom_face = np.zeros((nf, nbq, nq))
    dgeom = np.zeros((nf, nbq, nq))
    for f in range(nf):
        _, (ds_xi, ds_eta) = edge_start_and_direction(kind, f)
        phi_face[0, f] = basis(kind, order, edge_points(kind, f, sig))[0]
        phi_face[1, f] = basis(kind, order, edge_points(kind, f, 1.0 - sig))[0]
        gf, gfx, gfy = basis(kind, geometry_order, edge_points(kind, f, sig))
        geom_face[f] = gf
        dgeom[f] = gfx * ds_xi + gfy * ds_eta
    return RefTables(
        kind=kind,
        order=order,
        geometry_order=geometry_order,
        n_basis=nbf,
        n_basis_geom=nbq,
        points_vol=pts,
        w_vol=wv,
        phi_vol=phi,
        dphi_dxi_vol=dxi,
        dphi_deta_vol=deta,
        dgeom_dxi_vol=gdxi,
        dgeom_deta_vol=gdeta,
        geom_vol=g,
        w_face=wf,
        phi_face=phi_face,
        geom_face=geom_face,
        dgeom_dsigma_face=dgeom,
    )
