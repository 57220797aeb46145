// shapes.cuh -- compile-time element shapes and the constant-memory table layout.
//
// Sizes follow the reference element definitions (src/reference/elements.py:45-53,
// 224-241; src/reference/quadrature.py:48-144): NP Lagrange nodes, NQV volume
// points (1 / 3 / n*n collapsed rule on triangles, n*n Gauss on squares), NQF
// Gauss points per edge, NE = p + 1 nodes on each edge.
#pragma once
#include <stdint.h>

namespace nzb {

constexpr int MAX_ORDER = 3;

__host__ __device__ constexpr int n_basis(int kind, int p) { return kind == 0 ? (p + 1) * (p + 2) / 2 : (p + 1) * (p + 1); }
__host__ __device__ constexpr int n_faces(int kind) { return kind == 0 ? 3 : 4; }
__host__ __device__ constexpr int gauss_n(int degree) { return (degree + 2) / 2 < 1 ? 1 : (degree + 2) / 2; }
__host__ __device__ constexpr int n_qvol(int kind, int p) {
  return kind == 0 ? ((2 * p + 1) <= 1 ? 1 : ((2 * p + 1) == 2 ? 3 : gauss_n(2 * p + 1) * gauss_n(2 * p + 1)))
                   : gauss_n(2 * p + 1) * gauss_n(2 * p + 1);
}
__host__ __device__ constexpr int n_qface(int, int p) { return gauss_n(2 * p + 1); }
__host__ __device__ constexpr int n_edge_nodes(int p) { return p + 1; }

// Table slot of one (kind, p), in doubles:
//   PHI [NP][NQV]   basis at volume points
//   WXI [NP][NQV]   w_q * dphi/dxi          (unfolded weak-form gradient tables)
//   WETA[NP][NQV]   w_q * dphi/deta
//   MINV[NP][NP]    inverse of the reference mass matrix sum_q w phi_i phi_j
//   E1D [NE][NQF]   1D Lagrange basis of the edge nodes at the edge Gauss points
//   WF  [NQF]       edge Gauss weights
//   MW  [NP]        cell-average weights sum_q phi_i w_q / sum_q w_q
//   WV  [NQV]       volume weights
//   DGX [NV][NQV]   d(vertex shape function)/dxi at the volume points (NV = NF)
//   DGE [NV][NQV]   d(vertex shape function)/deta
//   PFE [2][NF][NE][NQF]  the reference's face basis phi_face[side, f, i, q]
//                   at the edge nodes i = edge_node(f, j)
//   GV  [NV][NQV]   vertex shape functions at the volume points (the initial
//                   state's point coordinates)
__host__ __device__ constexpr int slot_size(int kind, int p) {
  return 3 * n_basis(kind, p) * n_qvol(kind, p) + n_basis(kind, p) * n_basis(kind, p) +
         n_edge_nodes(p) * n_qface(kind, p) + n_qface(kind, p) + n_basis(kind, p) + n_qvol(kind, p) +
         2 * n_faces(kind) * n_qvol(kind, p) + 2 * n_faces(kind) * n_edge_nodes(p) * n_qface(kind, p) +
         n_faces(kind) * n_qvol(kind, p);
}
__host__ __device__ constexpr int slot_offset(int kind, int p) {
  int off = 0;
  for (int k = 0; k < 2; ++k)
    for (int q = 0; q <= MAX_ORDER; ++q) {
      if (k == kind && q == p) return off;
      off += slot_size(k, q);
    }
  return off;
}
constexpr int TABLE_DOUBLES = slot_offset(2, 0);

template <int K, int P>
struct Shape {
  static constexpr int NP = n_basis(K, P);
  static constexpr int NQV = n_qvol(K, P);
  static constexpr int NQF = n_qface(K, P);
  static constexpr int NF = n_faces(K);
  static constexpr int NE = n_edge_nodes(P);
  static constexpr int BASE = slot_offset(K, P);
  static constexpr int O_PHI = BASE;
  static constexpr int O_WXI = O_PHI + NP * NQV;
  static constexpr int O_WETA = O_WXI + NP * NQV;
  static constexpr int O_MINV = O_WETA + NP * NQV;
  static constexpr int O_E1D = O_MINV + NP * NP;
  static constexpr int O_WF = O_E1D + NE * NQF;
  static constexpr int O_MW = O_WF + NQF;
  static constexpr int O_WV = O_MW + NP;
  static constexpr int O_DGX = O_WV + NQV;
  static constexpr int O_DGE = O_DGX + NF * NQV;
  static constexpr int O_PFE = O_DGE + NF * NQV;
  static constexpr int O_GV = O_PFE + 2 * NF * NE * NQF;
  static constexpr int NPROBE = NQV + NF * NQF;  // limiter probe points
};

// Node index of lattice point (ix, iy) in the reference ordering
// (src/reference/elements.py:56-75).
__host__ __device__ constexpr int lattice_node(int kind, int p, int ix, int iy) {
  return kind == 0 ? iy * (p + 1) - iy * (iy - 1) / 2 + ix : iy * (p + 1) + ix;
}

// j-th node of local edge f, walking from its start vertex to its end vertex.
__host__ __device__ constexpr int edge_node(int kind, int p, int f, int j) {
  if (p == 0) return 0;
  if (kind == 0) {
    return f == 0 ? lattice_node(0, p, p - j, j) : (f == 1 ? lattice_node(0, p, 0, p - j) : lattice_node(0, p, j, 0));
  }
  return f == 0 ? lattice_node(1, p, j, 0)
                : (f == 1 ? lattice_node(1, p, p, j) : (f == 2 ? lattice_node(1, p, p - j, p) : lattice_node(1, p, 0, p - j)));
}

}  // namespace nzb
