// geometry.cuh -- the metric terms the kernels read, built on the device from node coordinates.
//
// The coordinate-dependent part of build_operators (src/spatial/operators.py:
// 240-303) for straight-sided (Q = 1) elements, in the device layout:
//   affine triangles  (xi_x, xi_y, eta_x, eta_y, det) from the vertex-shape
//                     derivatives at the first volume point;
//   general elements  the vertex coordinates and the inverse of the mass matrix
//                     M_ij = sum_q phi_iq phi_jq w_q det_q;
//   every element     area = sum_q w_q det_q;
//   every edge        from its owner's vertices: the tangent t = sum_v
//                     dgs[f][v] X_v, |t|, the unit normal (t_y, -t_x) / |t| and
//                     the length |t| sum_q w_q.
// The topology (connectivity, edge numbering) does not depend on the
// coordinates and stays as built once on the host; a design change -- a new
// wall, a new node set -- only reruns these two kernels.
#pragma once
#include "element.cuh"

namespace nzb {

template <int K, int P, bool AFF>
__global__ void __launch_bounds__(128) k_elem_geometry(const nzb_mesh m, const nzb_geometry_args a) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP, NQV = S::NQV, NV = S::NF;
  const int64_t E = m.n_elem;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  double xv[NV], yv[NV];
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const int64_t n = a.elem_nodes[e * NV + v];
    xv[v] = a.X[2 * n];
    yv[v] = a.X[2 * n + 1];
  }
  double area = 0.0;
  if (AFF) {
    double x_xi, x_eta, y_xi, y_eta;
    const double det = point_det<K, P>(xv, yv, 0, x_xi, x_eta, y_xi, y_eta);
    const double inv = 1.0 / det;
    a.geo[0 * E + e] = y_eta * inv;
    a.geo[1 * E + e] = -x_eta * inv;
    a.geo[2 * E + e] = -y_xi * inv;
    a.geo[3 * E + e] = x_xi * inv;
    a.geo[4 * E + e] = det;
#pragma unroll 1
    for (int q = 0; q < NQV; ++q) {
      const double dq = point_det<K, P>(xv, yv, q, x_xi, x_eta, y_xi, y_eta);
      area += tab<K, P>(S::O_WV + q) * dq;
    }
  } else {
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      a.geo[v * E + e] = xv[v];
      a.geo[(NV + v) * E + e] = yv[v];
    }
    // mass matrix, then its inverse in place (Gauss-Jordan; M is symmetric
    // positive definite, so no pivoting is needed)
    double M[NP][NP];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) M[i][j] = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQV; ++q) {
      double x_xi, x_eta, y_xi, y_eta;
      const double wd = tab<K, P>(S::O_WV + q) * point_det<K, P>(xv, yv, q, x_xi, x_eta, y_xi, y_eta);
      area += wd;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const double pi = tab<K, P>(S::O_PHI + i * NQV + q) * wd;
#pragma unroll
        for (int j = 0; j < NP; ++j) M[i][j] = fma(pi, tab<K, P>(S::O_PHI + j * NQV + q), M[i][j]);
      }
    }
#pragma unroll
    for (int k = 0; k < NP; ++k) {
      const double piv = 1.0 / M[k][k];
      M[k][k] = 1.0;
#pragma unroll
      for (int j = 0; j < NP; ++j) M[k][j] *= piv;
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        if (i == k) continue;
        const double f = M[i][k];
        M[i][k] = 0.0;
#pragma unroll
        for (int j = 0; j < NP; ++j) M[i][j] = fma(-f, M[k][j], M[i][j]);
      }
    }
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int j = 0; j < NP; ++j) a.minv[(i * NP + j) * E + e] = M[i][j];
  }
  a.area[e] = area;
}

template <int K, int P>
__global__ void __launch_bounds__(128) k_edge_geometry(const nzb_mesh m, const nzb_geometry_args a) {
  using S = Shape<K, P>;
  constexpr int NQF = S::NQF, NV = S::NF;
  const int64_t NK = m.n_edge;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NK) return;
  const int64_t e = a.edge_conn[k];
  const int f = a.edge_conn[2 * NK + k] & 7;
  double tx = 0.0, ty = 0.0;
#pragma unroll
  for (int v = 0; v < NV; ++v) {
    const int64_t n = a.elem_nodes[e * NV + v];
    tx = fma(a.dgs[4 * f + v], a.X[2 * n], tx);
    ty = fma(a.dgs[4 * f + v], a.X[2 * n + 1], ty);
  }
  const double jac = sqrt(tx * tx + ty * ty);
  double len = 0.0;
#pragma unroll
  for (int q = 0; q < NQF; ++q) len += jac * tab<K, P>(S::O_WF + q);
  a.edge_geo[4 * k + 0] = ty / jac;
  a.edge_geo[4 * k + 1] = -tx / jac;
  a.edge_geo[4 * k + 2] = jac;
  a.edge_geo[4 * k + 3] = len;
}

}  // namespace nzb
