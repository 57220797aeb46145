// gen_geometry.cuh -- the generic path's operators, built on the device from
// the node coordinates, for any order and any geometry order.
//
// The coordinate-dependent part of build_operators (src/spatial/operators.py:
// 209-342) in the reference's per-element layout, the arrays the generic
// kernels (generic.cuh) read:
//   per element (one block each)
//     the Jacobian at every volume point from the geometry nodes
//       (x_xi = sum_n dgeom_dxi[n, q] x_n, ...), det, the inverse metric
//       (xi_x, xi_y, eta_x, eta_y) = (y_eta, -x_eta, -y_xi, x_xi) / det and
//       wdet = w_q det;
//     area = sum_q wdet, mean weights sum_q phi_iq wdet / area;
//     grad_x[i, q] = wdet (dphi_dxi[i, q] xi_x + dphi_deta[i, q] eta_x), grad_y;
//     M_ij = sum_q phi_iq phi_jq wdet, inverted in place (Gauss-Jordan: M is
//       symmetric positive definite, so no pivoting is needed);
//     grad_x_m = M^-1 grad_x, grad_y_m, face_basis_m = M^-1 phi_face[side, f];
//   per edge (one thread each, from its owner element and face)
//     t = sum_n dgeom_dsigma[f, n, q] X_n at every face point, |t|, the unit
//     normal (t_y, -t_x) / |t| and the length sum_q |t| w_q.
// The sums run in the reference's index order; its matrix inverse is LAPACK's,
// so the results agree with the host build to round-off, not bit for bit.
#pragma once
#include "generic.cuh"

namespace nzb {

// Shared-memory layout of k_gen_elem_geometry, in doubles.
struct GenGeoSmem {
  int np, nqv, ng;
  __host__ __device__ int xg() const { return 0; }                   // [2][NG] node x, then y
  __host__ __device__ int met() const { return 2 * ng; }             // [5][NQV] xi_x xi_y eta_x eta_y wdet
  __host__ __device__ int gx() const { return met() + 5 * nqv; }     // [NP][NQV]
  __host__ __device__ int gy() const { return gx() + np * nqv; }     // [NP][NQV]
  __host__ __device__ int mass() const { return gy() + np * nqv; }   // [NP][NP]
  __host__ __device__ int col() const { return mass() + np * np; }   // [NP] pivot column
  __host__ __device__ int area() const { return col() + np; }        // [1]
  __host__ __device__ int total() const { return area() + 1; }
};

__global__ void __launch_bounds__(128) k_gen_elem_geometry(const nzb_gen_mesh m, const nzb_gen_geometry_args a) {
  extern __shared__ double sm[];
  const int NP = m.np, NQV = m.nqv, NF = m.nface, NQF = m.nqf, NG = a.ng;
  const GenGeoSmem L{NP, NQV, NG};
  const int64_t e = blockIdx.x;
  const int t = threadIdx.x, nt = blockDim.x;
  double* const xg = sm + L.xg();
  double* const met = sm + L.met();
  double* const gx = sm + L.gx();
  double* const gy = sm + L.gy();
  double* const M = sm + L.mass();
  double* const col = sm + L.col();

  for (int n = t; n < NG; n += nt) {
    const int64_t node = a.elem_nodes[e * NG + n];
    xg[n] = a.X[2 * node];
    xg[NG + n] = a.X[2 * node + 1];
  }
  __syncthreads();
  for (int q = t; q < NQV; q += nt) {
    double x_xi = 0.0, x_eta = 0.0, y_xi = 0.0, y_eta = 0.0;
    for (int n = 0; n < NG; ++n) {
      const double gxi = a.dgeom_dxi[n * NQV + q], geta = a.dgeom_deta[n * NQV + q];
      x_xi = fma(xg[n], gxi, x_xi);
      x_eta = fma(xg[n], geta, x_eta);
      y_xi = fma(xg[NG + n], gxi, y_xi);
      y_eta = fma(xg[NG + n], geta, y_eta);
    }
    const double det = x_xi * y_eta - x_eta * y_xi;
    if (!(det > 0.0)) atomicAdd(a.bad, 1);
    const double inv = 1.0 / det;
    met[0 * NQV + q] = y_eta * inv;
    met[1 * NQV + q] = -x_eta * inv;
    met[2 * NQV + q] = -y_xi * inv;
    met[3 * NQV + q] = x_xi * inv;
    met[4 * NQV + q] = a.w_vol[q] * det;
  }
  __syncthreads();
  if (t == 0) {
    double s = 0.0;
    for (int q = 0; q < NQV; ++q) s += met[4 * NQV + q];
    sm[L.area()] = s;
    a.elem_area[e] = s;
  }
  __syncthreads();
  const double area = sm[L.area()];
  const double* const wdet = met + 4 * NQV;
  for (int i = t; i < NP; i += nt) {
    double s = 0.0;
    for (int q = 0; q < NQV; ++q) s = fma(m.phi_vol[i * NQV + q], wdet[q], s);
    a.mean_weights[e * NP + i] = s / area;
  }
  const int64_t gbase = e * (int64_t)NP * NQV;
  for (int k = t; k < NP * NQV; k += nt) {
    const int q = k % NQV;
    const double dx = a.dphi_dxi[k], de = a.dphi_deta[k];
    const double vx = wdet[q] * (dx * met[q] + de * met[2 * NQV + q]);
    const double vy = wdet[q] * (dx * met[NQV + q] + de * met[3 * NQV + q]);
    gx[k] = vx;
    gy[k] = vy;
    a.grad_x[gbase + k] = vx;
    a.grad_y[gbase + k] = vy;
  }
  for (int k = t; k < NP * NP; k += nt) {
    const int i = k / NP, j = k % NP;
    double s = 0.0;
    for (int q = 0; q < NQV; ++q) s = fma(m.phi_vol[i * NQV + q] * m.phi_vol[j * NQV + q], wdet[q], s);
    M[k] = s;
  }
  __syncthreads();
  // Gauss-Jordan in place: step p scales the pivot row by 1 / M_pp and clears
  // column p from every other row; the cleared entries become the inverse's
  for (int p = 0; p < NP; ++p) {
    const double piv = 1.0 / M[p * NP + p];
    for (int i = t; i < NP; i += nt) col[i] = M[i * NP + p];
    __syncthreads();
    for (int j = t; j < NP; j += nt) M[p * NP + j] = (j == p ? 1.0 : M[p * NP + j]) * piv;
    __syncthreads();
    for (int k = t; k < NP * NP; k += nt) {
      const int i = k / NP, j = k % NP;
      if (i != p) M[k] = fma(-col[i], M[p * NP + j], j == p ? 0.0 : M[k]);
    }
    __syncthreads();
  }
  const int64_t mbase = e * (int64_t)NP * NP;
  for (int k = t; k < NP * NP; k += nt) a.inv_mass[mbase + k] = M[k];
  for (int k = t; k < NP * NQV; k += nt) {
    const int i = k / NQV, q = k % NQV;
    double sx = 0.0, sy = 0.0;
    for (int j = 0; j < NP; ++j) {
      sx = fma(M[i * NP + j], gx[j * NQV + q], sx);
      sy = fma(M[i * NP + j], gy[j * NQV + q], sy);
    }
    a.grad_x_m[gbase + k] = sx;
    a.grad_y_m[gbase + k] = sy;
  }
  const int64_t fbase = e * (int64_t)NF * NP * NQF;
  for (int k = t; k < NF * NP * NQF; k += nt) {
    const int f = k / (NP * NQF), i = (k / NQF) % NP, q = k % NQF;
    const int side = m.face_side[e * NF + f];
    double s = 0.0;
    for (int j = 0; j < NP; ++j) s = fma(M[i * NP + j], m.phi_face[((side * NF + f) * NP + j) * NQF + q], s);
    a.face_basis_m[fbase + k] = s;
  }
}

__global__ void __launch_bounds__(128) k_gen_edge_geometry(const nzb_gen_mesh m, const nzb_gen_geometry_args a) {
  const int64_t NK = m.n_int + m.n_bnd;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NK) return;
  const int NG = a.ng, NQF = m.nqf;
  const int64_t e = m.edge_elem[2 * k];
  const int f = m.edge_face[2 * k];
  double len = 0.0;
  for (int q = 0; q < NQF; ++q) {
    double tx = 0.0, ty = 0.0;
    for (int n = 0; n < NG; ++n) {
      const int64_t node = a.elem_nodes[e * NG + n];
      const double d = a.dgeom_dsigma[(f * NG + n) * NQF + q];
      tx = fma(d, a.X[2 * node], tx);
      ty = fma(d, a.X[2 * node + 1], ty);
    }
    const double jac = sqrt(tx * tx + ty * ty);
    a.edge_normal[(k * NQF + q) * 2 + 0] = ty / jac;
    a.edge_normal[(k * NQF + q) * 2 + 1] = -tx / jac;
    a.edge_jac[k * NQF + q] = jac;
    len += jac * m.w_face[q];
  }
  a.edge_length[k] = len;
}

}  // namespace nzb
