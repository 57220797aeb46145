// gen_initial.cuh -- the quasi-1D initial state on the generic path, L2-projected
// on the device (src/timestepping/initialize.py:41-102), for any order and any
// geometry order.
//
// One block per element.  At each volume point: the point's coordinates from
// the element's geometry nodes (x = sum_n geom_vol[n, q] x_n, curved Q = 2
// elements included) and w det from the geometry derivatives; density, axial
// velocity and pressure interpolated linearly in x from the quasi-1D solution;
// the wall half-height and its slope by the one-sided-at-the-inlet central
// difference with h = 1e-6 L; vy = vx clip(y / y_w, 0, 1) slope; the conserved
// state.  Then rhs_i = sum_q phi_iq w_q det_q u_q and U = M^-1 rhs with the
// element's own inverse mass, in the reference's (E, NP, 4) layout.  The wall
// and interpolation arithmetic is the specialised kernel's (initial.cuh).
#pragma once
#include "generic.cuh"
#include "initial.cuh"

namespace nzb {

struct GenInitSmem {
  int np, nqv, ng;
  __host__ __device__ int xg() const { return 0; }                 // [2][NG]
  __host__ __device__ int uq() const { return 2 * ng; }            // [NQV][4] point states
  __host__ __device__ int wd() const { return uq() + 4 * nqv; }    // [NQV] w det
  __host__ __device__ int rhs() const { return wd() + nqv; }       // [NP][4]
  __host__ __device__ int total() const { return rhs() + 4 * np; }
};

__global__ void __launch_bounds__(128) k_gen_initial_state(const nzb_gen_mesh m, const nzb_physics ph,
                                                           const nzb_gen_initial_args a) {
  extern __shared__ double sm[];
  const int NP = m.np, NQV = m.nqv, NG = a.ng;
  const GenInitSmem L{NP, NQV, NG};
  const int64_t e = blockIdx.x;
  const int t = threadIdx.x, nt = blockDim.x;
  double* const xg = sm + L.xg();
  double* const uq = sm + L.uq();
  double* const wd = sm + L.wd();
  double* const rhs = sm + L.rhs();
  for (int n = t; n < NG; n += nt) {
    const int64_t node = a.elem_nodes[e * NG + n];
    xg[n] = a.X[2 * node];
    xg[NG + n] = a.X[2 * node + 1];
  }
  __syncthreads();
  const double* W = a.wall;
  const int64_t nq1 = a.n_q1d;
  const double* xs = a.q1d;
  const double g = ph.gamma;
  const double h = W[WALL_H];
  for (int q = t; q < NQV; q += nt) {
    double x = 0.0, y = 0.0, x_xi = 0.0, x_eta = 0.0, y_xi = 0.0, y_eta = 0.0;
    for (int n = 0; n < NG; ++n) {
      const double gv = a.geom_vol[n * NQV + q];
      x = add(x, mul(gv, xg[n]));
      y = add(y, mul(gv, xg[NG + n]));
      const double gxi = a.dgeom_dxi[n * NQV + q], geta = a.dgeom_deta[n * NQV + q];
      x_xi = fma(xg[n], gxi, x_xi);
      x_eta = fma(xg[n], geta, x_eta);
      y_xi = fma(xg[NG + n], gxi, y_xi);
      y_eta = fma(xg[NG + n], geta, y_eta);
    }
    double f[3];
    interp3(xs, xs + nq1, xs + 2 * nq1, xs + 3 * nq1, nq1, x, f);
    const double rho = f[0], vx = f[1], p = f[2];
    const double yw = wall_y(W, x);
    const double xm = sub(x, h);
    const double slope = __ddiv_rn(sub(wall_y(W, add(x, h)), wall_y(W, xm > 0.0 ? xm : 0.0)), add(h, x < h ? x : h));
    const double yr = __ddiv_rn(y, yw > 1e-30 ? yw : 1e-30);
    const double vy = mul(mul(vx, clip01(yr)), slope);
    uq[q * 4 + 0] = rho;
    uq[q * 4 + 1] = mul(rho, vx);
    uq[q * 4 + 2] = mul(rho, vy);
    uq[q * 4 + 3] = add(__ddiv_rn(p, g - 1.0), mul(mul(0.5, rho), add(mul(vx, vx), mul(vy, vy))));
    wd[q] = a.w_vol[q] * (x_xi * y_eta - x_eta * y_xi);
  }
  __syncthreads();
  for (int k = t; k < NP * 4; k += nt) {
    const int i = k >> 2, s = k & 3;
    double acc = 0.0;
    for (int q = 0; q < NQV; ++q) acc = fma(m.phi_vol[i * NQV + q] * wd[q], uq[q * 4 + s], acc);
    rhs[k] = acc;
  }
  __syncthreads();
  const double* minv = a.inv_mass + e * (int64_t)NP * NP;
  for (int k = t; k < NP * 4; k += nt) {
    const int i = k >> 2, s = k & 3;
    double acc = 0.0;
    for (int j = 0; j < NP; ++j) acc = fma(minv[i * NP + j], rhs[j * 4 + s], acc);
    a.out[e * NP * 4 + k] = acc;
  }
}

}  // namespace nzb
