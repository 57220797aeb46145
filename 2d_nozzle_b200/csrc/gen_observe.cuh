// gen_observe.cuh -- the parity observables on the generic path (any order,
// curved elements), on the device.
//
// The integrals behind src/post/postprocess.py:56-75 (boundary_trace), :155-171
// (axial_momentum_flux, mass_flux), :174-192 (entropy_error) and :193-255
// (performance), the same NZB_NOBS sums as observe.cuh: the state traced onto
// the inflow, outflow and wall boundary edges with the owner-side face basis,
// with the normal and |dX/dsigma| of every face point (curved edges), and the
// entropy deviation at the volume points weighted by w det, det from the
// element's geometry nodes.  One block: each thread sums a fixed stride of
// edges and elements, the block a fixed tree, so a result is the same on every
// run.  The host forms thrust, mass flows and exit averages from the sums.
#pragma once
#include "generic.cuh"
#include "observe.cuh"

namespace nzb {

__global__ void __launch_bounds__(OBS_BT) k_gen_observables(const nzb_gen_mesh m, const nzb_physics ph,
                                                            const nzb_gen_obs_args a) {
  const int NP = m.np, NQV = m.nqv, NQF = m.nqf, NG = a.ng;
  const double g = ph.gamma;
  const double* __restrict__ U = a.U;
  const int t = threadIdx.x;
  double acc[NZB_NOBS];
#pragma unroll
  for (int k = 0; k < NZB_NOBS; ++k) acc[k] = 0.0;

  // ---- boundary edges: owner-side traces at the face points
  for (int64_t kb = t; kb < m.n_bnd; kb += OBS_BT) {
    const int64_t k = m.n_int + kb;
    const int tag = m.edge_tag[kb];
    if (tag != NZB_OUTFLOW && tag != NZB_INFLOW && tag != NZB_WALL) continue;
    const int64_t e = m.edge_elem[2 * k];
    const int f = m.edge_face[2 * k];
    const double* pf = m.phi_face + (int64_t)f * NP * NQF;  // side 0: the owner's walk
    for (int q = 0; q < NQF; ++q) {
      double tr[4] = {0.0, 0.0, 0.0, 0.0};
      for (int i = 0; i < NP; ++i) {
        const double c = pf[i * NQF + q];
#pragma unroll
        for (int s = 0; s < 4; ++s) tr[s] = fma(c, U[(e * NP + i) * 4 + s], tr[s]);
      }
      const Prim w = primitives(tr, g);
      const double nx = m.edge_normal[(k * NQF + q) * 2 + 0];
      const double ny = m.edge_normal[(k * NQF + q) * 2 + 1];
      const double ds = m.edge_jac[k * NQF + q] * m.w_face[q];
      const double vn = w.vx * nx + w.vy * ny;
      if (tag == NZB_OUTFLOW) {
        acc[NZB_OBS_MOM_OUT] += (w.rho * w.vx * vn + w.p * nx) * ds;
        acc[NZB_OBS_MASS_OUT] += w.rho * vn * ds;
        acc[NZB_OBS_EXIT_LEN] += ds;
        acc[NZB_OBS_EXIT_MACH] += sqrt((w.vx * w.vx + w.vy * w.vy) * w.rho / (g * w.p)) * ds;
        acc[NZB_OBS_EXIT_P] += w.p * ds;
        acc[NZB_OBS_EXIT_T] += w.p / (a.r_gas * w.rho) * ds;
      } else if (tag == NZB_INFLOW) {
        acc[NZB_OBS_MOM_IN] += (w.rho * w.vx * vn + w.p * nx) * ds;
        acc[NZB_OBS_MASS_IN] += w.rho * vn * ds;
      } else {
        acc[NZB_OBS_WALL_PX] += w.p * nx * ds;
      }
    }
  }

  // ---- elements: (s / s_t - 1)^2 w det at the volume points, and the area
  for (int64_t e = t; e < m.n_elem; e += OBS_BT) {
    double ent = 0.0;
    for (int q = 0; q < NQV; ++q) {
      double x_xi = 0.0, x_eta = 0.0, y_xi = 0.0, y_eta = 0.0;
      for (int n = 0; n < NG; ++n) {
        const int64_t node = a.elem_nodes[e * NG + n];
        const double gxi = a.dgeom_dxi[n * NQV + q], geta = a.dgeom_deta[n * NQV + q];
        const double xn = a.X[2 * node], yn = a.X[2 * node + 1];
        x_xi = fma(xn, gxi, x_xi);
        x_eta = fma(xn, geta, x_eta);
        y_xi = fma(yn, gxi, y_xi);
        y_eta = fma(yn, geta, y_eta);
      }
      double uq[4] = {0.0, 0.0, 0.0, 0.0};
      for (int i = 0; i < NP; ++i) {
        const double phi = m.phi_vol[i * NQV + q];
#pragma unroll
        for (int s = 0; s < 4; ++s) uq[s] = fma(phi, U[(e * NP + i) * 4 + s], uq[s]);
      }
      const Prim w = primitives(uq, g);
      const double r = (w.p / pow(w.rho, g)) / a.s_t - 1.0;
      ent += r * r * (a.w_vol[q] * (x_xi * y_eta - x_eta * y_xi));
    }
    acc[NZB_OBS_ENTROPY] += ent;
    acc[NZB_OBS_AREA] += m.elem_area[e];
  }

  // ---- block sums in a fixed tree
  __shared__ double red[NZB_NOBS][OBS_BT];
#pragma unroll
  for (int k = 0; k < NZB_NOBS; ++k) red[k][t] = acc[k];
  __syncthreads();
  for (int h = OBS_BT / 2; h > 0; h >>= 1) {
    if (t < h)
#pragma unroll
      for (int k = 0; k < NZB_NOBS; ++k) red[k][t] += red[k][t + h];
    __syncthreads();
  }
  if (t < NZB_NOBS) a.out[t] = red[t][0];
}

}  // namespace nzb
