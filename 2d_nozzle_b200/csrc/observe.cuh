// observe.cuh -- the parity observables of a converged state, on the device.
//
// Restates the integrals behind src/post/postprocess.py:56-75 (boundary_trace),
// :155-171 (axial_momentum_flux, mass_flux), :174-192 (entropy_error) and
// :193-255 (performance): the state traced onto the inflow, outflow and wall
// boundaries with the owner-side face basis, and the entropy deviation at the
// volume quadrature points.  One block per instance (a single mesh is one
// instance) sums its own boundary edges and elements, each thread in a fixed
// stride and the block in a fixed tree, so a result is the same on every run.
// The per-instance sums (NZB_OBS_* in nozzle_b200.h) go to the host, which
// forms thrust, mass flows, exit averages and their ratios from them.
#pragma once
#include "element.cuh"

namespace nzb {

constexpr int OBS_BT = 256;

template <int K, int P, bool AFF>
__global__ void __launch_bounds__(OBS_BT) k_observables(const nzb_mesh m, const nzb_physics ph,
                                                        const nzb_obs_args a) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP, NQV = S::NQV, NQF = S::NQF, NE = S::NE, NF = S::NF;
  const int64_t E = m.n_elem;
  const int64_t NK = m.n_edge;
  const double g = ph.gamma;
  const double* __restrict__ U = a.U;
  const int b = blockIdx.x, t = threadIdx.x;
  double acc[NZB_NOBS];
#pragma unroll
  for (int k = 0; k < NZB_NOBS; ++k) acc[k] = 0.0;

  // ---- boundary edges: owner-side traces at the face points
  for (int i = a.bseg[b] + t; i < a.bseg[b + 1]; i += OBS_BT) {
    const int k = a.bedges[i];
    const int e = m.edge_conn[k];
    const int code = m.edge_conn[2 * NK + k];
    const int f = code & 7;
    const int tag = code >> 6;
    const double nx = m.edge_geo[4 * (int64_t)k + 0];
    const double ny = m.edge_geo[4 * (int64_t)k + 1];
    const double jac = m.edge_geo[4 * (int64_t)k + 2];
    for (int q = 0; q < NQF; ++q) {
      double tr[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int j = 0; j < NE; ++j) {
        const double c = pfe<K, P>(0, f, j, q);
        const int n = edge_node(K, P, f, j);
#pragma unroll
        for (int s = 0; s < 4; ++s) tr[s] = fma(c, U[(s * NP + n) * E + e], tr[s]);
      }
      const Prim w = primitives(tr, g);
      const double ds = jac * tab<K, P>(S::O_WF + q);
      const double vn = w.vx * nx + w.vy * ny;
      const double mom = (w.rho * w.vx * vn + w.p * nx) * ds;
      const double mass = w.rho * vn * ds;
      if (tag == NZB_OUTFLOW) {
        acc[NZB_OBS_MOM_OUT] += mom;
        acc[NZB_OBS_MASS_OUT] += mass;
        acc[NZB_OBS_EXIT_LEN] += ds;
        acc[NZB_OBS_EXIT_MACH] += sqrt((w.vx * w.vx + w.vy * w.vy) * w.rho / (g * w.p)) * ds;
        acc[NZB_OBS_EXIT_P] += w.p * ds;
        acc[NZB_OBS_EXIT_T] += w.p / (a.r_gas * w.rho) * ds;
      } else if (tag == NZB_INFLOW) {
        acc[NZB_OBS_MOM_IN] += mom;
        acc[NZB_OBS_MASS_IN] += mass;
      } else if (tag == NZB_WALL) {
        acc[NZB_OBS_WALL_PX] += w.p * nx * ds;
      }
    }
  }

  // ---- elements: (s / s_t - 1)^2 at the volume points, and the area
  for (int64_t e = (int64_t)a.eseg[b] + t; e < a.eseg[b + 1]; e += OBS_BT) {
    double det = 1.0;
    double xv[NF], yv[NF];
    if (AFF) {
      det = m.geo[4 * E + e];
    } else {
#pragma unroll
      for (int v = 0; v < NF; ++v) {
        xv[v] = m.geo[v * E + e];
        yv[v] = m.geo[(NF + v) * E + e];
      }
    }
    double ent = 0.0;
    for (int q = 0; q < NQV; ++q) {
      double uq[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const double phi = tab<K, P>(S::O_PHI + i * NQV + q);
#pragma unroll
        for (int s = 0; s < 4; ++s) uq[s] = fma(phi, U[(s * NP + i) * E + e], uq[s]);
      }
      double dq = det;
      if (!AFF) {
        double x_xi, x_eta, y_xi, y_eta;
        dq = point_det<K, P>(xv, yv, q, x_xi, x_eta, y_xi, y_eta);
      }
      const Prim w = primitives(uq, g);
      const double r = (w.p / pow(w.rho, g)) / a.s_t - 1.0;
      ent += r * r * (tab<K, P>(S::O_WV + q) * dq);
    }
    acc[NZB_OBS_ENTROPY] += ent;
    acc[NZB_OBS_AREA] += m.area[e];
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
  if (t < NZB_NOBS) a.out[(int64_t)b * NZB_NOBS + t] = red[t][0];
}

}  // namespace nzb
