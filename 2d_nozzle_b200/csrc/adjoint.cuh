// adjoint.cuh -- the transposed linearisation of the DG residual, matrix-free.
//
// The discrete adjoint of src/sensitivity.py:289-383 needs two products with
// the transposed Jacobians of the unfolded residual R(U, X, p_back)
// (src/spatial/assembly.py:153-157, M dU/dt = -R):
//
//   k_vjp         v = (dR/dU)^T lam, and fused on top of it the adjoint
//                 pseudo-time march: the defect v - dJ/dU, the rate
//                 -M^-1 (v - dJ/dU), and one classical RK4 stage of
//                 dlam/dtau = that rate with a frozen local step;
//   k_vjp_coords  (dR/dX)^T lam per element vertex, and (dR/dp_back)^T lam.
//
// Both are element-centric, like the forward kernel: an element computes
// every term that lands in its own output from its own side, so nothing is
// scattered between threads and no edge array is needed.
//
// State VJP.  With U_q = sum_j phi_jq U_j at a volume point and
// R_i = sum_q (WXI_iq fx_q + WETA_iq fe_q) (the forward kernel's form, metric
// and sign folded in), lam . R is a function of U_q only through the Euler
// fluxes (F, G)(U_q), so
//   v_j += phi_jq (J_F(U_q)^T cF_q + J_G(U_q)^T cG_q),
// with cF, cG the lam-weighted metric combinations at q.  A face point
// contributes w jac (lam_L - lam_R) . Fhat(U_L, U_R, n) to lam . R over both
// elements of the edge; each element differentiates it with respect to its own
// trace.  The flux Jacobians are exact: the flux code is evaluated once in
// forward-mode dual numbers (dual.cuh) seeded on the four own-trace
// components, and its branches follow the values, as the reference's
// differentiated NumPy code does.
//
// Coordinate VJP.  For straight-sided elements det (xi_x, xi_y) =
// (y_eta, -x_eta) and det (eta_x, eta_y) = (-y_xi, x_xi) are linear in the
// vertex coordinates (src/spatial/operators.py:240-278), so the volume term's
// derivative is closed form.  An edge's term jac * sum_q w_q (lam_L - lam_R) .
// Fhat(n) depends on the owner's vertices through the tangent t = sum_v
// dgeom_dsigma[f, v] X_v, jac = |t| and n = (t_y, -t_x) / |t|
// (src/spatial/operators.py:296-303); the derivative through n comes from the
// flux in dual numbers seeded on (n_x, n_y, p_back).  Only the owner handles an
// edge, so each edge's geometry derivative is counted once.
#pragma once
#include "dual.cuh"
#include "element.cuh"

namespace nzb {

enum { ADJ_VJP = 0, ADJ_DEFECT = 1, ADJ_RATE = 2, ADJ_RK4 = 3 };

struct AdjWork {
  int mode;
  int stage;           // RK4 stage 0..3
  const double* U;     // linearisation state
  const double* lam;   // the adjoint the product is taken at (RK4: this stage's input)
  const double* seed;  // dJ/dU (defect, rate, RK4)
  double* out;         // VJP / defect / rate; RK4: the next stage's input
  double* lam0;        // RK4: the step's starting lambda; stage 3 overwrites it with the new lambda
  const double* dt;    // RK4: frozen local step
  double* f0;          // RK4: stored stage rates
  double* f1;
  double* f2;
  double* norm_partial;  // defect: per-block sum of squares (nullable)
  double* elem_norm;     // defect: per-element sum of squares (nullable)
};

struct CoordWork {
  const double* U;
  const double* lam;
  const double* verts;  // (2 NV, E): vertex x then y
  double* gvert;        // (2 NV, E): d(lam . R)/d(x_v), then /d(y_v)
  double* gpb;          // (E, nullable): d(lam . R)/d(p_back)
  double dgs[4][4];     // tangent of face f = sum_v dgs[f][v] X_v
};

// b = J_F(U)^T cF + J_G(U)^T cG for the Euler flux (F, G) of thermo.py:64-70,
// from the closed-form Jacobians (u = m / rho, v = n / rho, q^2 = u^2 + v^2,
// phi = (gamma - 1) q^2 / 2, H = (E + p) / rho):
//   dF/dU = [0, 1, 0, 0; phi - u^2, (3 - gamma) u, -(gamma - 1) v, gamma - 1;
//            -u v, v, u, 0; u (phi - H), H - (gamma - 1) u^2, -(gamma - 1) u v, gamma u]
// and dG/dU likewise with the roles of u and v exchanged.  Returns false --
// leaving b to the dual-number path -- where a floor of the density or the
// pressure is active, whose derivative these formulas do not have.
__device__ __forceinline__ bool euler_flux_vjp(const double (&U)[4], double g, const double (&cF)[4],
                                               const double (&cG)[4], double (&b)[4]) {
  const double rho = U[0];
  if (!(rho >= FLOOR)) return false;
  const double u = U[1] / rho, v = U[2] / rho;
  const double q2 = u * u + v * v;
  const double gm = g - 1.0;
  const double p = gm * (U[3] - 0.5 * rho * q2);
  if (!(p >= FLOOR)) return false;
  const double H = (U[3] + p) / rho;
  const double phi = 0.5 * gm * q2;
  const double uv = u * v;
  b[0] = cF[1] * (phi - u * u) - cF[2] * uv + cF[3] * u * (phi - H) - cG[1] * uv + cG[2] * (phi - v * v) +
         cG[3] * v * (phi - H);
  b[1] = cF[0] + cF[1] * (3.0 - g) * u + cF[2] * v + cF[3] * (H - gm * u * u) + cG[1] * v - cG[2] * gm * u -
         cG[3] * gm * uv;
  b[2] = -cF[1] * gm * v + cF[2] * u - cF[3] * gm * uv + cG[0] + cG[1] * u + cG[2] * (3.0 - g) * v +
         cG[3] * (H - gm * v * v);
  b[3] = gm * (cF[1] + cG[2]) + g * (cF[3] * u + cG[3] * v);
  return true;
}

// Resident blocks per SM asked of the compiler for k_vjp (as NZB_MINB_* for
// the forward kernels): registers per thread are capped at 65536 / (MINB * NT).
// Linear elements run with three blocks (170 registers): measured 13-20 %
// faster on the design sweep's p = 1 buckets; higher orders spill and slow down.
#ifndef NZB_MINB_VJP
#define NZB_MINB_VJP 1
#endif
template <int K, int P>
struct VjpBounds {
  static constexpr int MINB = (P <= 1 ? 3 : NZB_MINB_VJP) * 128 / Launch<K, P>::NT;
};

template <int K, int P, bool AFF>
__global__ void __launch_bounds__(Launch<K, P>::NT, VjpBounds<K, P>::MINB)
    k_vjp(const nzb_mesh m, const nzb_physics ph, const AdjWork w) {
  using S = Shape<K, P>;
  using D4 = Dual<4>;
  constexpr int NP = S::NP, NQV = S::NQV, NQF = S::NQF, NF = S::NF, NE = S::NE;
  constexpr int BT = Launch<K, P>::NT;
  __shared__ double vacc[NP * 4 * BT];  // vacc[(i * 4 + s) * BT + t]
  const int t = threadIdx.x;
  const int64_t E = m.n_elem;
  const int64_t blk = listed_block(m.vjp_blocks, E, BT);
  const int64_t e = blk * BT + t;
  int inst = -1;
  if (e < E && m.elem_inst) inst = __ldg(m.elem_inst + e);
  const bool active = e < E && (inst < 0 || __ldg(m.inst_status + inst) == 0);
  const double p_back = (inst >= 0 && m.inst_p_back) ? __ldg(m.inst_p_back + inst) : ph.p_back;
  const double g = ph.gamma;
  double dsq = 0.0;
  if (active) {
    const double* __restrict__ U = w.U;
    const double* __restrict__ L = w.lam;
    // the epilogue's operands (dJ/dU, the step's starting lambda, in the last
    // RK4 stage the stored stage rates) start toward the caches now, so the
    // loads after the face and volume loops need not wait on DRAM
    if (w.mode != ADJ_VJP) {
#pragma unroll
      for (int k = 0; k < NP * 4; ++k) {
        const int64_t o = (int64_t)k * E + e;
        prefetch_line(w.seed + o);
        if (w.mode == ADJ_RK4) {
          prefetch_line(w.lam0 + o);
          if (w.stage == 3) {
            prefetch_line(w.f0 + o);
            prefetch_line(w.f1 + o);
            prefetch_line(w.f2 + o);
          }
        }
      }
    }
#pragma unroll
    for (int i = 0; i < NP * 4; ++i) vacc[i * BT + t] = 0.0;
    double xx = 0, xy = 0, yx = 0, yy = 0, det = 1.0;
    double xv[NF], yv[NF];
    if (AFF) {
      xx = __ldg(m.geo + 0 * E + e);
      xy = __ldg(m.geo + 1 * E + e);
      yx = __ldg(m.geo + 2 * E + e);
      yy = __ldg(m.geo + 3 * E + e);
      det = __ldg(m.geo + 4 * E + e);
    } else {
#pragma unroll
      for (int v = 0; v < NF; ++v) {
        xv[v] = __ldg(m.geo + v * E + e);
        yv[v] = __ldg(m.geo + (NF + v) * E + e);
      }
    }

    // ---- faces: d/d(own trace) of w jac (lam_L - lam_R) . Fhat(U_L, U_R, n)
#pragma unroll 1
    for (int f = 0; f < NF; ++f) {
      const int code = __ldg(m.face_code + f * E + e);
      const int k = __ldg(m.face_edge + f * E + e);
      const int nb = __ldg(m.face_nbr + f * E + e);
      const int side = code & 1;
      const int nf = (code >> 1) & 7;
      const int tag = code >> 4;
      const double nx = __ldg(m.edge_geo + 4 * (int64_t)k + 0);
      const double ny = __ldg(m.edge_geo + 4 * (int64_t)k + 1);
      const double jac = __ldg(m.edge_geo + 4 * (int64_t)k + 2);
      // the neighbour's edge coefficients (scattered reads), once per face
      double un[NE][4], lnb[NE][4];
      if (nb >= 0) {
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const int n = edge_node(K, P, nf, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            un[j][s] = __ldg(U + (s * NP + n) * E + nb);
            lnb[j][s] = __ldg(L + (s * NP + n) * E + nb);
          }
        }
      }
#pragma unroll 1
      for (int q = 0; q < NQF; ++q) {
        double tc[4] = {0.0, 0.0, 0.0, 0.0}, lc[4] = {0.0, 0.0, 0.0, 0.0};
        double tn[4] = {0.0, 0.0, 0.0, 0.0}, ln[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const double c = pfe<K, P>(side, f, j, q);
          const int n = edge_node(K, P, f, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            tc[s] = fma(c, __ldg(U + (s * NP + n) * E + e), tc[s]);
            lc[s] = fma(c, __ldg(L + (s * NP + n) * E + e), lc[s]);
          }
        }
        if (nb >= 0) {
#pragma unroll
          for (int j = 0; j < NE; ++j) {
            const double c = pfe<K, P>(1 - side, nf, j, q);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
              tn[s] = fma(c, un[j][s], tn[s]);
              ln[s] = fma(c, lnb[j][s], ln[s]);
            }
          }
        }
        const double scale = jac * c_tab[S::O_WF + q];
        double xi[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) xi[s] = nb >= 0 ? scale * (side ? ln[s] - lc[s] : lc[s] - ln[s]) : scale * lc[s];
        // only the own trace is seeded; the neighbour's trace, the normal and
        // the back pressure enter as plain numbers
        D4 own[4], F[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) own[s] = D4::seed(tc[s], s);
        if (nb >= 0) {
          if (side)
            interface_flux(tn, own, nx, ny, ph, F);
          else
            interface_flux(own, tn, nx, ny, ph, F);
        } else {
          boundary_flux(tag, own, nx, ny, ph, p_back, F);
        }
        double a[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          double acc = 0.0;
#pragma unroll
          for (int s = 0; s < 4; ++s) acc = fma(xi[s], F[s].d[u], acc);
          a[u] = acc;
        }
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const double c = pfe<K, P>(side, f, j, q);
          const int n = edge_node(K, P, f, j);
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            double& r = vacc[(n * 4 + u) * BT + t];
            r = fma(c, a[u], r);
          }
        }
      }
    }

    // ---- volume: phi_jq (J_F^T cF + J_G^T cG) at every volume point
    const double vs = AFF ? -det : -1.0;
#pragma unroll 1
    for (int q = 0; q < NQV; ++q) {
      double uq[4] = {0.0, 0.0, 0.0, 0.0}, lx[4] = {0.0, 0.0, 0.0, 0.0}, le[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const double phi = c_tab[S::O_PHI + i * NQV + q];
        const double a = c_tab[S::O_WXI + i * NQV + q];
        const double b = c_tab[S::O_WETA + i * NQV + q];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const double us = __ldg(U + (s * NP + i) * E + e);
          const double ls = __ldg(L + (s * NP + i) * E + e);
          uq[s] = fma(phi, us, uq[s]);
          lx[s] = fma(a, ls, lx[s]);
          le[s] = fma(b, ls, le[s]);
        }
      }
      double a00 = xx, a01 = xy, a10 = yx, a11 = yy;
      if (!AFF) {
        double x_xi, x_eta, y_xi, y_eta;
        point_det<K, P>(xv, yv, q, x_xi, x_eta, y_xi, y_eta);
        a00 = y_eta;
        a01 = -x_eta;
        a10 = -y_xi;
        a11 = x_xi;
      }
      double cF[4], cG[4];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        cF[s] = vs * (a00 * lx[s] + a10 * le[s]);
        cG[s] = vs * (a01 * lx[s] + a11 * le[s]);
      }
      double b[4];
      if (!euler_flux_vjp(uq, g, cF, cG, b)) {
        // a floored density or pressure: differentiate the floored flux itself
        D4 Uq[4], F[4], G[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) Uq[s] = D4::seed(uq[s], s);
        euler_flux(Uq, g, F, G);
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          double acc = 0.0;
#pragma unroll
          for (int s = 0; s < 4; ++s) acc = fma(cF[s], F[s].d[u], fma(cG[s], G[s].d[u], acc));
          b[u] = acc;
        }
      }
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const double phi = c_tab[S::O_PHI + i * NQV + q];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          double& r = vacc[(i * 4 + u) * BT + t];
          r = fma(phi, b[u], r);
        }
      }
    }

    // ---- epilogue
    if (w.mode == ADJ_VJP) {
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int s = 0; s < 4; ++s) w.out[(s * NP + i) * E + e] = vacc[(i * 4 + s) * BT + t];
    } else if (w.mode == ADJ_DEFECT) {
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          const int64_t o = (s * NP + i) * E + e;
          const double d = vacc[(i * 4 + s) * BT + t] - __ldg(w.seed + o);
          if (w.out) w.out[o] = d;
          dsq = fma(d, d, dsq);
        }
      if (w.elem_norm) w.elem_norm[e] = dsq;
    } else {
      // rate = -M^-1 (v - seed), one component at a time
      const double dte = w.mode == ADJ_RK4 ? __ldg(w.dt + e) : 0.0;
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        double d[NP];
#pragma unroll
        for (int j = 0; j < NP; ++j) d[j] = vacc[(j * 4 + s) * BT + t] - __ldg(w.seed + (s * NP + j) * E + e);
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          double r = 0.0;
          if (AFF) {
#pragma unroll
            for (int j = 0; j < NP; ++j) r = fma(tab<K, P>(S::O_MINV + i * NP + j), d[j], r);
            r = -(r / det);
          } else {
#pragma unroll
            for (int j = 0; j < NP; ++j) r = fma(__ldg(m.minv + (i * NP + j) * E + e), d[j], r);
            r = -r;
          }
          const int64_t o = (s * NP + i) * E + e;
          if (w.mode == ADJ_RATE) {
            w.out[o] = r;
          } else if (w.stage == 0) {
            w.f0[o] = r;
            w.out[o] = w.lam0[o] + 0.5 * dte * r;
          } else if (w.stage == 1) {
            w.f1[o] = r;
            w.out[o] = w.lam0[o] + 0.5 * dte * r;
          } else if (w.stage == 2) {
            w.f2[o] = r;
            w.out[o] = w.lam0[o] + dte * r;
          } else {
            w.lam0[o] = w.lam0[o] + dte / 6.0 * (w.f0[o] + 2.0 * w.f1[o] + 2.0 * w.f2[o] + r);
          }
        }
      }
    }
  }
  if (w.mode == ADJ_DEFECT && w.norm_partial) block_sum_store<BT / 32>(dsq, w.norm_partial + blk);
}

template <int K, int P>
__global__ void __launch_bounds__(128) k_vjp_coords(const nzb_mesh m, const nzb_physics ph, const CoordWork w) {
  using S = Shape<K, P>;
  using D3 = Dual<3>;
  constexpr int NP = S::NP, NQV = S::NQV, NQF = S::NQF, NF = S::NF, NE = S::NE;
  const int64_t E = m.n_elem;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  int inst = -1;
  if (m.elem_inst) inst = __ldg(m.elem_inst + e);
  if (inst >= 0 && __ldg(m.inst_status + inst) != 0) return;
  const double p_back = (inst >= 0 && m.inst_p_back) ? __ldg(m.inst_p_back + inst) : ph.p_back;
  const double g = ph.gamma;
  const double* __restrict__ U = w.U;
  const double* __restrict__ L = w.lam;
  double xv[NF], yv[NF], gx[NF], gy[NF];
#pragma unroll
  for (int v = 0; v < NF; ++v) {
    xv[v] = __ldg(w.verts + v * E + e);
    yv[v] = __ldg(w.verts + (NF + v) * E + e);
    gx[v] = 0.0;
    gy[v] = 0.0;
  }
  // ---- volume: lam . R_vol = -sum_q [y_eta a - x_eta c - y_xi b + x_xi d],
  // a = Lxi . F, b = Leta . F, c = Lxi . G, d = Leta . G (weights folded into L)
#pragma unroll 1
  for (int q = 0; q < NQV; ++q) {
    double uq[4] = {0.0, 0.0, 0.0, 0.0}, lx[4] = {0.0, 0.0, 0.0, 0.0}, le[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double phi = c_tab[S::O_PHI + i * NQV + q];
      const double a = c_tab[S::O_WXI + i * NQV + q];
      const double b = c_tab[S::O_WETA + i * NQV + q];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double ls = __ldg(L + (s * NP + i) * E + e);
        uq[s] = fma(phi, __ldg(U + (s * NP + i) * E + e), uq[s]);
        lx[s] = fma(a, ls, lx[s]);
        le[s] = fma(b, ls, le[s]);
      }
    }
    double F[4], G[4];
    euler_flux(uq, g, F, G);
    double a = 0.0, b = 0.0, c = 0.0, d = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      a = fma(lx[s], F[s], a);
      b = fma(le[s], F[s], b);
      c = fma(lx[s], G[s], c);
      d = fma(le[s], G[s], d);
    }
#pragma unroll
    for (int v = 0; v < NF; ++v) {
      const double dx = c_tab[S::O_DGX + v * NQV + q], de = c_tab[S::O_DGE + v * NQV + q];
      gx[v] -= dx * d - de * c;
      gy[v] -= de * a - dx * b;
    }
  }
  // ---- edges this element owns
  double gp = 0.0;
#pragma unroll 1
  for (int f = 0; f < NF; ++f) {
    const int code = __ldg(m.face_code + f * E + e);
    if (code & 1) continue;  // the neighbour owns this edge
    const int k = __ldg(m.face_edge + f * E + e);
    const int nb = __ldg(m.face_nbr + f * E + e);
    const int nf = (code >> 1) & 7;
    const int tag = code >> 4;
    const double nx = __ldg(m.edge_geo + 4 * (int64_t)k + 0);
    const double ny = __ldg(m.edge_geo + 4 * (int64_t)k + 1);
    const double jac = __ldg(m.edge_geo + 4 * (int64_t)k + 2);
    double phi_sum = 0.0, gnx = 0.0, gny = 0.0, gpb = 0.0;
#pragma unroll 1
    for (int q = 0; q < NQF; ++q) {
      double tc[4] = {0.0, 0.0, 0.0, 0.0}, lc[4] = {0.0, 0.0, 0.0, 0.0};
      double tn[4] = {0.0, 0.0, 0.0, 0.0}, ln[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int j = 0; j < NE; ++j) {
        const double cc = pfe<K, P>(0, f, j, q);
        const int n = edge_node(K, P, f, j);
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          tc[s] = fma(cc, __ldg(U + (s * NP + n) * E + e), tc[s]);
          lc[s] = fma(cc, __ldg(L + (s * NP + n) * E + e), lc[s]);
        }
      }
      if (nb >= 0) {
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const double cc = pfe<K, P>(1, nf, j, q);
          const int n = edge_node(K, P, nf, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            tn[s] = fma(cc, __ldg(U + (s * NP + n) * E + nb), tn[s]);
            ln[s] = fma(cc, __ldg(L + (s * NP + n) * E + nb), ln[s]);
          }
        }
      }
      const double wq = c_tab[S::O_WF + q];
      // seeded on (n_x, n_y, p_back); the traces enter as plain numbers
      D3 F[4];
      const D3 dnx = D3::seed(nx, 0), dny = D3::seed(ny, 1);
      if (nb >= 0)
        interface_flux(tc, tn, dnx, dny, ph, F);
      else
        boundary_flux(tag, tc, dnx, dny, ph, D3::seed(p_back, 2), F);
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double xs = wq * (nb >= 0 ? lc[s] - ln[s] : lc[s]);
        phi_sum = fma(xs, F[s].v, phi_sum);
        gnx = fma(xs, F[s].d[0], gnx);
        gny = fma(xs, F[s].d[1], gny);
        gpb = fma(xs, F[s].d[2], gpb);
      }
    }
    // S = |t| phi(n(t)), n = (t_y, -t_x) / |t|:
    // dS/dt = phi t / |t| - ((G . t) / |t|) n
    double tx = 0.0, ty = 0.0;
#pragma unroll
    for (int v = 0; v < NF; ++v) {
      tx = fma(w.dgs[f][v], xv[v], tx);
      ty = fma(w.dgs[f][v], yv[v], ty);
    }
    const double r = sqrt(tx * tx + ty * ty);
    const double ux = tx / r, uy = ty / r;
    const double gt = gnx * ux + gny * uy;
    const double dtx = phi_sum * ux - gt * uy;
    const double dty = phi_sum * uy + gt * ux;
#pragma unroll
    for (int v = 0; v < NF; ++v) {
      gx[v] = fma(w.dgs[f][v], dtx, gx[v]);
      gy[v] = fma(w.dgs[f][v], dty, gy[v]);
    }
    gp = fma(jac, gpb, gp);
  }
#pragma unroll
  for (int v = 0; v < NF; ++v) {
    w.gvert[v * E + e] = gx[v];
    w.gvert[(NF + v) * E + e] = gy[v];
  }
  if (w.gpb) w.gpb[e] = gp;
}

}  // namespace nzb
