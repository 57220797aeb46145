// adjoint_split.cuh -- the state VJP kernel (k_vjp) with four threads per element.
//
// The layout of split.cuh: a block of four warps owns 32 elements, one per
// lane, and warp r does part r of each element's work, so every table operand
// is a warp-uniform constant-bank read.  Phases, separated by block barriers:
//
//   0  the block's U and lam are staged in shared memory (coalesced plane
//      loads: component s, node i, 32 consecutive elements);
//   A  warp r < NF differentiates face r's term at each of its points -- the
//      own traces of U and lam, the neighbour's (read from HBM once per face),
//      the flux in dual numbers seeded on the own trace -- and stores
//      a_u = sum_s xi_s dFhat_s/dU_u per point; a warp without a face
//      (triangles) takes the last volume points meanwhile; the volume points
//      are split over the warps, each storing b_u = (J_F^T cF + J_G^T cG)_u;
//   B  warp r gathers component u = r of every node: the face terms (faces in
//      turn, points in turn, the element's basis of its side of the face),
//      then the volume terms phi_iq b_u(q) -- the order k_vjp accumulates
//      them in -- and applies the epilogue of the mode to component u (the
//      product, the defect, the rate -M^-1 (v - dJ/dU), or an RK4 stage).
//
// The per-point arithmetic is k_vjp's, and each output is accumulated in
// k_vjp's order, so the two agree to the compiler's contraction choices; the
// defect's per-element sum of squares is summed by component first.
#pragma once
#include "adjoint.cuh"
#include "split.cuh"

#ifndef NZB_MINB_VJPS
#define NZB_MINB_VJPS 2
#endif

namespace nzb {

template <int K, int P>
struct VjpSplitSmem {
  using S = Shape<K, P>;
  static constexpr int U = 0;                                  // [NP*4]  state, slot i*4+s
  static constexpr int L = U + S::NP * 4 * SPLIT_EB;           // [NP*4]  lambda
  static constexpr int A = L + S::NP * 4 * SPLIT_EB;           // [NF*NQF*4] face terms a_u
  static constexpr int B = A + S::NF * S::NQF * 4 * SPLIT_EB;  // [NQV*4] volume terms b_u
  static constexpr int NRM = B;                                // after phase B: defect partials [4]
  static constexpr int TOTAL = B + S::NQV * 4 * SPLIT_EB;
  static constexpr int BYTES = TOTAL * 8;
  // resident blocks per SM asked of the compiler: the dual-number flux needs
  // about 200 registers, so NZB_MINB_VJPS (default 2: 255 registers, no
  // spills) rather than what the shared memory would allow
  static constexpr int BLOCKS = (228 * 1024) / (BYTES + 1024) < NZB_MINB_VJPS ? (228 * 1024) / (BYTES + 1024)
                                                                               : NZB_MINB_VJPS;
  static constexpr int MINB = BLOCKS < 1 ? 1 : BLOCKS;
};

// Volume points [Q0, Q0 + NQ): b_u at each, into the B slots.
template <int K, int P, bool AFF, int Q0, int NQ>
__device__ __forceinline__ void vjp_split_volume(const double* uc, const double* lcol, double* bcol, const nzb_mesh& m,
                                                 int64_t e, bool active, double g) {
  using S = Shape<K, P>;
  using D4 = Dual<4>;
  constexpr int NP = S::NP, NQV = S::NQV, NF = S::NF;
  const int64_t E = m.n_elem;
  double xx = 0, xy = 0, yx = 0, yy = 0, det = 1.0;
  double xv[NF], yv[NF];
#pragma unroll
  for (int v = 0; v < NF; ++v) xv[v] = yv[v] = 0.0;
  if (active) {
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
  }
  const double vs = AFF ? -det : -1.0;
#pragma unroll 1
  for (int q = Q0; q < Q0 + NQ; ++q) {
    double uq[4] = {0.0, 0.0, 0.0, 0.0}, lx[4] = {0.0, 0.0, 0.0, 0.0}, le[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double phi = c_tab[S::O_PHI + i * NQV + q];
      const double a = c_tab[S::O_WXI + i * NQV + q];
      const double b = c_tab[S::O_WETA + i * NQV + q];
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double us = uc[(i * 4 + s) * SPLIT_EB];
        const double ls = lcol[(i * 4 + s) * SPLIT_EB];
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
    double b[4] = {0.0, 0.0, 0.0, 0.0};
    if (active && !euler_flux_vjp(uq, g, cF, cG, b)) {
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
    for (int u = 0; u < 4; ++u) bcol[(q * 4 + u) * SPLIT_EB] = b[u];
  }
}

template <int K, int P, bool AFF>
__global__ void __launch_bounds__(SPLIT_T * 32, VjpSplitSmem<K, P>::MINB)
    k_vjp_split(const nzb_mesh m, const nzb_physics ph, const AdjWork w) {
  using S = Shape<K, P>;
  using L = VjpSplitSmem<K, P>;
  using PL = SplitPlan<K, P>;
  using D4 = Dual<4>;
  constexpr int NP = S::NP, NQV = S::NQV, NQF = S::NQF, NF = S::NF, NE = S::NE;
  constexpr int EB = SPLIT_EB;
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31, r = threadIdx.x >> 5;
  const int64_t E = m.n_elem;
  const int64_t blk = listed_block(m.vjp_blocks, E, EB);
  const int64_t e = blk * EB + lane;
  int inst = -1;
  if (e < E && m.elem_inst) inst = __ldg(m.elem_inst + e);
  const bool active = e < E && (inst < 0 || __ldg(m.inst_status + inst) == 0);
  // a block whose 32 elements are all retired (or past the end) has nothing to do: it leaves before
  // its first barrier, together (the test is block-uniform)
  if (!__syncthreads_or(active)) return;
  const double g = ph.gamma;
  double* const uc = smem + L::U + lane;
  double* const lcol = smem + L::L + lane;

  // ---- phase 0: U and lambda into shared memory
#pragma unroll
  for (int c = r; c < NP * 4; c += SPLIT_T) {
    const int i = c >> 2, s = c & 3;
    const int64_t o = ((int64_t)s * NP + i) * E + e;
    uc[c * EB] = active ? __ldg(w.U + o) : 0.0;
    lcol[c * EB] = active ? __ldg(w.lam + o) : 0.0;
  }
  __syncthreads();

  int sides = 0;
  if (active) sides = face_sides<K, P>(m, e);

  // ---- phase A: face r's terms, or the last volume points for a warp without a face
  if (r < NF) {
    const int f = r;
    double* acol = smem + L::A + f * NQF * 4 * EB + lane;
    if (active) {
      const int code = __ldg(m.face_code + f * E + e);
      const int k = __ldg(m.face_edge + f * E + e);
      const int nb = __ldg(m.face_nbr + f * E + e);
      const int side = code & 1;
      const int nf = (code >> 1) & 7;
      const int tag = code >> 4;
      const double nx = __ldg(m.edge_geo + 4 * (int64_t)k + 0);
      const double ny = __ldg(m.edge_geo + 4 * (int64_t)k + 1);
      const double jac = __ldg(m.edge_geo + 4 * (int64_t)k + 2);
      const double p_back = (inst >= 0 && m.inst_p_back) ? __ldg(m.inst_p_back + inst) : ph.p_back;
      double un[NE][4], lnb[NE][4];
      if (nb >= 0) {
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const int n = edge_node(K, P, nf, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            un[j][s] = __ldg(w.U + (s * NP + n) * E + nb);
            lnb[j][s] = __ldg(w.lam + (s * NP + n) * E + nb);
          }
        }
      }
      int own_node[NE];
#pragma unroll
      for (int j = 0; j < NE; ++j) own_node[j] = edge_node(K, P, f, j);
#pragma unroll 1
      for (int q = 0; q < NQF; ++q) {
        double tc[4] = {0.0, 0.0, 0.0, 0.0}, lc[4] = {0.0, 0.0, 0.0, 0.0};
        double tn[4] = {0.0, 0.0, 0.0, 0.0}, ln[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const double c = pfe<K, P>(side, f, j, q);
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            tc[s] = fma(c, uc[(own_node[j] * 4 + s) * EB], tc[s]);
            lc[s] = fma(c, lcol[(own_node[j] * 4 + s) * EB], lc[s]);
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
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          double acc = 0.0;
#pragma unroll
          for (int s = 0; s < 4; ++s) acc = fma(xi[s], F[s].d[u], acc);
          acol[(q * 4 + u) * EB] = acc;
        }
      }
    } else {
#pragma unroll
      for (int q = 0; q < NQF; ++q)
#pragma unroll
        for (int u = 0; u < 4; ++u) acol[(q * 4 + u) * EB] = 0.0;
    }
  } else {
    constexpr int n1 = PL::LATE;
    if constexpr (n1 > 0)
      vjp_split_volume<K, P, AFF, NQV - n1, n1>(uc, lcol, smem + L::B + lane, m, e, active, g);
  }
  for_part(r, [&](auto R) {
    constexpr SplitRanges pr = PL::even(NQV - PL::LATE);
    constexpr int q0 = pr.first[decltype(R)::value], nq = pr.count[decltype(R)::value];
    if constexpr (nq > 0) vjp_split_volume<K, P, AFF, q0, nq>(uc, lcol, smem + L::B + lane, m, e, active, g);
  });
  __syncthreads();

  // ---- phase B: component u = r of every node, in k_vjp's order (faces, then volume points)
  const int u = r;
  double acc[NP];
#pragma unroll
  for (int i = 0; i < NP; ++i) acc[i] = 0.0;
#pragma unroll
  for (int f = 0; f < NF; ++f) {
    const bool sd = (sides >> f) & 1;
#pragma unroll
    for (int q = 0; q < NQF; ++q) {
      const double a = smem[L::A + ((f * NQF + q) * 4 + u) * EB + lane];
#pragma unroll
      for (int j = 0; j < NE; ++j) {
        const double c = pfe<K, P>(sd ? 1 : 0, f, j, q);
        const int n = edge_node(K, P, f, j);
        acc[n] = fma(c, a, acc[n]);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NQV; ++q) {
    const double b = smem[L::B + (q * 4 + u) * EB + lane];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = fma(c_tab[S::O_PHI + i * NQV + q], b, acc[i]);
  }

  double dsq = 0.0;
  if (active) {
    if (w.mode == ADJ_VJP) {
#pragma unroll
      for (int i = 0; i < NP; ++i) w.out[((int64_t)u * NP + i) * E + e] = acc[i];
    } else if (w.mode == ADJ_DEFECT) {
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        const int64_t o = ((int64_t)u * NP + i) * E + e;
        const double d = acc[i] - __ldg(w.seed + o);
        if (w.out) w.out[o] = d;
        dsq = fma(d, d, dsq);
      }
    } else {
      const double dte = w.mode == ADJ_RK4 ? __ldg(w.dt + e) : 0.0;
      const double det = AFF ? __ldg(m.geo + 4 * E + e) : 1.0;
      double d[NP];
#pragma unroll
      for (int j = 0; j < NP; ++j) d[j] = acc[j] - __ldg(w.seed + ((int64_t)u * NP + j) * E + e);
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        double rr = 0.0;
        if (AFF) {
#pragma unroll
          for (int j = 0; j < NP; ++j) rr = fma(tab<K, P>(S::O_MINV + i * NP + j), d[j], rr);
          rr = -(rr / det);
        } else {
#pragma unroll
          for (int j = 0; j < NP; ++j) rr = fma(__ldg(m.minv + ((int64_t)i * NP + j) * E + e), d[j], rr);
          rr = -rr;
        }
        const int64_t o = ((int64_t)u * NP + i) * E + e;
        if (w.mode == ADJ_RATE) {
          w.out[o] = rr;
        } else if (w.stage == 0) {
          w.f0[o] = rr;
          w.out[o] = w.lam0[o] + 0.5 * dte * rr;
        } else if (w.stage == 1) {
          w.f1[o] = rr;
          w.out[o] = w.lam0[o] + 0.5 * dte * rr;
        } else if (w.stage == 2) {
          w.f2[o] = rr;
          w.out[o] = w.lam0[o] + dte * rr;
        } else {
          w.lam0[o] = w.lam0[o] + dte / 6.0 * (w.f0[o] + 2.0 * w.f1[o] + 2.0 * w.f2[o] + rr);
        }
      }
    }
  }
  if (w.mode == ADJ_DEFECT && (w.elem_norm || w.norm_partial)) {
    // the element's sum of squares over its four components (B slots are free after phase B)
    __syncthreads();
    smem[L::NRM + r * EB + lane] = dsq;
    __syncthreads();
    double tot = 0.0;
    if (r == 0) {
#pragma unroll
      for (int k = 0; k < SPLIT_T; ++k) tot += smem[L::NRM + k * EB + lane];
      if (w.elem_norm && active) w.elem_norm[e] = tot;
    }
    if (w.norm_partial) block_sum_store<SPLIT_T>(tot, w.norm_partial + blk);
  }
}

}  // namespace nzb
