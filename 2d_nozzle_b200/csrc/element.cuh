// element.cuh -- the fused element kernel: volume term, face fluxes, lift,
// inverse mass, stage update and positivity limiter in one pass per element.
//
// One thread owns one element.  Its NP x 4 coefficients and NP x 4 residual
// accumulators live in registers; the volume loops are fully unrolled, so each
// reference-element table entry is a constant-bank operand at a compile-time
// address and every multiply-add is a single DFMA with no load.  The face
// integral is computed from the element's own side in a rolled loop (one copy
// of the flux code): both traces are formed from the p + 1 coefficients on the
// shared edge -- the neighbour's read straight from HBM/L2 -- and the flux is
// evaluated with the owner's trace as the left state and the owner's normal,
// so both elements of an edge compute bit-identical fluxes and the scheme stays
// conservative with no edge array and no second pass.  The lift accumulates in
// a per-thread column of shared memory.
//
// Mathematics (src/spatial/assembly.py:52-162, src/backends/_numba_kernels.py:
// 484-777): R_i = -sum_q (gx_iq F_q + gy_iq G_q) + sum_f sign_f sum_q phi_f,iq fw_q
// with fw = flux * |dX/dsigma| * w_q, the rate -M^-1 R, and
// wave = sum_f max_q s_q * length_f, where gx = w det (dphi/dxi xi_x +
// dphi/deta eta_x).  Geometry comes in two layouts:
//   affine  (straight-sided triangles): xi_x, xi_y, eta_x, eta_y, det per
//           element; M = det M_ref, so M^-1 is a table divided by det;
//   general (bilinear quadrilaterals, or any straight-sided element): the
//           vertex coordinates, from which every volume point's Jacobian is
//           rebuilt (det * (xi_x, xi_y) = (y_eta, -x_eta) needs no division),
//           and the element's inverse mass matrix.
#pragma once
#include "physics.cuh"
#include "shapes.cuh"

namespace nzb {

// one copy per translation unit (each is uploaded by nzb_upload_tables)
static __constant__ double c_tab[TABLE_DOUBLES];

enum { OP_RESIDUAL = 0, OP_RATE = 1, OP_STAGE = 2, OP_LIMIT = 3 };

struct Work {
  int op;
  const double* V;   // state the rate is evaluated at
  const double* U0;  // step start state (stages 2 and 3)
  double* out;
  double* wave;
  double* dt;
  double* norm_partial;
  double* elem_norm;  // per-element stage-1 norm contribution (batches)
  unsigned long long* counters;
  uint8_t* flags;
  double dt_factor, a, b;
  int stage;
};

template <int K, int P>
__device__ __forceinline__ double tab(int idx) {
  return c_tab[idx];
}

// Reference face basis phi_face[side, f, edge_node(f, j), q] (runtime indices).
template <int K, int P>
__device__ __forceinline__ double pfe(int side, int f, int j, int q) {
  using S = Shape<K, P>;
  return c_tab[S::O_PFE + ((side * S::NF + f) * S::NE + j) * S::NQF + q];
}

// An element's coefficients as the limiter reads and writes them: a register
// array, or this thread's column of a shared-memory block (stride BT), where a
// kernel keeps them to leave registers free.
template <int NP>
struct RegCoef {
  double (&u)[NP][4];
  __device__ __forceinline__ double& operator()(int i, int s) const { return u[i][s]; }
};
template <int BT>
struct SmemCoef {
  double* col;  // &block[t]
  __device__ __forceinline__ double& operator()(int i, int s) const { return col[(i * 4 + s) * BT]; }
};

// One probe point of this element's solution: volume point pt < NQV, else the
// element's own trace at face point (f, q), with the basis of its side of that
// face (bit f of sides), as the reference's probe set (src/spatial/limiter.py:
// 78-95).  pt is the same on every lane of a warp (the loops over points are
// rolled), so the table reads are constant-cache broadcasts.
template <int K, int P, class A>
__device__ __forceinline__ void probe_point(const A& u, int pt, int sides, double (&w)[4]) {
  using S = Shape<K, P>;
  w[0] = w[1] = w[2] = w[3] = 0.0;
  if (pt < S::NQV) {
#pragma unroll
    for (int i = 0; i < S::NP; ++i) {
      const double phi = c_tab[S::O_PHI + i * S::NQV + pt];
#pragma unroll
      for (int s = 0; s < 4; ++s) w[s] = fma(phi, u(i, s), w[s]);
    }
  } else {
    const int f = (pt - S::NQV) / S::NQF, q = (pt - S::NQV) - f * S::NQF;
    const int side = (sides >> f) & 1;
#pragma unroll
    for (int j = 0; j < S::NE; ++j) {
      const double l = pfe<K, P>(side, f, j, q);
      // u at a runtime node: select among the unrolled candidates
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int ff = 0; ff < S::NF; ++ff) {
        if (ff == f) {
          const int nn = edge_node(K, P, ff, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) v[s] = u(nn, s);
        }
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) w[s] = fma(l, v[s], w[s]);
    }
  }
}

__device__ __forceinline__ double pressure_at(const double (&w)[4], double g) {
  const double r = w[0] < 1e-300 ? 1e-300 : w[0];
  return (g - 1.0) * (w[3] - 0.5 * (w[1] * w[1] + w[2] * w[2]) / r);
}

// Minimum pressure over the probe set of ubar + theta (u - ubar), through the
// reference's scaling formula (src/spatial/limiter.py:146-148,151-178).
template <int K, int P, class A>
__device__ __forceinline__ double pmin_at(const A& u, const double (&ub)[4], double theta,
                                          int sides, double g) {
  double pmin = 1e300;
#pragma unroll 1
  for (int pt = 0; pt < Shape<K, P>::NPROBE; ++pt) {
    double w[4];
    probe_point<K, P>(u, pt, sides, w);
#pragma unroll
    for (int s = 0; s < 4; ++s) w[s] = ub[s] + theta * (w[s] - ub[s]);
    const double pp = pressure_at(w, g);
    pmin = pp < pmin ? pp : pmin;
  }
  return pmin;
}

// One pass over the probe points: the raw minima the reference's violation
// test uses (src/spatial/limiter.py:224-228), and t*, the smallest positive t
// at which p(ubar + t (w - ubar)) = eps_p at some point w.  Along the segment
// h(t) = rho(t) (p(t) - eps_p) / (gamma - 1) = a t^2 + b t + c with
// h(0) = rho_bar (p_bar - eps_p) / (gamma - 1) > 0; t* = 1e300 when no point binds.
template <int K, int P, class A>
__device__ __forceinline__ void probe_scan(const A& u, const double (&ub)[4], int sides,
                                           double eps_p, double g, double& rmin, double& pmin, double& tstar) {
  const double e1 = eps_p / (g - 1.0);
  const double c = ub[3] * ub[0] - 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) - e1 * ub[0];
  rmin = 1e300;
  pmin = 1e300;
  tstar = 1e300;
#pragma unroll 1
  for (int pt = 0; pt < Shape<K, P>::NPROBE; ++pt) {
    double w[4];
    probe_point<K, P>(u, pt, sides, w);
    rmin = w[0] < rmin ? w[0] : rmin;
    const double pp = pressure_at(w, g);
    pmin = pp < pmin ? pp : pmin;
    // when the segment starts inside the bound (c > 0: the cell mean's
    // pressure exceeds eps_p), a point with positive density that meets the
    // bound at t = 1 cannot bind on (0, 1] (p is concave along the segment);
    // t <= theta <= 1 in every comparison with t*, so its root is not needed
    if (c > 0.0 && !(pp < eps_p) && w[0] > 0.0) continue;
    const double d0 = w[0] - ub[0], d1 = w[1] - ub[1], d2 = w[2] - ub[2], d3 = w[3] - ub[3];
    const double a = d3 * d0 - 0.5 * (d1 * d1 + d2 * d2);
    const double b = ub[3] * d0 + ub[0] * d3 - (ub[1] * d1 + ub[2] * d2) - e1 * d0;
    // h stays positive for t > 0 when it starts increasing and curves up
    if (a >= 0.0 && b >= 0.0) continue;
    const double disc = b * b - 4.0 * a * c;
    if (disc < 0.0) continue;
    const double q = -0.5 * (b + copysign(sqrt(disc), b));
    const double r1 = a != 0.0 ? q / a : 1e300, r2 = q != 0.0 ? c / q : 1e300;
    const double p1 = r1 > 0.0 ? r1 : 1e300, p2 = r2 > 0.0 ? r2 : 1e300;
    const double t = p1 < p2 ? p1 : p2;
    tstar = t < tstar ? t : tstar;
  }
}

// Jacobian of the element map at volume point q (general geometry, Q = 1),
// from the vertex coordinates: returns det = x_xi y_eta - x_eta y_xi.
template <int K, int P>
__device__ __forceinline__ double point_det(const double (&xv)[Shape<K, P>::NF], const double (&yv)[Shape<K, P>::NF],
                                            int q, double& x_xi, double& x_eta, double& y_xi, double& y_eta) {
  using S = Shape<K, P>;
  x_xi = x_eta = y_xi = y_eta = 0.0;
#pragma unroll
  for (int v = 0; v < S::NF; ++v) {
    const double dx = tab<K, P>(S::O_DGX + v * S::NQV + q), de = tab<K, P>(S::O_DGE + v * S::NQV + q);
    x_xi = fma(dx, xv[v], x_xi);
    x_eta = fma(de, xv[v], x_eta);
    y_xi = fma(dx, yv[v], y_xi);
    y_eta = fma(de, yv[v], y_eta);
  }
  return x_xi * y_eta - x_eta * y_xi;
}

// Cell-average weights of element e: a table for affine elements (M = det
// M_ref), else sum_q phi_iq w_q det_q / area, as the reference builds them
// (src/spatial/operators.py:283-287).
template <int K, int P, bool AFF>
__device__ __forceinline__ void mean_weights(const nzb_mesh& m, int64_t e, double (&mw)[Shape<K, P>::NP]) {
  using S = Shape<K, P>;
  const int64_t E = m.n_elem;
  if (AFF) {
#pragma unroll
    for (int i = 0; i < S::NP; ++i) mw[i] = tab<K, P>(S::O_MW + i);
  } else {
    double xv[S::NF], yv[S::NF];
#pragma unroll
    for (int v = 0; v < S::NF; ++v) {
      xv[v] = __ldg(m.geo + v * E + e);
      yv[v] = __ldg(m.geo + (S::NF + v) * E + e);
    }
#pragma unroll
    for (int i = 0; i < S::NP; ++i) mw[i] = 0.0;
#pragma unroll
    for (int q = 0; q < S::NQV; ++q) {
      double a, b, c, d;
      const double wdet = tab<K, P>(S::O_WV + q) * point_det<K, P>(xv, yv, q, a, b, c, d);
#pragma unroll
      for (int i = 0; i < S::NP; ++i) mw[i] = fma(tab<K, P>(S::O_PHI + i * S::NQV + q), wdet, mw[i]);
    }
    const double area = __ldg(m.area + e);
#pragma unroll
    for (int i = 0; i < S::NP; ++i) mw[i] = mw[i] / area;
  }
}

// Zhang-Shu positivity limiter of one element, in place
// (src/spatial/limiter.py:103-243; the O(NP) Lebesgue screen of
// src/backends/_numba_kernels.py:1010-1026 skips provably admissible elements).
template <int K, int P, bool AFF, class A>
__device__ __forceinline__ void limit_element(const A& u, const nzb_mesh& m,
                                              const nzb_physics& ph, int64_t e, int sides, int& scaled,
                                              int& repaired) {
  using S = Shape<K, P>;
  const double g = ph.gamma;
  const int64_t E = m.n_elem;
  double mw[S::NP];
  mean_weights<K, P, AFF>(m, e, mw);
  double ub[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < S::NP; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) ub[s] = fma(mw[i], u(i, s), ub[s]);

  // last-resort repair of a non-physical cell average
  const double rho_new = ub[0] < ph.rho_floor ? ph.rho_floor : ub[0];
  const double e_min = ph.p_floor / (g - 1.0) + 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) / rho_new;
  const double rhoE_new = ub[3] < e_min ? e_min : ub[3];
  if (ub[0] < ph.rho_floor || ub[3] < e_min) {
    const double d0 = rho_new - ub[0], d3 = rhoE_new - ub[3];
#pragma unroll
    for (int i = 0; i < S::NP; ++i) {
      u(i, 0) += d0;
      u(i, 3) += d3;
    }
    repaired = 1;
#pragma unroll
    for (int s = 0; s < 4; ++s) ub[s] = 0.0;
#pragma unroll
    for (int i = 0; i < S::NP; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) ub[s] = fma(mw[i], u(i, s), ub[s]);
  }
  const double pbar = (g - 1.0) * (ub[3] - 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) / ub[0]);
  double eps_r = ph.lim_fraction * ub[0];
  eps_r = eps_r < 0.5 * ph.rho_floor ? 0.5 * ph.rho_floor : eps_r;
  double eps_p = ph.lim_fraction * pbar;
  eps_p = eps_p < 0.5 * ph.p_floor ? 0.5 * ph.p_floor : eps_p;

  // sufficient screen: bound every probe through the Lebesgue constant
  double dev[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < S::NP; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) dev[s] = fmax(dev[s], fabs(u(i, s) - ub[s]));
  const double lam = ph.lebesgue;
  const double rho_lo = ub[0] - lam * dev[0];
  if (rho_lo >= eps_r) {
    const double m_hi = sqrt(ub[1] * ub[1] + ub[2] * ub[2]) + lam * sqrt(dev[1] * dev[1] + dev[2] * dev[2]);
    const double p_lo = (g - 1.0) * (ub[3] - lam * dev[3] - 0.5 * m_hi * m_hi / rho_lo);
    if (p_lo >= eps_p) return;
  }
  double rmin, pmin, tstar;
  probe_scan<K, P>(u, ub, sides, eps_p, g, rmin, pmin, tstar);
  if (!(rmin < eps_r) && !(pmin < eps_p)) return;

  double theta = 1.0;
  if (rmin < eps_r) {
    const double gap = ub[0] - rmin;
    theta = (ub[0] - eps_r) / (gap > 0.0 ? gap : 1.0);
    theta = theta < 0.0 ? 0.0 : (theta > 1.0 ? 1.0 : theta);
  }
  // The reference bisects on min_x p(ubar + t (u(x) - ubar)) >= eps_p over
  // [0, theta] (12 steps, src/spatial/limiter.py:151-178).  p is concave along
  // the segment, so that test is exactly "t <= t*" for one t* per element, and
  // t* is the smallest positive root over the probe points of the quadratic
  // rho(t) (p(t) - eps_p).  The probe scan above found t*; the bisection is then
  // replayed on the scalar t* with the reference's own midpoints.  A decision
  // within 1e-7 theta of t* -- where the root's rounding could disagree with
  // the reference's pointwise arithmetic -- is taken with that arithmetic.
  auto admissible = [&](double t) -> bool {
    if (fabs(t - tstar) > 1e-7 * theta) return t < tstar;
    return pmin_at<K, P>(u, ub, t, sides, g) >= eps_p;
  };
  if (!admissible(theta)) {
    double lo = 0.0, hi = theta;
    for (int it = 0; it < ph.lim_steps; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (admissible(mid))
        lo = mid;
      else
        hi = mid;
    }
    theta = lo;
  }
#pragma unroll
  for (int i = 0; i < S::NP; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) u(i, s) = ub[s] + theta * (u(i, s) - ub[s]);
  scaled = 1;
}

// The block of the mesh this CTA runs: entry blockIdx.x of a block list (the
// blocks of a batch that still hold marching elements), or blockIdx.x itself.
// An entry outside [0, ceil(E / W)) maps to the first block past the end, whose
// elements are all inactive.
__device__ __forceinline__ int64_t listed_block(const int32_t* __restrict__ list, int64_t E, int W) {
  if (!list) return blockIdx.x;
  const int64_t end = (E + W - 1) / W;
  const int64_t b = __ldg(list + blockIdx.x);
  return (b < 0 || b > end) ? end : b;
}

template <int NW>
__device__ __forceinline__ void block_sum_store(double v, double* dst) {
  __shared__ double red[NW];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < NW; ++k) t += red[k];
    *dst = t;
  }
}

// Start a global cache line toward L2; no register holds it.  The adjoint
// kernel issues these at entry for operands it reads only in its epilogue.
__device__ __forceinline__ void prefetch_line(const double* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// Threads per block: 128, or 64 where the per-thread face accumulator would
// push static shared memory past 48 KB (cubic quadrilaterals).
//
// MINB_* is the minimum of resident blocks per SM asked of the compiler
// (__launch_bounds__), which caps registers per thread at 65536 / (MINB * NT).
#ifndef NZB_MINB_RES
#define NZB_MINB_RES 1
#endif
#ifndef NZB_MINB_STAGE
#define NZB_MINB_STAGE 1
#endif
// Resident 128-thread blocks per SM asked of the compiler for the edge pass:
// 4 caps it at 128 registers (from 168, with a few spills), 16 warps per SM
// instead of 12 -- measured 14 % faster on 1 M linear triangles.
#ifndef NZB_MINB_EDGE
#define NZB_MINB_EDGE 4
#endif

template <int K, int P>
struct Launch {
  static constexpr int NP = Shape<K, P>::NP;
  static constexpr int NT = (NP * 4 * 8 * 128 <= 40 * 1024) ? 128 : 64;
  // counted in 128-thread blocks: a 64-thread block asks for twice as many
  static constexpr int MINB_RES = NZB_MINB_RES * 128 / NT;
  static constexpr int MINB_STAGE = NZB_MINB_STAGE * 128 / NT;
};

// Face bits of this element (bit f = its side of face f) from the mesh arrays.
template <int K, int P>
__device__ __forceinline__ int face_sides(const nzb_mesh& m, int64_t e) {
  int sides = 0;
#pragma unroll
  for (int f = 0; f < Shape<K, P>::NF; ++f) sides |= (__ldg(m.face_code + f * m.n_elem + e) & 1) << f;
  return sides;
}

// The edge pass: one thread per edge evaluates the numerical flux at the
// edge's points, once -- the owner's trace (phi_face[0, f]) as the left state,
// the neighbour's (phi_face[1, nf]) as the right, the owner's normal -- and
// stores w_q |dX/dsigma| Fhat (edge_flux, (n_edge, NQF, 4): an edge's values
// contiguous, read as whole 32-byte sectors by both its elements) and max_q s_q
// (edge_speed), the reference's edge_pass (src/backends/_numba_kernels.py:
// 484-583).  The element kernel with EP = true lifts them.  The arithmetic is
// the fused kernel's, so both variants agree to round-off.
template <int K, int P>
__global__ void __launch_bounds__(128, NZB_MINB_EDGE) k_edge(const nzb_mesh m, const nzb_physics ph, const double* __restrict__ V) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP, NQF = S::NQF, NE = S::NE;
  const int64_t NK = m.n_edge, E = m.n_elem;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= NK) return;
  const int own = __ldg(m.edge_conn + k);
  const int nb = __ldg(m.edge_conn + NK + k);
  const int code = __ldg(m.edge_conn + 2 * NK + k);
  const int f = code & 7, nf = (code >> 3) & 7, tag = code >> 6;
  int inst = -1;
  if (m.elem_inst) inst = __ldg(m.elem_inst + own);
  if (inst >= 0 && __ldg(m.inst_status + inst) != 0) return;
  const double p_back = (inst >= 0 && m.inst_p_back) ? __ldg(m.inst_p_back + inst) : ph.p_back;
  const double nx = __ldg(m.edge_geo + 4 * k + 0);
  const double ny = __ldg(m.edge_geo + 4 * k + 1);
  const double jac = __ldg(m.edge_geo + 4 * k + 2);
  double uo[NE][4], un[NE][4];
#pragma unroll
  for (int j = 0; j < NE; ++j) {
    const int n = edge_node(K, P, f, j);
#pragma unroll
    for (int s = 0; s < 4; ++s) uo[j][s] = __ldg(V + (s * NP + n) * E + own);
  }
  if (nb >= 0) {
#pragma unroll
    for (int j = 0; j < NE; ++j) {
      const int n = edge_node(K, P, nf, j);
#pragma unroll
      for (int s = 0; s < 4; ++s) un[j][s] = __ldg(V + (s * NP + n) * E + nb);
    }
  }
  double smax = 0.0;
#pragma unroll 1
  for (int q = 0; q < NQF; ++q) {
    double tc[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < NE; ++j) {
      const double c = pfe<K, P>(0, f, j, q);
#pragma unroll
      for (int s = 0; s < 4; ++s) tc[s] = fma(c, uo[j][s], tc[s]);
    }
    double F[4], sp;
    if (nb >= 0) {
      double tn[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int j = 0; j < NE; ++j) {
        const double c = pfe<K, P>(1, nf, j, q);
#pragma unroll
        for (int s = 0; s < 4; ++s) tn[s] = fma(c, un[j][s], tn[s]);
      }
      sp = interface_flux(tc, tn, nx, ny, ph, F);
    } else {
      sp = boundary_flux(tag, tc, nx, ny, ph, p_back, F);
    }
    smax = sp > smax ? sp : smax;
    const double scale = jac * c_tab[S::O_WF + q];
    double2* dst = reinterpret_cast<double2*>(m.edge_flux + ((int64_t)k * NQF + q) * 4);
    dst[0] = make_double2(F[0] * scale, F[1] * scale);
    dst[1] = make_double2(F[2] * scale, F[3] * scale);
  }
  m.edge_speed[k] = smax;
}

// LIM = false compiles the residual / rate variant, without the stage update
// and the limiter (a smaller kernel: fewer registers, no instruction-cache
// pressure from code it never runs); LIM = true handles stages and the limiter.
template <int K, int P, bool AFF, bool LIM, bool EP>
__global__ void __launch_bounds__(Launch<K, P>::NT, LIM ? Launch<K, P>::MINB_STAGE : Launch<K, P>::MINB_RES)
    k_element(const nzb_mesh m, const nzb_physics ph, const Work w) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP, NQV = S::NQV, NQF = S::NQF, NF = S::NF, NE = S::NE;
  constexpr int BT = Launch<K, P>::NT;
  // face contributions, one column per thread: facc[(i * 4 + s) * BT + t]
  __shared__ double facc[NP * 4 * BT];
  const int t = threadIdx.x;
  const int64_t E = m.n_elem;
  const int64_t blk = listed_block(m.fwd_blocks, E, BT);
  const int64_t e = blk * BT + t;
  // a retired instance of a batch is left untouched
  int inst = -1;
  if (e < E && m.elem_inst) inst = __ldg(m.elem_inst + e);
  const bool active = e < E && (inst < 0 || __ldg(m.inst_status + inst) == 0);
  const double p_back = (inst >= 0 && m.inst_p_back) ? __ldg(m.inst_p_back + inst) : ph.p_back;
  const double g = ph.gamma;
  double nrm = 0.0;
  int scaled = 0, repaired = 0;

  if (LIM && active && w.op == OP_LIMIT) {
    double u[NP][4];
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) u[i][s] = w.V[(s * NP + i) * E + e];
    if (ph.limiter == 1 && P > 0)
      limit_element<K, P, AFF>(RegCoef<NP>{u}, m, ph, e, face_sides<K, P>(m, e), scaled, repaired);
#pragma unroll
    for (int i = 0; i < NP; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) w.out[(s * NP + i) * E + e] = u[i][s];
    if (w.flags) w.flags[e] = (uint8_t)(scaled | (repaired << 1));
  } else if (active) {
    const bool rate = w.op != OP_RESIDUAL;
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
#pragma unroll
    for (int i = 0; i < NP * 4; ++i) facc[i * BT + t] = 0.0;

    // ---- face terms: a rolled loop over (face, point), so the flux code is
    // inlined once.  Traces use the reference's face basis phi_face[side, f] at
    // the p + 1 edge nodes; the lift goes to the shared-memory column.
    const double fs = (AFF && rate) ? -1.0 / det : 1.0;
    double wave = 0.0;
    int sides = 0;
    if constexpr (EP) {
      // the edge pass (k_edge) has left w |dX/dsigma| Fhat at every edge point
      // and max_q s_q per edge; lift them with this element's side of the face
#pragma unroll 1
      for (int f = 0; f < NF; ++f) {
        const int code = __ldg(m.face_code + f * E + e);
        const int k = __ldg(m.face_edge + f * E + e);
        const int side = code & 1;
        sides |= side << f;
        const double coef = (side ? -1.0 : 1.0) * fs;
#pragma unroll 1
        for (int q = 0; q < NQF; ++q) {
          const double2* src = reinterpret_cast<const double2*>(m.edge_flux + ((int64_t)k * NQF + q) * 4);
          const double2 f01 = __ldg(src), f23 = __ldg(src + 1);
          const double fwc[4] = {f01.x * coef, f01.y * coef, f23.x * coef, f23.y * coef};
#pragma unroll
          for (int j = 0; j < NE; ++j) {
            const double cj = pfe<K, P>(side, f, j, q);
            const int n = edge_node(K, P, f, j);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
              double& a = facc[(n * 4 + s) * BT + t];
              a = fma(cj, fwc[s], a);
            }
          }
        }
        wave += __ldg(m.edge_speed + k) * __ldg(m.edge_geo + 4 * (int64_t)k + 3);
      }
    } else {
#pragma unroll 1
    for (int f = 0; f < NF; ++f) {
      const int code = __ldg(m.face_code + f * E + e);
      const int k = __ldg(m.face_edge + f * E + e);
      const int nb = __ldg(m.face_nbr + f * E + e);
      const int side = code & 1;
      const int nf = (code >> 1) & 7;
      const int tag = code >> 4;
      sides |= side << f;
      const double nx = __ldg(m.edge_geo + 4 * (int64_t)k + 0);
      const double ny = __ldg(m.edge_geo + 4 * (int64_t)k + 1);
      const double jac = __ldg(m.edge_geo + 4 * (int64_t)k + 2);
      const double len = __ldg(m.edge_geo + 4 * (int64_t)k + 3);
      double ue[NE][4], un[NE][4];
      int node[NE];
#pragma unroll
      for (int j = 0; j < NE; ++j) {
        node[j] = edge_node(K, P, f, j);
#pragma unroll
        for (int s = 0; s < 4; ++s) ue[j][s] = __ldg(w.V + (s * NP + node[j]) * E + e);
      }
      if (nb >= 0) {
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          const int n = edge_node(K, P, nf, j);
#pragma unroll
          for (int s = 0; s < 4; ++s) un[j][s] = __ldg(w.V + (s * NP + n) * E + nb);
        }
      }
      const double coef = (side ? -1.0 : 1.0) * fs;
      double smax = 0.0;
#pragma unroll 1
      for (int q = 0; q < NQF; ++q) {
        // canonical (owner's) point q: own trace with phi_face[side, f],
        // the neighbour's with phi_face[1 - side, nf]
        double tc[4] = {0.0, 0.0, 0.0, 0.0}, tn[4] = {0.0, 0.0, 0.0, 0.0}, cj[NE];
#pragma unroll
        for (int j = 0; j < NE; ++j) {
          cj[j] = pfe<K, P>(side, f, j, q);
#pragma unroll
          for (int s = 0; s < 4; ++s) tc[s] = fma(cj[j], ue[j][s], tc[s]);
        }
        double F[4], sp;
        if (nb >= 0) {
#pragma unroll
          for (int j = 0; j < NE; ++j) {
            const double l = pfe<K, P>(1 - side, nf, j, q);
#pragma unroll
            for (int s = 0; s < 4; ++s) tn[s] = fma(l, un[j][s], tn[s]);
          }
          double L[4], R[4];
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            L[s] = side ? tn[s] : tc[s];
            R[s] = side ? tc[s] : tn[s];
          }
          sp = interface_flux(L, R, nx, ny, ph, F);
        } else {
          sp = boundary_flux(tag, tc, nx, ny, ph, p_back, F);
        }
        smax = sp > smax ? sp : smax;
        const double scale = jac * c_tab[S::O_WF + q];
        double fwc[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) fwc[s] = (F[s] * scale) * coef;
#pragma unroll
        for (int j = 0; j < NE; ++j)
#pragma unroll
          for (int s = 0; s < 4; ++s) {
            double& a = facc[(node[j] * 4 + s) * BT + t];
            a = fma(cj[j], fwc[s], a);
          }
      }
      wave += smax * len;
    }
    }
    if (w.wave) w.wave[e] = wave;

    // ---- volume term, fully unrolled, tables as constant-bank operands.
    // With NP >= 9 the coefficients and the accumulators together would not fit
    // in registers, so the coefficients move into this thread's shared-memory
    // column (free once its face sums are in the accumulators).
    constexpr bool USM = NP >= 9;
    double acc[NP][4];
    {
      double u[USM ? 1 : NP][4];
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          acc[i][s] = facc[(i * 4 + s) * BT + t];
          const double v = __ldg(w.V + (s * NP + i) * E + e);
          if constexpr (USM)
            facc[(i * 4 + s) * BT + t] = v;
          else
            u[i][s] = v;
        }
      auto coef = [&](int i, int s) -> double {
        if constexpr (USM)
          return facc[(i * 4 + s) * BT + t];
        else
          return u[i][s];
      };
      // affine: (xi_x F + xi_y G) det, det only for the residual (the rate
      // divides it out again); general: det (xi_x, xi_y) = (y_eta, -x_eta)
      const double vs = AFF ? (rate ? 1.0 : -det) : -1.0;
      // cubic quadrilaterals: a rolled point loop (64 accumulators leave no
      // room for a fully unrolled one)
      constexpr int QUNROLL = NP >= 16 ? 1 : NQV;
#pragma unroll QUNROLL
      for (int q = 0; q < NQV; ++q) {
        double uq[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const double phi = tab<K, P>(S::O_PHI + i * NQV + q);
#pragma unroll
          for (int s = 0; s < 4; ++s) uq[s] = fma(phi, coef(i, s), uq[s]);
        }
        const Prim pr = primitives_fast(uq, g);
        const double F[4] = {pr.rho * pr.vx, pr.rho * pr.vx * pr.vx + pr.p, pr.rho * pr.vx * pr.vy, pr.rho * pr.vx * pr.H};
        const double G[4] = {pr.rho * pr.vy, pr.rho * pr.vx * pr.vy, pr.rho * pr.vy * pr.vy + pr.p, pr.rho * pr.vy * pr.H};
        double a00 = xx, a01 = xy, a10 = yx, a11 = yy;
        if (!AFF) {
          double x_xi, x_eta, y_xi, y_eta;
          point_det<K, P>(xv, yv, q, x_xi, x_eta, y_xi, y_eta);
          a00 = y_eta;
          a01 = -x_eta;
          a10 = -y_xi;
          a11 = x_xi;
        }
        double fx[4], fe[4];
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          fx[s] = (a00 * F[s] + a01 * G[s]) * vs;
          fe[s] = (a10 * F[s] + a11 * G[s]) * vs;
        }
#pragma unroll
        for (int i = 0; i < NP; ++i) {
          const double a = tab<K, P>(S::O_WXI + i * NQV + q);
          const double b = tab<K, P>(S::O_WETA + i * NQV + q);
#pragma unroll
          for (int s = 0; s < 4; ++s) acc[i][s] = fma(a, fx[s], fma(b, fe[s], acc[i][s]));
        }
      }
    }

    if (w.op == OP_RESIDUAL) {
#pragma unroll
      for (int i = 0; i < NP; ++i)
#pragma unroll
        for (int s = 0; s < 4; ++s) w.out[(s * NP + i) * E + e] = acc[i][s];
    } else {
      double dt = 0.0;
      if (LIM && w.op == OP_STAGE) {
        if (w.stage == 1) {
          const double d = wave < FLOOR ? FLOOR : wave;
          dt = w.dt_factor * 2.0 * __ldg(m.area + e) / d;
          w.dt[e] = dt;
        } else {
          dt = w.dt[e];
        }
      }
      // rate = -M^-1 R row by row: each inverse-mass entry is loaded once and
      // used at once; the new state goes to this thread's shared-memory column
      // in place of the old one (USM) or to registers
      const bool stage = LIM && w.op == OP_STAGE;
      double u[USM ? 1 : NP][4];
#pragma unroll
      for (int i = 0; i < NP; ++i) {
        double r[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int j = 0; j < NP; ++j) {
          const double mij = AFF ? tab<K, P>(S::O_MINV + i * NP + j) : __ldg(m.minv + (i * NP + j) * E + e);
#pragma unroll
          for (int s = 0; s < 4; ++s) r[s] = fma(mij, acc[j][s], r[s]);
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
          if (!AFF) r[s] = -r[s];
          if (!stage) {
            w.out[(s * NP + i) * E + e] = r[s];
            continue;
          }
          double v;
          if constexpr (USM)
            v = facc[(i * 4 + s) * BT + t];
          else
            v = __ldg(w.V + (s * NP + i) * E + e);
          double un;
          if (w.stage == 1) {
            const double rw = r[s] * ph.norm_w[s];
            nrm = fma(rw, rw, nrm);
            un = v + dt * r[s];
          } else {
            const double u0 = __ldg(w.U0 + (s * NP + i) * E + e);
            un = w.a * u0 + w.b * (v + dt * r[s]);
          }
          if constexpr (USM)
            facc[(i * 4 + s) * BT + t] = un;
          else
            u[i][s] = un;
        }
      }
      if (stage) {
        if (w.elem_norm && w.stage == 1) w.elem_norm[e] = nrm;
        // the limiter works where the new state is: this thread's shared-memory
        // column (USM) or the registers -- no copy, no spilled array
        if constexpr (USM) {
          const SmemCoef<BT> col{facc + t};
          if (ph.limiter == 1 && P > 0) limit_element<K, P, AFF>(col, m, ph, e, sides, scaled, repaired);
#pragma unroll
          for (int i = 0; i < NP; ++i)
#pragma unroll
            for (int s = 0; s < 4; ++s) w.out[(s * NP + i) * E + e] = col(i, s);
        } else {
          if (ph.limiter == 1 && P > 0) limit_element<K, P, AFF>(RegCoef<NP>{u}, m, ph, e, sides, scaled, repaired);
#pragma unroll
          for (int i = 0; i < NP; ++i)
#pragma unroll
            for (int s = 0; s < 4; ++s) w.out[(s * NP + i) * E + e] = u[i][s];
        }
        if (w.flags) w.flags[e] = (uint8_t)(scaled | (repaired << 1));
      }
    }
  }
  // block-level reductions (every thread of the block reaches these)
  if (LIM && w.op == OP_STAGE && w.norm_partial && w.stage == 1)
    block_sum_store<BT / 32>(nrm, w.norm_partial + blk);
  if (LIM && (w.op == OP_STAGE || w.op == OP_LIMIT) && w.counters) {
    const int ns = __syncthreads_count(scaled);
    const int nr = __syncthreads_count(repaired);
    if (t == 0) {
      if (ns) atomicAdd(w.counters + 0, (unsigned long long)ns);
      if (nr) atomicAdd(w.counters + 1, (unsigned long long)nr);
    }
  }
}

}  // namespace nzb
