// generic.cuh -- the DG step for any order and curved (Q = 2) elements, from
// the reference's per-element operators.
//
// The specialised kernels (element.cuh, split.cuh) hold every table of an
// element type in the constant bank and rebuild the metric terms of straight
// elements at each point; they are instantiated for straight elements of
// order 0..3.  For higher orders (up to 21 basis functions and beyond) and for
// curved elements, whose metric terms vary point by point, this path reads
// the operators the reference itself builds (src/spatial/operators.py:209-
// 342): per element the weak-form gradients at the volume points, unfolded
// (grad_x, grad_y) and with the inverse mass folded in (grad_x_m, grad_y_m),
// the folded face basis (face_basis_m), per edge point the normal and
// |dX/dsigma|, and the reference tables in global memory.  Arrays are in the
// reference's layout; the state is (E, NP, 4).  The passes follow the
// reference's compiled path (src/backends/_numba_kernels.py):
//
//   k_gen_edge     one thread per edge: both traces at each edge point, the
//                  Riemann or boundary flux, fw = flux |dX/dsigma| w, the
//                  edge's largest signal speed;
//   k_gen_element  one thread per element: the volume term and the gathered
//                  face terms -- the residual (unfolded operators and the
//                  reference face basis with the face sign) or the rate
//                  -M^-1 R (folded operators) -- and the wave-speed sum;
//   k_gen_limit    one thread per element: the positivity limiter in place
//                  (mean repair, Lebesgue screen, probe minima at the volume
//                  points and the element's own face points, closed-form
//                  density factor, 12-step pressure bisection);
//   k_gen_update   the local step from the wave sums (stage 1), the stage
//                  update a U0 + b (V + dt F) and the weighted norm's per-block
//                  partial sums of stage 1's rate.
// The flux, boundary and primitive formulas are physics.cuh's, shared with
// the specialised kernels.  Each element's scratch (its NP x 4 accumulators)
// is a compile-time-sized array: the kernels are instantiated per NP.
#pragma once
#include <cstdint>

#include "element.cuh"
#include "physics.cuh"
#include "slope.cuh"

namespace nzb {

// The largest number of basis functions an instantiation serves, per bucket.
__host__ __device__ constexpr int gen_np_bucket(int np) {
  return np <= 4 ? 4 : np <= 6 ? 6 : np <= 10 ? 10 : np <= 16 ? 16 : np <= 21 ? 21 : np <= 28 ? 28 : 36;
}
constexpr int GEN_NP_MAX = 36;

__global__ void __launch_bounds__(128) k_gen_edge(const nzb_gen_mesh m, const nzb_physics ph, const double* __restrict__ U,
                                                  double* __restrict__ fw, double* __restrict__ smax) {
  const int64_t n_edge = m.n_int + m.n_bnd;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n_edge) return;
  const int np = m.np, nqf = m.nqf, nf = m.nface;
  const bool interior = k < m.n_int;
  const int64_t le = m.edge_elem[2 * k], re = m.edge_elem[2 * k + 1];
  const int lf = m.edge_face[2 * k], rf = m.edge_face[2 * k + 1];
  const int tag = interior ? 0 : m.edge_tag[k - m.n_int];
  const double* Ul = U + le * np * 4;
  const double* Ur = U + (interior ? re : le) * np * 4;
  double best = 0.0;
  for (int q = 0; q < nqf; ++q) {
    double UL[4] = {0.0, 0.0, 0.0, 0.0}, UR[4] = {0.0, 0.0, 0.0, 0.0}, F[4];
    for (int i = 0; i < np; ++i) {
      const double bl = m.phi_face[(((int64_t)0 * nf + lf) * np + i) * nqf + q];
#pragma unroll
      for (int s = 0; s < 4; ++s) UL[s] = fma(bl, Ul[i * 4 + s], UL[s]);
      if (interior) {
        const double br = m.phi_face[(((int64_t)1 * nf + rf) * np + i) * nqf + q];
#pragma unroll
        for (int s = 0; s < 4; ++s) UR[s] = fma(br, Ur[i * 4 + s], UR[s]);
      }
    }
    const double nx = m.edge_normal[(k * nqf + q) * 2], ny = m.edge_normal[(k * nqf + q) * 2 + 1];
    const double sp = interior ? interface_flux(UL, UR, nx, ny, ph, F) : boundary_flux(tag, UL, nx, ny, ph, ph.p_back, F);
    best = sp > best ? sp : best;
    const double scale = m.edge_jac[k * nqf + q] * m.w_face[q];
#pragma unroll
    for (int s = 0; s < 4; ++s) fw[(k * nqf + q) * 4 + s] = F[s] * scale;
  }
  smax[k] = best;
}

template <int NPB>
__global__ void __launch_bounds__(128) k_gen_element(const nzb_gen_mesh m, const nzb_physics ph, int unfolded,
                                                     const double* __restrict__ U, const double* __restrict__ fw,
                                                     const double* __restrict__ smax, double* __restrict__ out,
                                                     double* __restrict__ wave) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elem) return;
  const int np = m.np, nqv = m.nqv, nqf = m.nqf, nf = m.nface;
  const double g = ph.gamma;
  const double* Ue = U + e * np * 4;
  const double* gx = (unfolded ? m.grad_x : m.grad_x_m) + e * np * nqv;
  const double* gy = (unfolded ? m.grad_y : m.grad_y_m) + e * np * nqv;
  double R[NPB][4];
#pragma unroll
  for (int i = 0; i < NPB; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) R[i][s] = 0.0;
  for (int q = 0; q < nqv; ++q) {
    double u[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NPB; ++i) {
      if (i < np) {
        const double b = m.phi_vol[i * nqv + q];
#pragma unroll
        for (int s = 0; s < 4; ++s) u[s] = fma(b, Ue[i * 4 + s], u[s]);
      }
    }
    const Prim pr = primitives_fast(u, g);
    const double F[4] = {pr.rho * pr.vx, pr.rho * pr.vx * pr.vx + pr.p, pr.rho * pr.vx * pr.vy, pr.rho * pr.vx * pr.H};
    const double G[4] = {pr.rho * pr.vy, pr.rho * pr.vx * pr.vy, pr.rho * pr.vy * pr.vy + pr.p, pr.rho * pr.vy * pr.H};
#pragma unroll
    for (int i = 0; i < NPB; ++i) {
      if (i < np) {
        const double a = gx[i * nqv + q], b = gy[i * nqv + q];
#pragma unroll
        for (int s = 0; s < 4; ++s) R[i][s] -= a * F[s] + b * G[s];
      }
    }
  }
  double acc = 0.0;
  for (int f = 0; f < nf; ++f) {
    const int64_t k = m.face_edge[e * nf + f];
    const double sg = m.face_sign[e * nf + f];
    const int sd = m.face_side[e * nf + f];
    for (int q = 0; q < nqf; ++q) {
      const double* w = fw + (k * nqf + q) * 4;
#pragma unroll
      for (int i = 0; i < NPB; ++i) {
        if (i < np) {
          const double b = sg * (unfolded ? m.phi_face[(((int64_t)sd * nf + f) * np + i) * nqf + q]
                                          : m.face_basis_m[((e * nf + f) * np + i) * nqf + q]);
#pragma unroll
          for (int s = 0; s < 4; ++s) R[i][s] = fma(b, w[s], R[i][s]);
        }
      }
    }
    acc += smax[k] * m.edge_length[k];
  }
  if (wave) wave[e] = acc;
#pragma unroll
  for (int i = 0; i < NPB; ++i) {
    if (i < np) {
#pragma unroll
      for (int s = 0; s < 4; ++s) out[(e * np + i) * 4 + s] = unfolded ? R[i][s] : -R[i][s];
    }
  }
}

// The minimum density and pressure of ubar + theta (u - ubar) over the element's probe points: the
// volume points, then its own trace at each face point (src/backends/_numba_kernels.py:856-924).
template <int NPB>
__device__ void gen_probe_minima(const nzb_gen_mesh& m, const double* Ue, const double (&ub)[4], double theta,
                                 const int* fside, double g, double& rmin, double& pmin) {
  const int np = m.np, nqv = m.nqv, nqf = m.nqf, nf = m.nface;
  double rm = 1e300, pm = 1e300;
  const int npt = nqv + nf * nqf;
  for (int pt = 0; pt < npt; ++pt) {
    double u[4] = {0.0, 0.0, 0.0, 0.0};
    const double* basis;
    int stride;
    if (pt < nqv) {
      basis = m.phi_vol + pt;
      stride = nqv;
    } else {
      const int f = (pt - nqv) / nqf, q = (pt - nqv) - f * nqf;
      basis = m.phi_face + (((int64_t)fside[f] * nf + f) * np) * nqf + q;
      stride = nqf;
    }
#pragma unroll
    for (int i = 0; i < NPB; ++i) {
      if (i < np) {
        const double b = basis[i * stride];
#pragma unroll
        for (int s = 0; s < 4; ++s) u[s] = fma(b, Ue[i * 4 + s], u[s]);
      }
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) u[s] = ub[s] + theta * (u[s] - ub[s]);
    rm = u[0] < rm ? u[0] : rm;
    const double r = u[0] > 1e-300 ? u[0] : 1e-300;
    const double pp = (g - 1.0) * (u[3] - 0.5 * (u[1] * u[1] + u[2] * u[2]) / r);
    pm = pp < pm ? pp : pm;
  }
  rmin = rm;
  pmin = pm;
}

// The positivity limiter of one element in place (src/backends/_numba_kernels.py:927-1093;
// src/spatial/limiter.py:103-243): an element it leaves alone is not rewritten.
template <int NPB>
__device__ __forceinline__ void gen_limit_element(const nzb_gen_mesh& m, const nzb_physics& ph, int64_t e,
                                                  double* __restrict__ Ue, int& scaled, int& repaired) {
  const int np = m.np, nf = m.nface;
  const double g = ph.gamma, g1 = g - 1.0, lam = ph.lebesgue;
  double ub[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int i = 0; i < NPB; ++i) {
    if (i < np) {
      const double w = m.mean_weights[e * np + i];
#pragma unroll
      for (int s = 0; s < 4; ++s) ub[s] = fma(w, Ue[i * 4 + s], ub[s]);
    }
  }
  const double rho_new = ub[0] > ph.rho_floor ? ub[0] : ph.rho_floor;
  const double e_min = ph.p_floor / g1 + 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) / rho_new;
  const double rhoE_new = ub[3] > e_min ? ub[3] : e_min;
  const double d0 = rho_new - ub[0], d3 = rhoE_new - ub[3];
  if (d0 != 0.0 || d3 != 0.0) {
    for (int i = 0; i < np; ++i) {
      Ue[i * 4] += d0;
      Ue[i * 4 + 3] += d3;
    }
    ub[0] = rho_new;
    ub[3] = rhoE_new;
    repaired = 1;
  }
  const double pbar = g1 * (ub[3] - 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) / ub[0]);
  double eps_r = ph.lim_fraction * ub[0], eps_p = ph.lim_fraction * pbar;
  eps_r = eps_r < 0.5 * ph.rho_floor ? 0.5 * ph.rho_floor : eps_r;
  eps_p = eps_p < 0.5 * ph.p_floor ? 0.5 * ph.p_floor : eps_p;
  double dv[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = 0; i < np; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) dv[s] = fmax(dv[s], fabs(Ue[i * 4 + s] - ub[s]));
  const double rho_lo = ub[0] - lam * dv[0];
  if (rho_lo >= eps_r) {
    const double m_hi = sqrt(ub[1] * ub[1] + ub[2] * ub[2]) + lam * sqrt(dv[1] * dv[1] + dv[2] * dv[2]);
    if (g1 * (ub[3] - lam * dv[3] - 0.5 * m_hi * m_hi / rho_lo) >= eps_p) return;
  }
  int fside[8];
  for (int f = 0; f < nf; ++f) fside[f] = m.face_side[e * nf + f];
  double rmin, pmin;
  gen_probe_minima<NPB>(m, Ue, ub, 1.0, fside, g, rmin, pmin);
  if (!(rmin < eps_r) && !(pmin < eps_p)) return;
  double theta = 1.0;
  if (rmin < eps_r) {
    const double gap = ub[0] - rmin;
    theta = gap <= 0.0 ? 0.0 : (ub[0] - eps_r) / gap;
    theta = theta < 0.0 ? 0.0 : (theta > 1.0 ? 1.0 : theta);
  }
  double rr, ph_;
  gen_probe_minima<NPB>(m, Ue, ub, theta, fside, g, rr, ph_);
  if (ph_ < eps_p) {
    double lo = 0.0, hi = theta;
    for (int it = 0; it < ph.lim_steps; ++it) {
      const double mid = 0.5 * (lo + hi);
      double pm;
      gen_probe_minima<NPB>(m, Ue, ub, mid, fside, g, rr, pm);
      if (pm >= eps_p)
        lo = mid;
      else
        hi = mid;
    }
    theta = lo;
  }
  for (int i = 0; i < np; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) Ue[i * 4 + s] = ub[s] + theta * (Ue[i * 4 + s] - ub[s]);
  scaled = 1;
}

__device__ __forceinline__ void gen_count(unsigned long long* counters, int scaled, int repaired) {
  if (counters) {
    const int ns = __syncthreads_count(scaled), nr = __syncthreads_count(repaired);
    if (threadIdx.x == 0) {
      if (ns) atomicAdd(counters + 0, (unsigned long long)ns);
      if (nr) atomicAdd(counters + 1, (unsigned long long)nr);
    }
  }
}

// The positivity limiter in place, one thread per element.
template <int NPB>
__global__ void __launch_bounds__(128) k_gen_limit(const nzb_gen_mesh m, const nzb_physics ph, double* __restrict__ U,
                                                   unsigned long long* counters) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int scaled = 0, repaired = 0;
  if (e < m.n_elem) gen_limit_element<NPB>(m, ph, e, U + e * m.np * 4, scaled, repaired);
  gen_count(counters, scaled, repaired);
}

// The Superbee TVB slope limiter (src/spatial/limiter.py:246-429) on the generic path, in the
// specialised kernels' three passes (slope.cuh): the cell averages ubar (E, 4); their maxima
// max_e |ubar_s| (one block; exact in any order); then per element the factor theta = the
// minimum over interior faces and components of clip(superbee(a, d) / d, 0, 1), with d the
// face-averaged own trace minus ubar and a the jump of cell averages across the face, a face
// quiet where |d| <= 1e-12 or |d| <= tvb (A_e / A_domain) max|ubar_s|; U <- ubar + theta (U -
// ubar); then the positivity limiter, as apply_limiter runs them.  An element counts as scaled
// when either limiter changed it.
__global__ void __launch_bounds__(128) k_gen_cell_means(const nzb_gen_mesh m, const double* __restrict__ U,
                                                        double* __restrict__ means) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= m.n_elem) return;
  const int np = m.np;
  double ub[4] = {0.0, 0.0, 0.0, 0.0};
  for (int i = 0; i < np; ++i) {
    const double w = m.mean_weights[e * np + i];
#pragma unroll
    for (int s = 0; s < 4; ++s) ub[s] = fma(w, U[(e * np + i) * 4 + s], ub[s]);
  }
#pragma unroll
  for (int s = 0; s < 4; ++s) means[e * 4 + s] = ub[s];
}

__global__ void __launch_bounds__(1024) k_gen_lim_scale(const double* __restrict__ means, int64_t E,
                                                        double* __restrict__ scale) {
  __shared__ double red[4][32];
  double mx[4] = {0.0, 0.0, 0.0, 0.0};
  for (int64_t e = threadIdx.x; e < E; e += blockDim.x)
#pragma unroll
    for (int s = 0; s < 4; ++s) mx[s] = fmax(mx[s], fabs(means[e * 4 + s]));
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    double v = mx[s];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    if ((threadIdx.x & 31) == 0) red[s][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double v = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) v = fmax(v, red[threadIdx.x][k]);
    scale[threadIdx.x] = v;
  }
}

template <int NPB>
__global__ void __launch_bounds__(128) k_gen_superbee(const nzb_gen_mesh m, const nzb_physics ph,
                                                      double* __restrict__ U, const double* __restrict__ means,
                                                      const double* __restrict__ scale,
                                                      const double* __restrict__ share,
                                                      unsigned long long* counters) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int scaled = 0, repaired = 0;
  if (e < m.n_elem) {
    const int np = m.np, nf = m.nface, nqf = m.nqf;
    double* Ue = U + e * np * 4;
    double ub[4], sc[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      ub[s] = means[e * 4 + s];
      sc[s] = scale[s];
    }
    const double sh = share[e];
    double wsum = 0.0;
    for (int q = 0; q < nqf; ++q) wsum += m.w_face[q];
    double theta = 1.0;
    for (int f = 0; f < nf; ++f) {
      const int64_t k = m.face_edge[e * nf + f];
      if (k >= m.n_int) continue;  // a boundary face is not limited against
      const int64_t a0 = m.edge_elem[2 * k], a1 = m.edge_elem[2 * k + 1];
      const int64_t nb = a0 == e ? a1 : a0;
      const int side = m.face_side[e * nf + f];
      const double* pf = m.phi_face + (int64_t)(side * nf + f) * np * nqf;
      double tm[4] = {0.0, 0.0, 0.0, 0.0};
      for (int q = 0; q < nqf; ++q) {
        double tr[4] = {0.0, 0.0, 0.0, 0.0};
        for (int i = 0; i < np; ++i) {
          const double c = pf[i * nqf + q];
#pragma unroll
          for (int s = 0; s < 4; ++s) tr[s] = fma(c, Ue[i * 4 + s], tr[s]);
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) tm[s] = fma(m.w_face[q], tr[s], tm[s]);
      }
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double d = tm[s] / wsum - ub[s];
        const double a = means[nb * 4 + s] - ub[s];
        const bool quiet = fabs(d) <= 1e-12 || fabs(d) <= ph.tvb_constant * sh * sc[s];
        if (!quiet) {
          double tf = superbee2(a, d) / d;
          tf = tf < 0.0 ? 0.0 : (tf > 1.0 ? 1.0 : tf);
          theta = tf < theta ? tf : theta;
        }
      }
    }
    bool changed = false;
    for (int i = 0; i < np; ++i)
#pragma unroll
      for (int s = 0; s < 4; ++s) {
        const double v = ub[s] + theta * (Ue[i * 4 + s] - ub[s]);
        changed |= v != Ue[i * 4 + s];
        Ue[i * 4 + s] = v;
      }
    gen_limit_element<NPB>(m, ph, e, Ue, scaled, repaired);
    scaled |= changed ? 1 : 0;
  }
  gen_count(counters, scaled, repaired);
}

// One stage's update per element: stage 1 forms the local step dt = c 2 A / max(wave, FLOOR) and the
// weighted squares of its rate (per-block partial sums); out = a U0 + b (V + dt F) (a = 0: V + dt F).
__global__ void __launch_bounds__(128) k_gen_update(const nzb_gen_mesh m, const nzb_physics ph, int stage,
                                                    double dt_factor, double a, double b, const double* __restrict__ V,
                                                    const double* __restrict__ U0, const double* __restrict__ F,
                                                    const double* __restrict__ wave, double* __restrict__ dt,
                                                    double* __restrict__ out, double* __restrict__ partial) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double sq = 0.0;
  if (e < m.n_elem) {
    const int n = m.np * 4;
    double d;
    if (stage == 1) {
      const double w = wave[e] < FLOOR ? FLOOR : wave[e];
      d = dt_factor * 2.0 * m.elem_area[e] / w;
      dt[e] = d;
    } else {
      d = dt[e];
    }
    for (int k = 0; k < n; ++k) {
      const int64_t o = e * n + k;
      const double f = F[o];
      if (stage == 1) {
        const double r = f * ph.norm_w[k & 3];
        sq = fma(r, r, sq);
      }
      out[o] = a == 0.0 ? V[o] + d * f : a * U0[o] + b * (V[o] + d * f);
    }
  }
  if (stage == 1 && partial) block_sum_store<4>(sq, partial + blockIdx.x);
}

}  // namespace nzb
