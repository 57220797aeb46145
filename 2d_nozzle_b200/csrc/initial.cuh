// initial.cuh -- the quasi-1D initial state, L2-projected on the device
// (src/timestepping/initialize.py:41-102).
//
// One thread per element.  At each volume point: the point's coordinates from
// the vertices (vertex shape functions, table GV), density, axial velocity and
// pressure interpolated linearly in x from the instance's quasi-1D solution
// (np.interp: the bracketing interval found by bisection, slope times offset
// plus the left value), the wall half-height y_w(x) and its slope by a
// one-sided-at-the-inlet central difference with h = 1e-6 L, the transverse
// velocity vy = vx clip(y / y_w, 0, 1) slope, and the conserved state; then
// U = M^-1 sum_q phi_q w_q det_q u_q.
//
// The wall is the instance's contour family (src/geometry/contour.py:264-311,
// plus bezier8): a cubic-Hermite converging section with flat ends, and a
// diverging section that is straight (conical), a cubic Hermite with the
// family's end slopes (bell / smooth / moc), a cubic Bezier (bezier), or a
// flat-ended Hermite plus y_th times a degree-9 Bernstein bump (bezier8).  The
// host evaluates the angles' tangents; the polynomial arithmetic here runs in
// the host's order without fused multiply-adds, and integer powers are rounded
// once from a double-double product, so the wall agrees with the host's to the
// last bit or within one.
#pragma once
#include "element.cuh"

namespace nzb {

enum { WALL_FAMILY = 0, WALL_LEN, WALL_XTH, WALL_SPAN, WALL_YTH, WALL_YIN, WALL_YEX, WALL_M0, WALL_M1, WALL_C1, WALL_C2,
       WALL_H, WALL_OFF };
static_assert(WALL_OFF + 8 == NZB_WALL_PARAMS, "wall parameter layout");

__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double clip01(double v) { return v < 0.0 ? 0.0 : (v > 1.0 ? 1.0 : v); }

// t^k, k >= 0, rounded once: the product is carried as a double-double.
__device__ __forceinline__ double ipow(double t, int k) {
  double hi = 1.0, lo = 0.0;
  for (int i = 0; i < k; ++i) {
    const double p = hi * t;
    const double e = fma(hi, t, -p);  // the product's rounding error, exactly
    lo = fma(lo, t, e);
    hi = p;
  }
  return hi + lo;
}

__device__ __forceinline__ double hermite(double s, double y0, double y1, double m0, double m1) {
  const double s2 = mul(s, s), s3 = mul(s2, s);
  const double a = add(sub(mul(2.0, s3), mul(3.0, s2)), 1.0);
  const double b = add(sub(s3, mul(2.0, s2)), s);
  const double c = add(mul(-2.0, s3), mul(3.0, s2));
  const double d = sub(s3, s2);
  return add(add(add(mul(a, y0), mul(b, m0)), mul(c, y1)), mul(d, m1));
}

static __device__ double wall_y(const double* __restrict__ W, double x) {
  const double xi = __ddiv_rn(x, W[WALL_LEN]);
  const double x_th = W[WALL_XTH], y_th = W[WALL_YTH], y_ex = W[WALL_YEX];
  if (xi <= x_th) return hermite(clip01(__ddiv_rn(xi, x_th)), W[WALL_YIN], y_th, 0.0, 0.0);
  const double s = clip01(__ddiv_rn(sub(xi, x_th), W[WALL_SPAN]));
  const int family = (int)W[WALL_FAMILY];
  if (family == 0) return add(y_th, mul(sub(y_ex, y_th), s));
  if (family == 1) return hermite(s, y_th, y_ex, W[WALL_M0], W[WALL_M1]);
  if (family == 2) {
    const double u = sub(1.0, s);
    const double t0 = mul(ipow(u, 3), y_th);
    const double t1 = mul(mul(mul(3.0, ipow(u, 2)), s), W[WALL_C1]);
    const double t2 = mul(mul(mul(3.0, u), ipow(s, 2)), W[WALL_C2]);
    const double t3 = mul(ipow(s, 3), y_ex);
    return add(add(add(t0, t1), t2), t3);
  }
  // bezier8: Bernstein weights of degree 9, control points 1..8
  constexpr double comb9[10] = {1.0, 9.0, 36.0, 84.0, 126.0, 126.0, 84.0, 36.0, 9.0, 1.0};
  const double base = hermite(s, y_th, y_ex, 0.0, W[WALL_M1]);
  const double u = sub(1.0, s);
  double bump = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const double b = mul(mul(comb9[k + 1], ipow(s, k + 1)), ipow(u, 8 - k));
    bump = add(bump, mul(b, W[WALL_OFF + k]));
  }
  return add(base, mul(y_th, bump));
}

// np.interp(x, xs, fs) for sorted xs of n >= 2 points.
__device__ __forceinline__ void interp3(const double* __restrict__ xs, const double* __restrict__ f0,
                                        const double* __restrict__ f1, const double* __restrict__ f2, int64_t n,
                                        double x, double (&out)[3]) {
  const double* f[3] = {f0, f1, f2};
  if (!(x >= xs[0])) {
    for (int c = 0; c < 3; ++c) out[c] = f[c][0];
    return;
  }
  if (x >= xs[n - 1]) {
    for (int c = 0; c < 3; ++c) out[c] = f[c][n - 1];
    return;
  }
  int64_t lo = 0, hi = n - 1;  // xs[lo] <= x < xs[hi]
  while (hi - lo > 1) {
    const int64_t mid = (lo + hi) >> 1;
    if (xs[mid] <= x)
      lo = mid;
    else
      hi = mid;
  }
  for (int c = 0; c < 3; ++c) {
    if (xs[lo] == x) {
      out[c] = f[c][lo];
    } else {
      const double slope = __ddiv_rn(sub(f[c][lo + 1], f[c][lo]), sub(xs[lo + 1], xs[lo]));
      out[c] = add(mul(slope, sub(x, xs[lo])), f[c][lo]);
    }
  }
}

template <int K, int P, bool AFF>
__global__ void __launch_bounds__(128) k_initial_state(const nzb_mesh m, const nzb_physics ph, const nzb_initial_args a) {
  using S = Shape<K, P>;
  constexpr int NP = S::NP, NQV = S::NQV, NF = S::NF;
  const int64_t E = m.n_elem;
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const int inst = m.elem_inst ? __ldg(m.elem_inst + e) : 0;
  const double* W = a.wall + (int64_t)inst * NZB_WALL_PARAMS;
  const int64_t b0 = a.q1d_begin[inst], n = a.q1d_begin[inst + 1] - b0;
  const double* xs = a.q1d + 4 * b0;
  const double g = ph.gamma;
  const double h = W[WALL_H];
  double xv[NF], yv[NF];
#pragma unroll
  for (int v = 0; v < NF; ++v) {
    xv[v] = __ldg(a.verts + v * E + e);
    yv[v] = __ldg(a.verts + (NF + v) * E + e);
  }
  double rhs[NP][4];
#pragma unroll
  for (int i = 0; i < NP; ++i)
#pragma unroll
    for (int s = 0; s < 4; ++s) rhs[i][s] = 0.0;
#pragma unroll 1
  for (int q = 0; q < NQV; ++q) {
    double x = 0.0, y = 0.0;
#pragma unroll
    for (int v = 0; v < NF; ++v) {
      x = add(x, mul(tab<K, P>(S::O_GV + v * NQV + q), xv[v]));
      y = add(y, mul(tab<K, P>(S::O_GV + v * NQV + q), yv[v]));
    }
    double f[3];
    interp3(xs, xs + n, xs + 2 * n, xs + 3 * n, n, x, f);
    const double rho = f[0], vx = f[1], p = f[2];
    const double yw = wall_y(W, x);
    const double xm = sub(x, h);
    const double slope = __ddiv_rn(sub(wall_y(W, add(x, h)), wall_y(W, xm > 0.0 ? xm : 0.0)), add(h, x < h ? x : h));
    const double yr = __ddiv_rn(y, yw > 1e-30 ? yw : 1e-30);
    const double vy = mul(mul(vx, clip01(yr)), slope);
    const double rhoE = add(__ddiv_rn(p, g - 1.0), mul(mul(0.5, rho), add(mul(vx, vx), mul(vy, vy))));
    const double u[4] = {rho, mul(rho, vx), mul(rho, vy), rhoE};
    double wq = tab<K, P>(S::O_WV + q);
    if (!AFF) {
      double x_xi, x_eta, y_xi, y_eta;
      wq *= point_det<K, P>(xv, yv, q, x_xi, x_eta, y_xi, y_eta);
    }
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      const double c = tab<K, P>(S::O_PHI + i * NQV + q) * wq;
#pragma unroll
      for (int s = 0; s < 4; ++s) rhs[i][s] = fma(c, u[s], rhs[i][s]);
    }
  }
  // M^-1: affine M = det M_ref (det cancels against the unscaled weights); general: the element's inverse
#pragma unroll
  for (int i = 0; i < NP; ++i) {
    double r[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int j = 0; j < NP; ++j) {
      const double mij = AFF ? tab<K, P>(S::O_MINV + i * NP + j) : __ldg(m.minv + ((int64_t)i * NP + j) * E + e);
#pragma unroll
      for (int s = 0; s < 4; ++s) r[s] = fma(mij, rhs[j][s], r[s]);
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) a.out[((int64_t)s * NP + i) * E + e] = r[s];
  }
}

}  // namespace nzb
