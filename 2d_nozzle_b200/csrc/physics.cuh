// physics.cuh -- pointwise Euler physics: primitives, Riemann solvers, boundary fluxes.
//
// Scalar device restatements of the reference's NumPy formulas, keeping their
// operation order so results agree to round-off:
//   primitives / normal flux   src/physics/thermo.py:46-80
//   Roe + Harten-Hyman         src/physics/fluxes.py:38-103
//   HLLC (Batten, low-Mach)    src/physics/fluxes.py:106-255
//   AUSM+-up                   src/physics/fluxes.py:262-445
//   wall / inflow / outflow    src/physics/boundary.py:20-214
// max(x, FLOOR) is written so that a NaN propagates, as numpy.maximum does:
// a diverging march must surface as a non-finite residual, not be masked.
//
// Every function is a template over the scalar type T: double for the forward
// kernels, Dual<N> (dual.cuh) where the adjoint needs flux Jacobians.
#pragma once
#include "dual.cuh"
#include "nozzle_b200.h"

namespace nzb {

constexpr double FLOOR = 1e-10;

template <class T>
__device__ __forceinline__ T floor_at(const T& x, double f) {
  return x < f ? T(f) : x;
}

template <class T>
struct PrimT {
  T rho, vx, vy, p, H, inv;  // inv = 1 / rho
};
using Prim = PrimT<double>;

// Primitives with one reciprocal of the (floored) density: vx = U1 (1/rho)
// differs from the reference's U1 / rho in the last bit at most, and saves
// two divisions -- each an iterative sequence on the FP64 pipe -- per state,
// which is most of a face flux's cost.
template <class T>
__device__ __forceinline__ PrimT<T> primitives(const T* U, double g) {
  PrimT<T> s;
  s.rho = floor_at(U[0], FLOOR);
  s.inv = 1.0 / s.rho;
  s.vx = U[1] * s.inv;
  s.vy = U[2] * s.inv;
  s.p = floor_at((g - 1.0) * (U[3] - 0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy)), FLOOR);
  s.H = (U[3] + s.p) * s.inv;
  return s;
}

// The volume-point primitives (feeding only the weak-form projection).
__device__ __forceinline__ Prim primitives_fast(const double* U, double g) { return primitives(U, g); }

// Every function below takes each operand group with its own scalar type --
// the two traces (TL, TR), the normal (TN), the back pressure (TP) -- so that
// a group the caller does not differentiate stays a plain double and costs
// plain arithmetic; intermediate quantities take the mixed type (Mix).  With
// every type double the expressions are exactly the forward kernels' ones.
template <class T, class TN, class TF>
__device__ __forceinline__ void normal_flux(const PrimT<T>& s, const TN& nx, const TN& ny, TF* F) {
  const auto vn = s.vx * nx + s.vy * ny;
  F[0] = s.rho * vn;
  F[1] = s.rho * s.vx * vn + s.p * nx;
  F[2] = s.rho * s.vy * vn + s.p * ny;
  F[3] = s.rho * s.H * vn;
}

// The Euler flux pair (F, G) of src/physics/thermo.py:64-70.
template <class T>
__device__ __forceinline__ void euler_flux(const T* U, double g, T* F, T* G) {
  const PrimT<T> s = primitives(U, g);
  F[0] = s.rho * s.vx;
  F[1] = s.rho * s.vx * s.vx + s.p;
  F[2] = s.rho * s.vx * s.vy;
  F[3] = s.rho * s.vx * s.H;
  G[0] = s.rho * s.vy;
  G[1] = s.rho * s.vx * s.vy;
  G[2] = s.rho * s.vy * s.vy + s.p;
  G[3] = s.rho * s.vy * s.H;
}

template <class TL, class TR, class TN, class TF>
__device__ __forceinline__ TF roe_flux(const TL* UL, const TR* UR, const TN& nx, const TN& ny, double g,
                                       double efix, TF* F) {
  const PrimT<TL> L = primitives(UL, g);
  const PrimT<TR> R = primitives(UR, g);
  Mix<TL, TN> FL[4];
  Mix<TR, TN> FR[4];
  normal_flux(L, nx, ny, FL);
  normal_flux(R, nx, ny, FR);
  const TL sL = sqrt(L.rho);
  const TR sR = sqrt(R.rho);
  const auto iden = 1.0 / (sL + sR);
  const auto vx = (sL * L.vx + sR * R.vx) * iden;
  const auto vy = (sL * L.vy + sR * R.vy) * iden;
  const auto H = (sL * L.H + sR * R.H) * iden;
  const auto q2 = vx * vx + vy * vy;
  const auto c = sqrt(floor_at((g - 1.0) * (H - 0.5 * q2), FLOOR));
  const auto vn = vx * nx + vy * ny;
  auto l1 = fabs(vn + c), l2 = fabs(vn - c), l3 = fabs(vn);
  const TF smax = l1 < l2 ? l2 : l1;
  const auto eps = efix * c;
  if (l1 < eps) l1 = (l1 * l1 + eps * eps) / (2.0 * eps);
  if (l2 < eps) l2 = (l2 * l2 + eps * eps) / (2.0 * eps);
  if (l3 < eps) l3 = (l3 * l3 + eps * eps) / (2.0 * eps);
  const auto d0 = UR[0] - UL[0], d1 = UR[1] - UL[1], d2 = UR[2] - UL[2], d3 = UR[3] - UL[3];
  const auto G1 = (g - 1.0) * (0.5 * q2 * d0 - vx * d1 - vy * d2 + d3);
  const auto G2 = -vn * d0 + d1 * nx + d2 * ny;
  const auto s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
  const auto ic = 1.0 / c;
  const auto C1 = (G1 * (ic * ic)) * (s1 - l3) + (G2 * ic) * s2;
  const auto C2 = (G1 * ic) * s2 + (s1 - l3) * G2;
  F[0] = 0.5 * (FL[0] + FR[0]) - 0.5 * (l3 * d0 + C1);
  F[1] = 0.5 * (FL[1] + FR[1]) - 0.5 * (l3 * d1 + C1 * vx + C2 * nx);
  F[2] = 0.5 * (FL[2] + FR[2]) - 0.5 * (l3 * d2 + C1 * vy + C2 * ny);
  F[3] = 0.5 * (FL[3] + FR[3]) - 0.5 * (l3 * d3 + C1 * H + C2 * vn);
  return smax;
}

template <class T>
__device__ __forceinline__ T guard(const T& x) {
  return fabs(x) > FLOOR ? x : T(FLOOR);
}

template <class TL, class TR, class TN, class TF>
__device__ __forceinline__ TF hllc_flux(const TL* UL, const TR* UR, const TN& nx, const TN& ny, double g,
                                        double low_mach, TF* F) {
  using TM = Mix<TL, TR>;
  const PrimT<TL> L = primitives(UL, g);
  const PrimT<TR> R = primitives(UR, g);
  const auto vnL = L.vx * nx + L.vy * ny;
  const auto vnR = R.vx * nx + R.vy * ny;
  const TL aL = sqrt(floor_at(g * L.p * L.inv, FLOOR));
  const TR aR = sqrt(floor_at(g * R.p * R.inv, FLOOR));
  const TL sL = sqrt(L.rho);
  const TR sR = sqrt(R.rho);
  const auto iden = 1.0 / (sL + sR);
  const auto vx = (sL * L.vx + sR * R.vx) * iden;
  const auto vy = (sL * L.vy + sR * R.vy) * iden;
  const auto H = (sL * L.H + sR * R.H) * iden;
  const auto vt = vx * nx + vy * ny;
  const auto at = sqrt(floor_at((g - 1.0) * (H - 0.5 * (vx * vx + vy * vy)), FLOOR));
  TF SL = fmin(vnL - aL, vt - at);
  TF SR = fmax(vnR + aR, vt + at);
  if (low_mach > 0.0) {
    const TF mach = fmax(fabs(vnL) / aL, fabs(vnR) / aR);
    const TF phi = fmin(TF(1.0), mach / low_mach);
    const TF bL = fmin(vnL, vt), bR = fmax(vnR, vt);
    SL = bL - phi * (bL - SL);
    SR = bR + phi * (SR - bR);
  }
  const TF smax = fmax(fabs(SL), fabs(SR));
  Mix<TL, TN> FL[4];
  normal_flux(L, nx, ny, FL);
  if (SL >= 0.0) {
    F[0] = FL[0]; F[1] = FL[1]; F[2] = FL[2]; F[3] = FL[3];
    return smax;
  }
  Mix<TR, TN> FR[4];
  normal_flux(R, nx, ny, FR);
  if (SR <= 0.0) {
    F[0] = FR[0]; F[1] = FR[1]; F[2] = FR[2]; F[3] = FR[3];
    return smax;
  }
  const auto mL = L.rho * (SL - vnL), mR = R.rho * (SR - vnR);
  const TF dm = fabs(mR - mL) > FLOOR ? mR - mL : TF(FLOOR);
  const TF SM = (R.rho * vnR * (SR - vnR) - L.rho * vnL * (SL - vnL) + L.p - R.p) / dm;
  // one side's star state: contact normal speed, own tangential velocity
  const bool left = SM >= 0.0;
  const PrimT<TM> K = left ? PrimT<TM>{L.rho, L.vx, L.vy, L.p, L.H, L.inv} : PrimT<TM>{R.rho, R.vx, R.vy, R.p, R.H, R.inv};
  TM UK[4];
  TF FK[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    UK[c] = left ? TM(UL[c]) : TM(UR[c]);
    FK[c] = left ? TF(FL[c]) : TF(FR[c]);
  }
  const TF S = left ? SL : SR;
  const TF vn = left ? TF(vnL) : TF(vnR);
  const TF fac = (S - vn) / guard(S - SM);
  const TF rs = K.rho * fac;
  const TF vxs = K.vx + (SM - vn) * nx;
  const TF vys = K.vy + (SM - vn) * ny;
  const TF Es = UK[3] * K.inv + (SM - vn) * (SM + K.p / guard(K.rho * (S - vn)));
  F[0] = FK[0] + S * (rs - UK[0]);
  F[1] = FK[1] + S * (rs * vxs - UK[1]);
  F[2] = FK[2] + S * (rs * vys - UK[2]);
  F[3] = FK[3] + S * (rs * Es - UK[3]);
  return smax;
}

template <class TL, class TR, class TN, class TF>
__device__ __forceinline__ TF ausm_up_flux(const TL* UL, const TR* UR, const TN& nx, const TN& ny, double g,
                                           TF* F) {
  constexpr double BETA = 0.125, ALPHA = 0.1875, KP = 0.4, KU = 0.2;
  const PrimT<TL> L = primitives(UL, g);
  const PrimT<TR> R = primitives(UR, g);
  const auto vnL = L.vx * nx + L.vy * ny;
  const auto vnR = R.vx * nx + R.vy * ny;
  const TL aL = sqrt(g * L.p * L.inv);
  const TR aR = sqrt(g * R.p * R.inv);
  const auto ah = 0.5 * (aL + aR), rh = 0.5 * (L.rho + R.rho);
  const auto iah = 1.0 / ah;
  const auto mL = vnL * iah, mR = vnR * iah;
  const auto mb2 = 0.5 * (mL * mL + mR * mR);
  const auto pL2 = 0.25 * ((mL + 1.0) * (mL + 1.0)), mL2 = -0.25 * ((mL - 1.0) * (mL - 1.0));
  const auto pR2 = 0.25 * ((mR + 1.0) * (mR + 1.0)), mR2 = -0.25 * ((mR - 1.0) * (mR - 1.0));
  const auto m4p = fabs(mL) >= 1.0 ? 0.5 * (mL + fabs(mL)) : pL2 * (1.0 - 16.0 * BETA * mL2);
  const auto m4m = fabs(mR) >= 1.0 ? 0.5 * (mR - fabs(mR)) : mR2 * (1.0 + 16.0 * BETA * pR2);
  const auto dif = 1.0 - mb2;
  const TF uh = ah * (m4p + m4m) + KP * (dif < 0.0 ? like(dif, 0.0) : dif) * (L.p - R.p) * iah / rh;
  const auto p5p = fabs(mL) >= 1.0 ? like(mL, mL > 0.0 ? 1.0 : 0.0) : pL2 * ((2.0 - mL) - 16.0 * ALPHA * mL * mL2);
  const auto p5m = fabs(mR) >= 1.0 ? like(mR, mR > 0.0 ? 0.0 : 1.0) : mR2 * ((-2.0 - mR) + 16.0 * ALPHA * mR * pR2);
  const TF ph = p5p * L.p + p5m * R.p + KU * p5p * p5m * rh * ah * (vnL - vnR);
  const TL PL[4] = {L.rho, L.rho * L.vx, L.rho * L.vy, UL[3] + L.p};
  const TR PR[4] = {R.rho, R.rho * R.vx, R.rho * R.vy, UR[3] + R.p};
  const TF au = fabs(uh);
#pragma unroll
  for (int s = 0; s < 4; ++s) F[s] = 0.5 * uh * (PL[s] + PR[s]) - 0.5 * au * (PR[s] - PL[s]);
  F[1] = F[1] + ph * nx;
  F[2] = F[2] + ph * ny;
  F[0] = F[0] + ph * 0.0;
  F[3] = F[3] + ph * 0.0;
  return fmax(fabs(vnL) + aL, fabs(vnR) + aR);
}

template <class T, class TN, class TF>
__device__ __forceinline__ TF wall_flux(const T* U, const TN& nx, const TN& ny, double g, TF* F) {
  const T rho = floor_at(U[0], FLOOR);
  const T vx = U[1] / rho, vy = U[2] / rho;
  const auto vn = vx * nx + vy * ny;
  const auto tx = vx - vn * nx, ty = vy - vn * ny;
  const auto pb = floor_at((g - 1.0) * (U[3] - 0.5 * rho * (tx * tx + ty * ty)), FLOOR);
  F[0] = TF(0.0);
  F[1] = pb * nx;
  F[2] = pb * ny;
  F[3] = TF(0.0);
  return sqrt(g * pb / rho);
}

template <class T, class TN, class TF>
__device__ __forceinline__ TF inflow_flux(const T* U, const TN& nx, const TN& ny, const nzb_physics& ph, TF* F) {
  const double g = ph.gamma;
  const PrimT<T> s = primitives(U, g);
  const T a = sqrt(g * s.p / s.rho);
  const auto vn = s.vx * nx + s.vy * ny;
  const auto Jp = vn + 2.0 * a / (g - 1.0);
  const auto r = Jp / ph.in_at;
  const auto beta = r * r;
  const TN nd = nx * ph.in_cos + ny * ph.in_sin;
  auto qa = 0.5 * (g - 1.0) * beta - nd * nd;
  const TN qb = -4.0 * nd / (g - 1.0);
  const double k = 2.0 / (g - 1.0);
  const auto qc = beta - k * k;
  if (fabs(qa) < 1e-12) qa = like(qa, qa >= 0.0 ? 1e-12 : -1e-12);
  auto disc = qb * qb - 4.0 * qa * qc;
  disc = disc < 0.0 ? like(disc, 0.0) : disc;
  const auto sq = sqrt(disc);
  const auto r1 = (-qb + sq) / (2.0 * qa), r2 = (-qb - sq) / (2.0 * qa);
  const auto c1 = r1 >= 0.0 ? r1 : like(r1, 1e30), c2 = r2 >= 0.0 ? r2 : like(r2, 1e30);
  auto M = fmin(c1, c2);
  M = M > 0.5e30 ? like(M, 0.0) : M;
  M = M < 0.0 ? like(M, 0.0) : (M > 1.0 ? like(M, 1.0) : M);
  const auto fac = 1.0 + 0.5 * (g - 1.0) * M * M;
  const auto ab = sqrt(ph.in_at2 / fac);
  const auto qbv = M * ab;
  const auto vxb = qbv * ph.in_cos, vyb = qbv * ph.in_sin;
  const auto rhob = ph.in_rho_t * pow(fac, -1.0 / (g - 1.0));
  const auto pb = rhob * ab * ab / g;
  const double Hb = ph.in_at2 / (g - 1.0);
  const TF vnb = vxb * nx + vyb * ny;
  F[0] = rhob * vnb;
  F[1] = rhob * vxb * vnb + pb * nx;
  F[2] = rhob * vyb * vnb + pb * ny;
  F[3] = rhob * Hb * vnb;
  return fabs(vnb) + ab;
}

template <class T, class TN, class TP, class TF>
__device__ __forceinline__ TF outflow_flux(const T* U, const TN& nx, const TN& ny, const nzb_physics& ph,
                                           const TP& p_back, TF* F) {
  const double g = ph.gamma;
  const PrimT<T> s = primitives(U, g);
  const T a = sqrt(g * s.p / s.rho);
  const auto vn = s.vx * nx + s.vy * ny;
  TF Ub[4];
  if (vn / a >= 1.0) {
    Ub[0] = U[0]; Ub[1] = U[1]; Ub[2] = U[2]; Ub[3] = U[3];
  } else {
    const TP pb = p_back;
    const auto rhob = s.rho * pow(pb / s.p, 1.0 / g);
    const auto ab = sqrt(g * pb / rhob);
    const auto vnb = vn + 2.0 / (g - 1.0) * (a - ab);
    const auto vxb = (s.vx - vn * nx) + vnb * nx;
    const auto vyb = (s.vy - vn * ny) + vnb * ny;
    const auto Eb = pb / ((g - 1.0) * rhob) + 0.5 * (vxb * vxb + vyb * vyb);
    Ub[0] = rhob; Ub[1] = rhob * vxb; Ub[2] = rhob * vyb; Ub[3] = rhob * Eb;
    if (ph.bf_rho_t > 0.0) {
      const TP rf = ph.bf_rho_t * pow(pb / ph.bf_p_t, 1.0 / g);
      const TP af = sqrt(g * pb / rf);
      const auto vnf = vn + 2.0 / (g - 1.0) * (a - af);
      const auto vxf = vnf * nx, vyf = vnf * ny;
      const auto Ef = pb / ((g - 1.0) * rf) + 0.5 * (vxf * vxf + vyf * vyf);
      const TF Uf[4] = {rf, rf * vxf, rf * vyf, rf * Ef};
      auto t = (vn / a) / ::fmax(ph.bf_band, 1e-12);
      t = t < 0.0 ? like(t, 0.0) : (t > 1.0 ? like(t, 1.0) : t);
#pragma unroll
      for (int c = 0; c < 4; ++c) Ub[c] = t * Ub[c] + (1.0 - t) * Uf[c];
    }
  }
  const PrimT<TF> o = primitives(Ub, g);
  normal_flux(o, nx, ny, F);
  return fabs(o.vx * nx + o.vy * ny) + sqrt(g * o.p / o.rho);
}

template <class TL, class TR, class TN, class TF>
__device__ __forceinline__ TF interface_flux(const TL* UL, const TR* UR, const TN& nx, const TN& ny,
                                             const nzb_physics& ph, TF* F) {
  if (ph.flux == NZB_HLLC) return hllc_flux(UL, UR, nx, ny, ph.gamma, ph.hllc_low_mach, F);
  if (ph.flux == NZB_AUSMUP) return ausm_up_flux(UL, UR, nx, ny, ph.gamma, F);
  return roe_flux(UL, UR, nx, ny, ph.gamma, ph.entropy_fix, F);
}

template <class T, class TN, class TP, class TF>
__device__ __forceinline__ TF boundary_flux(int tag, const T* U, const TN& nx, const TN& ny, const nzb_physics& ph,
                                            const TP& p_back, TF* F) {
  if (tag == NZB_INFLOW) return inflow_flux(U, nx, ny, ph, F);
  if (tag == NZB_OUTFLOW) return outflow_flux(U, nx, ny, ph, p_back, F);
  return wall_flux(U, nx, ny, ph.gamma, F);
}

}  // namespace nzb
