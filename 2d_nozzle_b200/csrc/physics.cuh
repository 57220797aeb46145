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
#pragma once
#include "nozzle_b200.h"

namespace nzb {

constexpr double FLOOR = 1e-10;

struct Q4 {
  double v[4];
};

__device__ __forceinline__ double floor_at(double x, double f) { return x < f ? f : x; }

struct Prim {
  double rho, vx, vy, p, H;
};

__device__ __forceinline__ Prim primitives(const double* U, double g) {
  Prim s;
  s.rho = floor_at(U[0], FLOOR);
  s.vx = U[1] / s.rho;
  s.vy = U[2] / s.rho;
  s.p = floor_at((g - 1.0) * (U[3] - 0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy)), FLOOR);
  s.H = (U[3] + s.p) / s.rho;
  return s;
}

// The same primitives with one division: vx = U1 (1/rho) differs from U1 / rho
// in the last bit at most.  Used for the volume-point fluxes, which feed only
// the weak-form projection, never a branch.
__device__ __forceinline__ Prim primitives_fast(const double* U, double g) {
  Prim s;
  s.rho = floor_at(U[0], FLOOR);
  const double inv = 1.0 / s.rho;
  s.vx = U[1] * inv;
  s.vy = U[2] * inv;
  s.p = floor_at((g - 1.0) * (U[3] - 0.5 * s.rho * (s.vx * s.vx + s.vy * s.vy)), FLOOR);
  s.H = (U[3] + s.p) * inv;
  return s;
}

__device__ __forceinline__ void normal_flux(const Prim& s, double nx, double ny, double* F) {
  const double vn = s.vx * nx + s.vy * ny;
  F[0] = s.rho * vn;
  F[1] = s.rho * s.vx * vn + s.p * nx;
  F[2] = s.rho * s.vy * vn + s.p * ny;
  F[3] = s.rho * s.H * vn;
}

__device__ __forceinline__ double roe_flux(const double* UL, const double* UR, double nx, double ny, double g,
                                           double efix, double* F) {
  const Prim L = primitives(UL, g), R = primitives(UR, g);
  double FL[4], FR[4];
  normal_flux(L, nx, ny, FL);
  normal_flux(R, nx, ny, FR);
  const double sL = sqrt(L.rho), sR = sqrt(R.rho);
  const double den = sL + sR;
  const double vx = (sL * L.vx + sR * R.vx) / den;
  const double vy = (sL * L.vy + sR * R.vy) / den;
  const double H = (sL * L.H + sR * R.H) / den;
  const double q2 = vx * vx + vy * vy;
  const double c = sqrt(floor_at((g - 1.0) * (H - 0.5 * q2), FLOOR));
  const double vn = vx * nx + vy * ny;
  double l1 = fabs(vn + c), l2 = fabs(vn - c), l3 = fabs(vn);
  const double smax = l1 < l2 ? l2 : l1;
  const double eps = efix * c;
  if (l1 < eps) l1 = (l1 * l1 + eps * eps) / (2.0 * eps);
  if (l2 < eps) l2 = (l2 * l2 + eps * eps) / (2.0 * eps);
  if (l3 < eps) l3 = (l3 * l3 + eps * eps) / (2.0 * eps);
  const double d0 = UR[0] - UL[0], d1 = UR[1] - UL[1], d2 = UR[2] - UL[2], d3 = UR[3] - UL[3];
  const double G1 = (g - 1.0) * (0.5 * q2 * d0 - vx * d1 - vy * d2 + d3);
  const double G2 = -vn * d0 + d1 * nx + d2 * ny;
  const double s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
  const double C1 = (G1 / (c * c)) * (s1 - l3) + (G2 / c) * s2;
  const double C2 = (G1 / c) * s2 + (s1 - l3) * G2;
  F[0] = 0.5 * (FL[0] + FR[0]) - 0.5 * (l3 * d0 + C1);
  F[1] = 0.5 * (FL[1] + FR[1]) - 0.5 * (l3 * d1 + C1 * vx + C2 * nx);
  F[2] = 0.5 * (FL[2] + FR[2]) - 0.5 * (l3 * d2 + C1 * vy + C2 * ny);
  F[3] = 0.5 * (FL[3] + FR[3]) - 0.5 * (l3 * d3 + C1 * H + C2 * vn);
  return smax;
}

__device__ __forceinline__ double guard(double x) { return fabs(x) > FLOOR ? x : FLOOR; }

__device__ __forceinline__ double hllc_flux(const double* UL, const double* UR, double nx, double ny, double g,
                                            double low_mach, double* F) {
  const Prim L = primitives(UL, g), R = primitives(UR, g);
  const double vnL = L.vx * nx + L.vy * ny, vnR = R.vx * nx + R.vy * ny;
  const double aL = sqrt(floor_at(g * L.p / L.rho, FLOOR));
  const double aR = sqrt(floor_at(g * R.p / R.rho, FLOOR));
  const double sL = sqrt(L.rho), sR = sqrt(R.rho);
  const double den = sL + sR;
  const double vx = (sL * L.vx + sR * R.vx) / den;
  const double vy = (sL * L.vy + sR * R.vy) / den;
  const double H = (sL * L.H + sR * R.H) / den;
  const double vt = vx * nx + vy * ny;
  const double at = sqrt(floor_at((g - 1.0) * (H - 0.5 * (vx * vx + vy * vy)), FLOOR));
  double SL = fmin(vnL - aL, vt - at);
  double SR = fmax(vnR + aR, vt + at);
  if (low_mach > 0.0) {
    const double mach = fmax(fabs(vnL) / aL, fabs(vnR) / aR);
    const double phi = fmin(1.0, mach / low_mach);
    const double bL = fmin(vnL, vt), bR = fmax(vnR, vt);
    SL = bL - phi * (bL - SL);
    SR = bR + phi * (SR - bR);
  }
  const double smax = fmax(fabs(SL), fabs(SR));
  double FL[4];
  normal_flux(L, nx, ny, FL);
  if (SL >= 0.0) {
    F[0] = FL[0]; F[1] = FL[1]; F[2] = FL[2]; F[3] = FL[3];
    return smax;
  }
  double FR[4];
  normal_flux(R, nx, ny, FR);
  if (SR <= 0.0) {
    F[0] = FR[0]; F[1] = FR[1]; F[2] = FR[2]; F[3] = FR[3];
    return smax;
  }
  const double mL = L.rho * (SL - vnL), mR = R.rho * (SR - vnR);
  const double dm = fabs(mR - mL) > FLOOR ? mR - mL : FLOOR;
  const double SM = (R.rho * vnR * (SR - vnR) - L.rho * vnL * (SL - vnL) + L.p - R.p) / dm;
  // one side's star state: contact normal speed, own tangential velocity
  const bool left = SM >= 0.0;
  const Prim& K = left ? L : R;
  const double* UK = left ? UL : UR;
  const double* FK = left ? FL : FR;
  const double S = left ? SL : SR;
  const double vn = left ? vnL : vnR;
  const double fac = (S - vn) / guard(S - SM);
  const double rs = K.rho * fac;
  const double vxs = K.vx + (SM - vn) * nx;
  const double vys = K.vy + (SM - vn) * ny;
  const double Es = UK[3] / K.rho + (SM - vn) * (SM + K.p / guard(K.rho * (S - vn)));
  F[0] = FK[0] + S * (rs - UK[0]);
  F[1] = FK[1] + S * (rs * vxs - UK[1]);
  F[2] = FK[2] + S * (rs * vys - UK[2]);
  F[3] = FK[3] + S * (rs * Es - UK[3]);
  return smax;
}

__device__ __forceinline__ double ausm_up_flux(const double* UL, const double* UR, double nx, double ny, double g,
                                               double* F) {
  constexpr double BETA = 0.125, ALPHA = 0.1875, KP = 0.4, KU = 0.2;
  const Prim L = primitives(UL, g), R = primitives(UR, g);
  const double vnL = L.vx * nx + L.vy * ny, vnR = R.vx * nx + R.vy * ny;
  const double aL = sqrt(g * L.p / L.rho), aR = sqrt(g * R.p / R.rho);
  const double ah = 0.5 * (aL + aR), rh = 0.5 * (L.rho + R.rho);
  const double mL = vnL / ah, mR = vnR / ah;
  const double mb2 = 0.5 * (mL * mL + mR * mR);
  const double pL2 = 0.25 * ((mL + 1.0) * (mL + 1.0)), mL2 = -0.25 * ((mL - 1.0) * (mL - 1.0));
  const double pR2 = 0.25 * ((mR + 1.0) * (mR + 1.0)), mR2 = -0.25 * ((mR - 1.0) * (mR - 1.0));
  const double m4p = fabs(mL) >= 1.0 ? 0.5 * (mL + fabs(mL)) : pL2 * (1.0 - 16.0 * BETA * mL2);
  const double m4m = fabs(mR) >= 1.0 ? 0.5 * (mR - fabs(mR)) : mR2 * (1.0 + 16.0 * BETA * pR2);
  const double dif = 1.0 - mb2;
  const double uh = ah * (m4p + m4m) + KP * (dif < 0.0 ? 0.0 : dif) * (L.p - R.p) / (rh * ah);
  const double p5p = fabs(mL) >= 1.0 ? (mL > 0.0 ? 1.0 : 0.0) : pL2 * ((2.0 - mL) - 16.0 * ALPHA * mL * mL2);
  const double p5m = fabs(mR) >= 1.0 ? (mR > 0.0 ? 0.0 : 1.0) : mR2 * ((-2.0 - mR) + 16.0 * ALPHA * mR * pR2);
  const double ph = p5p * L.p + p5m * R.p + KU * p5p * p5m * rh * ah * (vnL - vnR);
  const double PL[4] = {L.rho, L.rho * L.vx, L.rho * L.vy, UL[3] + L.p};
  const double PR[4] = {R.rho, R.rho * R.vx, R.rho * R.vy, UR[3] + R.p};
  const double au = fabs(uh);
#pragma unroll
  for (int s = 0; s < 4; ++s) F[s] = 0.5 * uh * (PL[s] + PR[s]) - 0.5 * au * (PR[s] - PL[s]);
  F[1] = F[1] + ph * nx;
  F[2] = F[2] + ph * ny;
  F[0] = F[0] + ph * 0.0;
  F[3] = F[3] + ph * 0.0;
  return fmax(fabs(vnL) + aL, fabs(vnR) + aR);
}

__device__ __forceinline__ double wall_flux(const double* U, double nx, double ny, double g, double* F) {
  const double rho = floor_at(U[0], FLOOR);
  const double vx = U[1] / rho, vy = U[2] / rho;
  const double vn = vx * nx + vy * ny;
  const double tx = vx - vn * nx, ty = vy - vn * ny;
  const double pb = floor_at((g - 1.0) * (U[3] - 0.5 * rho * (tx * tx + ty * ty)), FLOOR);
  F[0] = 0.0;
  F[1] = pb * nx;
  F[2] = pb * ny;
  F[3] = 0.0;
  return sqrt(g * pb / rho);
}

__device__ __forceinline__ double inflow_flux(const double* U, double nx, double ny, const nzb_physics& ph,
                                              double* F) {
  const double g = ph.gamma;
  const Prim s = primitives(U, g);
  const double a = sqrt(g * s.p / s.rho);
  const double vn = s.vx * nx + s.vy * ny;
  const double Jp = vn + 2.0 * a / (g - 1.0);
  const double r = Jp / ph.in_at;
  const double beta = r * r;
  const double nd = nx * ph.in_cos + ny * ph.in_sin;
  double qa = 0.5 * (g - 1.0) * beta - nd * nd;
  const double qb = -4.0 * nd / (g - 1.0);
  const double k = 2.0 / (g - 1.0);
  const double qc = beta - k * k;
  if (fabs(qa) < 1e-12) qa = qa >= 0.0 ? 1e-12 : -1e-12;
  double disc = qb * qb - 4.0 * qa * qc;
  disc = disc < 0.0 ? 0.0 : disc;
  const double sq = sqrt(disc);
  const double r1 = (-qb + sq) / (2.0 * qa), r2 = (-qb - sq) / (2.0 * qa);
  const double c1 = r1 >= 0.0 ? r1 : 1e30, c2 = r2 >= 0.0 ? r2 : 1e30;
  double M = fmin(c1, c2);
  M = M > 0.5e30 ? 0.0 : M;
  M = M < 0.0 ? 0.0 : (M > 1.0 ? 1.0 : M);
  const double fac = 1.0 + 0.5 * (g - 1.0) * M * M;
  const double ab = sqrt(ph.in_at2 / fac);
  const double qbv = M * ab;
  const double vxb = qbv * ph.in_cos, vyb = qbv * ph.in_sin;
  const double rhob = ph.in_rho_t * pow(fac, -1.0 / (g - 1.0));
  const double pb = rhob * ab * ab / g;
  const double Hb = ph.in_at2 / (g - 1.0);
  const double vnb = vxb * nx + vyb * ny;
  F[0] = rhob * vnb;
  F[1] = rhob * vxb * vnb + pb * nx;
  F[2] = rhob * vyb * vnb + pb * ny;
  F[3] = rhob * Hb * vnb;
  return fabs(vnb) + ab;
}

__device__ __forceinline__ double outflow_flux(const double* U, double nx, double ny, const nzb_physics& ph,
                                               double p_back, double* F) {
  const double g = ph.gamma;
  const Prim s = primitives(U, g);
  const double a = sqrt(g * s.p / s.rho);
  const double vn = s.vx * nx + s.vy * ny;
  double Ub[4];
  if (vn / a >= 1.0) {
    Ub[0] = U[0]; Ub[1] = U[1]; Ub[2] = U[2]; Ub[3] = U[3];
  } else {
    const double pb = p_back;
    const double rhob = s.rho * pow(pb / s.p, 1.0 / g);
    const double ab = sqrt(g * pb / rhob);
    const double vnb = vn + 2.0 / (g - 1.0) * (a - ab);
    const double vxb = (s.vx - vn * nx) + vnb * nx;
    const double vyb = (s.vy - vn * ny) + vnb * ny;
    const double Eb = pb / ((g - 1.0) * rhob) + 0.5 * (vxb * vxb + vyb * vyb);
    Ub[0] = rhob; Ub[1] = rhob * vxb; Ub[2] = rhob * vyb; Ub[3] = rhob * Eb;
    if (ph.bf_rho_t > 0.0) {
      const double rf = ph.bf_rho_t * pow(pb / ph.bf_p_t, 1.0 / g);
      const double af = sqrt(g * pb / rf);
      const double vnf = vn + 2.0 / (g - 1.0) * (a - af);
      const double vxf = vnf * nx, vyf = vnf * ny;
      const double Ef = pb / ((g - 1.0) * rf) + 0.5 * (vxf * vxf + vyf * vyf);
      const double Uf[4] = {rf, rf * vxf, rf * vyf, rf * Ef};
      double t = (vn / a) / fmax(ph.bf_band, 1e-12);
      t = t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
#pragma unroll
      for (int c = 0; c < 4; ++c) Ub[c] = t * Ub[c] + (1.0 - t) * Uf[c];
    }
  }
  const Prim o = primitives(Ub, g);
  normal_flux(o, nx, ny, F);
  return fabs(o.vx * nx + o.vy * ny) + sqrt(g * o.p / o.rho);
}

__device__ __forceinline__ double interface_flux(const double* UL, const double* UR, double nx, double ny,
                                                 const nzb_physics& ph, double* F) {
  if (ph.flux == NZB_HLLC) return hllc_flux(UL, UR, nx, ny, ph.gamma, ph.hllc_low_mach, F);
  if (ph.flux == NZB_AUSMUP) return ausm_up_flux(UL, UR, nx, ny, ph.gamma, F);
  return roe_flux(UL, UR, nx, ny, ph.gamma, ph.entropy_fix, F);
}

__device__ __forceinline__ double boundary_flux(int tag, const double* U, double nx, double ny,
                                                const nzb_physics& ph, double p_back, double* F) {
  if (tag == NZB_INFLOW) return inflow_flux(U, nx, ny, ph, F);
  if (tag == NZB_OUTFLOW) return outflow_flux(U, nx, ny, ph, p_back, F);
  return wall_flux(U, nx, ny, ph.gamma, F);
}

}  // namespace nzb
