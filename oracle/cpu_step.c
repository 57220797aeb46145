/* cpu_step.c -- TEST INFRASTRUCTURE: the reference's compiled CPU step, restated
 * in C with OpenMP, so the CPU baseline is timed on the same kind of code the
 * reference runs (its Numba backend), not on a vectorised NumPy restatement.
 *
 * It is never part of the product: only the CPU-baseline legs of bench.py and
 * the tests that check it against the NumPy oracle load it.
 *
 * The execution strategy follows src/backends/numba_backend.py:283-337 and
 * src/backends/_numba_kernels.py:
 *   - the reference layout U (E, NP, 4) and its per-element operators with the
 *     inverse mass folded in (grad_x_m, grad_y_m (E, NP, nqv); face_basis_m
 *     (E, nface, NP, nqf); src/spatial/operators.py:309-320);
 *   - an edge pass, one iteration per edge (interior edges first, then the
 *     boundary edges): both traces, the Riemann solver or the boundary flux,
 *     fw = flux * |dX/dsigma| * w and the edge's largest signal speed
 *     (_numba_kernels.py:484-583);
 *   - an element pass: the volume term, then the face terms gathered through
 *     face_edge with face_sign, the rate -M^-1 R and the wave-speed sum
 *     (:586-664);
 *   - the local step, the weighted norm of stage 1's rate, the stage and
 *     combine updates (:789-850) and the positivity limiter in place after
 *     every stage: mean repair, the Lebesgue screen, the probe minima, the
 *     closed-form density factor and the 12-step pressure bisection
 *     (:856-1093).
 * Fluxes: Roe with the Harten-Hyman fix, HLLC with Batten's speeds and the
 * optional low-Mach scaling, AUSM+-up; slip wall, stagnation inflow, pressure
 * outflow with the optional backflow blend (:60-471).  The pressure is
 * (gamma - 1)(rhoE - |m|^2 / (2 rho)) with rho and p floored at 1e-10, as the
 * compiled path forms it.
 *
 * Built with -O3, FMA contraction and reassociation allowed (the reference
 * compiles with fastmath), OpenMP over edges and elements.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define FLOOR 1e-10
enum { INFLOW = 1, OUTFLOW = 2, WALL = 3, AXIS = 4 };

typedef struct {
  int64_t n_elem, n_int, n_bnd;
  int32_t nbf, nqv, nqf, nface;
  const double *phi_vol;      /* (nbf, nqv) */
  const double *phi_face;     /* (2, nface, nbf, nqf) */
  const double *w_face;       /* (nqf) */
  const double *grad_x_m;     /* (E, nbf, nqv) */
  const double *grad_y_m;     /* (E, nbf, nqv) */
  const double *face_basis_m; /* (E, nface, nbf, nqf) */
  const int64_t *face_edge;   /* (E, nface) */
  const int64_t *face_side;   /* (E, nface) */
  const double *face_sign;    /* (E, nface) */
  const double *edge_normal;  /* (n_edge, nqf, 2) */
  const double *edge_jac;     /* (n_edge, nqf) */
  const double *edge_length;  /* (n_edge) */
  const double *elem_area;    /* (E) */
  const double *mean_weights; /* (E, nbf) */
  const int64_t *iedge_elem;  /* (n_int, 2) */
  const int64_t *iedge_face;  /* (n_int, 2) */
  const int64_t *bedge_elem;  /* (n_bnd) */
  const int64_t *bedge_face;  /* (n_bnd) */
  const int64_t *bedge_tag;   /* (n_bnd) */
  double gamma, efix, low_mach;
  double rho_t_bf, p_t_bf, band_bf; /* backflow: reservoir density (0: off), total pressure, band */
  double at2, at, rho_t, ca, sa, p_back;
  int32_t flux_id;                  /* 0 Roe, 1 HLLC, 2 AUSM+-up */
  int32_t limiter;                  /* 0 none, 1 positivity */
  double rho_floor, p_floor, fraction, lebesgue;
  int32_t steps, pad;
  double dt_factor; /* positivity scale * cfl / (2p + 1) */
  double weight[4]; /* norm weights per component */
  /* caller-allocated work arrays */
  double *fw, *smax, *wave, *dt, *F0, *F1, *F2, *S0, *S1, *S2;
} cpu_case;

static inline double pressure(double u0, double u1, double u2, double u3, double g) {
  const double rho = u0 > FLOOR ? u0 : FLOOR;
  const double p = (g - 1.0) * (u3 - 0.5 * (u1 * u1 + u2 * u2) / rho);
  return p > FLOOR ? p : FLOOR;
}

static inline void normal_flux(double u0, double u1, double u2, double u3, double nx, double ny, double g, double *f) {
  const double rho = u0 > FLOOR ? u0 : FLOOR;
  const double vx = u1 / rho, vy = u2 / rho;
  const double p = pressure(u0, u1, u2, u3, g);
  const double H = (u3 + p) / rho, vn = vx * nx + vy * ny;
  f[0] = rho * vn;
  f[1] = rho * vx * vn + p * nx;
  f[2] = rho * vy * vn + p * ny;
  f[3] = rho * H * vn;
}

/* The left/right primitive states a Riemann solver starts from. */
typedef struct { double r, vx, vy, p, H, vn; } side_t;

static inline side_t side_state(const double *U, double nx, double ny, double g) {
  side_t s;
  s.r = U[0] > FLOOR ? U[0] : FLOOR;
  s.vx = U[1] / s.r;
  s.vy = U[2] / s.r;
  s.p = pressure(U[0], U[1], U[2], U[3], g);
  s.H = (U[3] + s.p) / s.r;
  s.vn = s.vx * nx + s.vy * ny;
  return s;
}

static double roe(const double *UL, const double *UR, double nx, double ny, double g, double efix, double *out) {
  const side_t L = side_state(UL, nx, ny, g), R = side_state(UR, nx, ny, g);
  const double fL[4] = {L.r * L.vn, L.r * L.vx * L.vn + L.p * nx, L.r * L.vy * L.vn + L.p * ny, L.r * L.H * L.vn};
  const double fR[4] = {R.r * R.vn, R.r * R.vx * R.vn + R.p * nx, R.r * R.vy * R.vn + R.p * ny, R.r * R.H * R.vn};
  const double sl = sqrt(L.r), sr = sqrt(R.r), den = sl + sr;
  const double vx = (sl * L.vx + sr * R.vx) / den, vy = (sl * L.vy + sr * R.vy) / den;
  const double H = (sl * L.H + sr * R.H) / den, q2 = vx * vx + vy * vy;
  double c2 = (g - 1.0) * (H - 0.5 * q2);
  if (c2 < FLOOR) c2 = FLOOR;
  const double c = sqrt(c2), vn = vx * nx + vy * ny;
  double l1 = fabs(vn + c), l2 = fabs(vn - c), l3 = fabs(vn);
  const double smax = l1 > l2 ? l1 : l2;
  const double eps = efix * c;
  if (eps > 0.0) {
    if (l1 < eps) l1 = (l1 * l1 + eps * eps) / (2.0 * eps);
    if (l2 < eps) l2 = (l2 * l2 + eps * eps) / (2.0 * eps);
    if (l3 < eps) l3 = (l3 * l3 + eps * eps) / (2.0 * eps);
  }
  const double d0 = UR[0] - UL[0], d1 = UR[1] - UL[1], d2 = UR[2] - UL[2], d3 = UR[3] - UL[3];
  const double G1 = (g - 1.0) * (0.5 * q2 * d0 - vx * d1 - vy * d2 + d3);
  const double G2 = -vn * d0 + d1 * nx + d2 * ny;
  const double s1 = 0.5 * (l1 + l2), s2 = 0.5 * (l1 - l2);
  const double C1 = (G1 / c2) * (s1 - l3) + (G2 / c) * s2;
  const double C2 = (G1 / c) * s2 + (s1 - l3) * G2;
  out[0] = 0.5 * (fL[0] + fR[0]) - 0.5 * (l3 * d0 + C1);
  out[1] = 0.5 * (fL[1] + fR[1]) - 0.5 * (l3 * d1 + C1 * vx + C2 * nx);
  out[2] = 0.5 * (fL[2] + fR[2]) - 0.5 * (l3 * d2 + C1 * vy + C2 * ny);
  out[3] = 0.5 * (fL[3] + fR[3]) - 0.5 * (l3 * d3 + C1 * H + C2 * vn);
  return smax;
}

static double hllc(const double *UL, const double *UR, double nx, double ny, double g, double low_mach, double *out) {
  const side_t L = side_state(UL, nx, ny, g), R = side_state(UR, nx, ny, g);
  const double aL = sqrt(fmax(g * L.p / L.r, FLOOR)), aR = sqrt(fmax(g * R.p / R.r, FLOOR));
  const double sl = sqrt(L.r), sr = sqrt(R.r), den = sl + sr;
  const double vx = (sl * L.vx + sr * R.vx) / den, vy = (sl * L.vy + sr * R.vy) / den;
  const double H = (sl * L.H + sr * R.H) / den, vt = vx * nx + vy * ny;
  double c2 = (g - 1.0) * (H - 0.5 * (vx * vx + vy * vy));
  if (c2 < FLOOR) c2 = FLOOR;
  const double at = sqrt(c2);
  double SL = fmin(L.vn - aL, vt - at), SR = fmax(R.vn + aR, vt + at);
  if (low_mach > 0.0) {
    const double mach = fmax(fabs(L.vn) / aL, fabs(R.vn) / aR);
    const double phi = fmin(1.0, mach / low_mach);
    const double bL = fmin(L.vn, vt), bR = fmax(R.vn, vt);
    SL = bL - phi * (bL - SL);
    SR = bR + phi * (SR - bR);
  }
  const double smax = fmax(fabs(SL), fabs(SR));
  const double fL[4] = {L.r * L.vn, L.r * L.vx * L.vn + L.p * nx, L.r * L.vy * L.vn + L.p * ny, L.r * L.H * L.vn};
  if (SL >= 0.0) {
    memcpy(out, fL, sizeof fL);
    return smax;
  }
  const double fR[4] = {R.r * R.vn, R.r * R.vx * R.vn + R.p * nx, R.r * R.vy * R.vn + R.p * ny, R.r * R.H * R.vn};
  if (SR <= 0.0) {
    memcpy(out, fR, sizeof fR);
    return smax;
  }
  double dm = R.r * (SR - R.vn) - L.r * (SL - L.vn);
  if (fabs(dm) < FLOOR) dm = FLOOR;
  const double SM = (R.r * R.vn * (SR - R.vn) - L.r * L.vn * (SL - L.vn) + L.p - R.p) / dm;
  /* the star state on the side of the contact that holds the interface */
  const int left = SM >= 0.0;
  const side_t *Q = left ? &L : &R;
  const double *UQ = left ? UL : UR, *fQ = left ? fL : fR;
  const double S = left ? SL : SR;
  double d2 = S - SM;
  if (fabs(d2) < FLOOR) d2 = FLOOR;
  const double rs = Q->r * ((S - Q->vn) / d2);
  const double vxs = Q->vx + (SM - Q->vn) * nx, vys = Q->vy + (SM - Q->vn) * ny;
  double d3 = Q->r * (S - Q->vn);
  if (fabs(d3) < FLOOR) d3 = FLOOR;
  const double Es = UQ[3] / Q->r + (SM - Q->vn) * (SM + Q->p / d3);
  out[0] = fQ[0] + S * (rs - UQ[0]);
  out[1] = fQ[1] + S * (rs * vxs - UQ[1]);
  out[2] = fQ[2] + S * (rs * vys - UQ[2]);
  out[3] = fQ[3] + S * (rs * Es - UQ[3]);
  return smax;
}

/* AUSM+-up split functions (beta 1/8, alpha 3/16) */
static inline double m4(double m, int plus) {
  if (fabs(m) >= 1.0) return 0.5 * (m + (plus ? fabs(m) : -fabs(m)));
  const double mp = 0.25 * (m + 1.0) * (m + 1.0), mm = -0.25 * (m - 1.0) * (m - 1.0);
  return plus ? mp * (1.0 - 2.0 * mm) : mm * (1.0 + 2.0 * mp);
}
static inline double p5(double m, int plus) {
  if (m >= 1.0) return plus ? 1.0 : 0.0;
  if (m <= -1.0) return plus ? 0.0 : 1.0;
  const double mp = 0.25 * (m + 1.0) * (m + 1.0), mm = -0.25 * (m - 1.0) * (m - 1.0);
  return plus ? mp * ((2.0 - m) - 3.0 * m * mm) : mm * ((-2.0 - m) + 3.0 * m * mp);
}

static double ausm_up(const double *UL, const double *UR, double nx, double ny, double g, double *out) {
  const side_t L = side_state(UL, nx, ny, g), R = side_state(UR, nx, ny, g);
  const double aL = sqrt(fmax(g * L.p / L.r, FLOOR)), aR = sqrt(fmax(g * R.p / R.r, FLOOR));
  const double ah = 0.5 * (aL + aR), rh = 0.5 * (L.r + R.r);
  const double mL = L.vn / ah, mR = R.vn / ah;
  double diff = 1.0 - 0.5 * (mL * mL + mR * mR);
  if (diff < 0.0) diff = 0.0;
  const double uh = ah * (m4(mL, 1) + m4(mR, 0)) + 0.4 * diff * (L.p - R.p) / (rh * ah);
  const double pp = p5(mL, 1), pm = p5(mR, 0);
  const double ph = pp * L.p + pm * R.p + 0.2 * pp * pm * rh * ah * (L.vn - R.vn);
  const double *U = uh > 0.0 ? UL : UR;
  const double r = uh > 0.0 ? L.r : R.r, p = uh > 0.0 ? L.p : R.p;
  out[0] = uh * r;
  out[1] = uh * U[1] + ph * nx;
  out[2] = uh * U[2] + ph * ny;
  out[3] = uh * (U[3] + p);
  const double sL = fabs(L.vn) + aL, sR = fabs(R.vn) + aR;
  return sL > sR ? sL : sR;
}

static double wall(const double *U, double nx, double ny, double g, double *out) {
  const double rho = U[0] > FLOOR ? U[0] : FLOOR;
  const double vx = U[1] / rho, vy = U[2] / rho, vn = vx * nx + vy * ny;
  const double tx = vx - vn * nx, ty = vy - vn * ny;
  double pb = (g - 1.0) * (U[3] - 0.5 * rho * (tx * tx + ty * ty));
  if (pb < FLOOR) pb = FLOOR;
  out[0] = 0.0;
  out[1] = pb * nx;
  out[2] = pb * ny;
  out[3] = 0.0;
  return sqrt(g * pb / rho);
}

static double inflow(const double *U, double nx, double ny, const cpu_case *c, double *out) {
  const double g = c->gamma;
  const double rho = U[0] > FLOOR ? U[0] : FLOOR;
  const double vx = U[1] / rho, vy = U[2] / rho;
  const double p = pressure(U[0], U[1], U[2], U[3], g);
  const double a = sqrt(g * p / rho), vn = vx * nx + vy * ny;
  const double Jp = vn + 2.0 * a / (g - 1.0);
  const double beta = (Jp / c->at) * (Jp / c->at), nd = nx * c->ca + ny * c->sa;
  double aa = 0.5 * (g - 1.0) * beta - nd * nd;
  const double bb = -4.0 * nd / (g - 1.0), cc = beta - (2.0 / (g - 1.0)) * (2.0 / (g - 1.0));
  if (fabs(aa) < 1e-12) aa = aa >= 0.0 ? 1e-12 : -1e-12;
  double disc = bb * bb - 4.0 * aa * cc;
  if (disc < 0.0) disc = 0.0;
  const double sq = sqrt(disc), r1 = (-bb + sq) / (2.0 * aa), r2 = (-bb - sq) / (2.0 * aa);
  double M = -1.0;  /* the smallest non-negative root, clamped to [0, 1] */
  if (r1 >= 0.0) M = r1;
  if (r2 >= 0.0 && (M < 0.0 || r2 < M)) M = r2;
  M = M < 0.0 ? 0.0 : (M > 1.0 ? 1.0 : M);
  const double fac = 1.0 + 0.5 * (g - 1.0) * M * M;
  const double ab = sqrt(c->at2 / fac), qb = M * ab;
  const double vxb = qb * c->ca, vyb = qb * c->sa;
  const double rhob = c->rho_t * pow(fac, -1.0 / (g - 1.0));
  const double pb = rhob * ab * ab / g, Hb = c->at2 / (g - 1.0), vnb = vxb * nx + vyb * ny;
  out[0] = rhob * vnb;
  out[1] = rhob * vxb * vnb + pb * nx;
  out[2] = rhob * vyb * vnb + pb * ny;
  out[3] = rhob * Hb * vnb;
  return fabs(vnb) + ab;
}

static double outflow(const double *U, double nx, double ny, const cpu_case *c, double *out) {
  const double g = c->gamma, pbk = c->p_back;
  const double rho = U[0] > FLOOR ? U[0] : FLOOR;
  const double vx = U[1] / rho, vy = U[2] / rho;
  const double p = pressure(U[0], U[1], U[2], U[3], g);
  const double a = sqrt(g * p / rho), vn = vx * nx + vy * ny;
  if (vn / a >= 1.0) {  /* supersonic: extrapolate */
    normal_flux(U[0], U[1], U[2], U[3], nx, ny, g, out);
    return fabs(vn) + a;
  }
  const double rhob = rho * pow(pbk / p, 1.0 / g), ab = sqrt(g * pbk / rhob);
  const double vnb = vn + 2.0 / (g - 1.0) * (a - ab);
  const double vxb = (vx - vn * nx) + vnb * nx, vyb = (vy - vn * ny) + vnb * ny;
  const double Eb = pbk / ((g - 1.0) * rhob) + 0.5 * (vxb * vxb + vyb * vyb);
  if (c->rho_t_bf > 0.0 && vn / a < c->band_bf) {  /* backflow: blend toward the reservoir state */
    const double rf = c->rho_t_bf * pow(pbk / c->p_t_bf, 1.0 / g), af = sqrt(g * pbk / rf);
    const double vnf = vn + 2.0 / (g - 1.0) * (a - af), vxf = vnf * nx, vyf = vnf * ny;
    const double Ef = pbk / ((g - 1.0) * rf) + 0.5 * (vxf * vxf + vyf * vyf);
    double t = (vn / a) / c->band_bf;
    if (t < 0.0) t = 0.0;
    normal_flux(t * rhob + (1.0 - t) * rf, t * (rhob * vxb) + (1.0 - t) * (rf * vxf),
                t * (rhob * vyb) + (1.0 - t) * (rf * vyf), t * (rhob * Eb) + (1.0 - t) * (rf * Ef), nx, ny, g, out);
    return fabs(vnb) + ab;
  }
  normal_flux(rhob, rhob * vxb, rhob * vyb, rhob * Eb, nx, ny, g, out);
  return fabs(vnb) + ab;
}

/* ---- edge pass: fw (n_edge, nqf, 4), smax (n_edge) */
static void edge_pass(const cpu_case *c, const double *U) {
  const int nbf = c->nbf, nqf = c->nqf, nface = c->nface;
  const int64_t n_int = c->n_int, n_edge = c->n_int + c->n_bnd;
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < n_edge; ++k) {
    double UL[4], UR[4], F[4], best = 0.0;
    const int interior = k < n_int;
    int64_t le, re = 0;
    int lf, rf = 0, tag = 0;
    if (interior) {
      le = c->iedge_elem[2 * k];
      re = c->iedge_elem[2 * k + 1];
      lf = (int)c->iedge_face[2 * k];
      rf = (int)c->iedge_face[2 * k + 1];
    } else {
      const int64_t b = k - n_int;
      le = c->bedge_elem[b];
      lf = (int)c->bedge_face[b];
      tag = (int)c->bedge_tag[b];
    }
    const double *Ul = U + le * nbf * 4, *Ur = U + re * nbf * 4;
    for (int q = 0; q < nqf; ++q) {
      for (int s = 0; s < 4; ++s) UL[s] = UR[s] = 0.0;
      for (int i = 0; i < nbf; ++i) {
        const double bl = c->phi_face[((0 * nface + lf) * nbf + i) * nqf + q];
        for (int s = 0; s < 4; ++s) UL[s] += bl * Ul[i * 4 + s];
        if (interior) {
          const double br = c->phi_face[((1 * nface + rf) * nbf + i) * nqf + q];
          for (int s = 0; s < 4; ++s) UR[s] += br * Ur[i * 4 + s];
        }
      }
      const double nx = c->edge_normal[(k * nqf + q) * 2], ny = c->edge_normal[(k * nqf + q) * 2 + 1];
      double sp;
      if (interior) {
        sp = c->flux_id == 1 ? hllc(UL, UR, nx, ny, c->gamma, c->low_mach, F)
           : c->flux_id == 2 ? ausm_up(UL, UR, nx, ny, c->gamma, F)
                             : roe(UL, UR, nx, ny, c->gamma, c->efix, F);
      } else if (tag == INFLOW) {
        sp = inflow(UL, nx, ny, c, F);
      } else if (tag == OUTFLOW) {
        sp = outflow(UL, nx, ny, c, F);
      } else {
        sp = wall(UL, nx, ny, c->gamma, F);
      }
      if (sp > best) best = sp;
      const double scale = c->edge_jac[k * nqf + q] * c->w_face[q];
      for (int s = 0; s < 4; ++s) c->fw[(k * nqf + q) * 4 + s] = F[s] * scale;
    }
    c->smax[k] = best;
  }
}

/* ---- element pass: out = -M^-1 R (E, nbf, 4), wave (E) */
static void element_rate(const cpu_case *c, const double *U, double *out) {
  const int nbf = c->nbf, nqv = c->nqv, nqf = c->nqf, nface = c->nface;
  const double g = c->gamma;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < c->n_elem; ++e) {
    double Rm[64 * 4];
    memset(Rm, 0, sizeof(double) * 4 * nbf);
    const double *Ue = U + e * nbf * 4;
    const double *gx = c->grad_x_m + e * nbf * nqv, *gy = c->grad_y_m + e * nbf * nqv;
    for (int q = 0; q < nqv; ++q) {
      double u[4] = {0.0, 0.0, 0.0, 0.0};
      for (int i = 0; i < nbf; ++i) {
        const double b = c->phi_vol[i * nqv + q];
        for (int s = 0; s < 4; ++s) u[s] += b * Ue[i * 4 + s];
      }
      const double rho = u[0] > FLOOR ? u[0] : FLOOR;
      const double vx = u[1] / rho, vy = u[2] / rho;
      const double p = pressure(u[0], u[1], u[2], u[3], g), H = (u[3] + p) / rho;
      const double F[4] = {rho * vx, rho * vx * vx + p, rho * vx * vy, rho * vx * H};
      const double G[4] = {rho * vy, rho * vx * vy, rho * vy * vy + p, rho * vy * H};
      for (int i = 0; i < nbf; ++i) {
        const double a = gx[i * nqv + q], b = gy[i * nqv + q];
        for (int s = 0; s < 4; ++s) Rm[i * 4 + s] -= a * F[s] + b * G[s];
      }
    }
    double acc = 0.0;
    for (int f = 0; f < nface; ++f) {
      const int64_t k = c->face_edge[e * nface + f];
      const double sg = c->face_sign[e * nface + f];
      const double *fb = c->face_basis_m + (e * nface + f) * nbf * nqf;
      for (int q = 0; q < nqf; ++q) {
        const double *fw = c->fw + (k * nqf + q) * 4;
        for (int i = 0; i < nbf; ++i) {
          const double b = sg * fb[i * nqf + q];
          for (int s = 0; s < 4; ++s) Rm[i * 4 + s] += b * fw[s];
        }
      }
      acc += c->smax[k] * c->edge_length[k];
    }
    c->wave[e] = acc;
    for (int i = 0; i < 4 * nbf; ++i) out[e * nbf * 4 + i] = -Rm[i];
  }
}

/* ---- positivity limiter, in place; counts into n[0] (scaled), n[1] (repaired) */
static void probe_minima(const cpu_case *c, const double *Ue, const double *ub, double theta, const int64_t *fside,
                         double *rmin, double *pmin) {
  const int nbf = c->nbf, nqv = c->nqv, nqf = c->nqf, nface = c->nface;
  const double g = c->gamma;
  double rm = 1e300, pm = 1e300;
  const int npt = nqv + nface * nqf;
  for (int pt = 0; pt < npt; ++pt) {
    double u[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < nbf; ++i) {
      double b;
      if (pt < nqv) {
        b = c->phi_vol[i * nqv + pt];
      } else {
        const int f = (pt - nqv) / nqf, q = (pt - nqv) % nqf;
        b = c->phi_face[((fside[f] * nface + f) * nbf + i) * nqf + q];
      }
      for (int s = 0; s < 4; ++s) u[s] += b * Ue[i * 4 + s];
    }
    for (int s = 0; s < 4; ++s) u[s] = ub[s] + theta * (u[s] - ub[s]);
    if (u[0] < rm) rm = u[0];
    const double r = u[0] > 1e-300 ? u[0] : 1e-300;
    const double pp = (g - 1.0) * (u[3] - 0.5 * (u[1] * u[1] + u[2] * u[2]) / r);
    if (pp < pm) pm = pp;
  }
  *rmin = rm;
  *pmin = pm;
}

static void limit(const cpu_case *c, double *U, int64_t *counters) {
  if (!c->limiter) return;
  const int nbf = c->nbf, nface = c->nface;
  const double g1 = c->gamma - 1.0, lam = c->lebesgue;
  int64_t n_scaled = 0, n_repair = 0;
#pragma omp parallel for schedule(static) reduction(+ : n_scaled, n_repair)
  for (int64_t e = 0; e < c->n_elem; ++e) {
    double *Ue = U + e * nbf * 4;
    double ub[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < nbf; ++i) {
      const double w = c->mean_weights[e * nbf + i];
      for (int s = 0; s < 4; ++s) ub[s] += w * Ue[i * 4 + s];
    }
    const double rho_new = ub[0] > c->rho_floor ? ub[0] : c->rho_floor;
    const double e_min = c->p_floor / g1 + 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) / rho_new;
    const double rhoE_new = ub[3] > e_min ? ub[3] : e_min;
    const double d0 = rho_new - ub[0], d3 = rhoE_new - ub[3];
    if (d0 != 0.0 || d3 != 0.0) {
      for (int i = 0; i < nbf; ++i) {
        Ue[i * 4] += d0;
        Ue[i * 4 + 3] += d3;
      }
      ub[0] = rho_new;
      ub[3] = rhoE_new;
      ++n_repair;
    }
    const double pbar = g1 * (ub[3] - 0.5 * (ub[1] * ub[1] + ub[2] * ub[2]) / ub[0]);
    double eps_r = c->fraction * ub[0], eps_p = c->fraction * pbar;
    if (eps_r < 0.5 * c->rho_floor) eps_r = 0.5 * c->rho_floor;
    if (eps_p < 0.5 * c->p_floor) eps_p = 0.5 * c->p_floor;
    double dv[4] = {0.0, 0.0, 0.0, 0.0};
    for (int i = 0; i < nbf; ++i)
      for (int s = 0; s < 4; ++s) {
        const double a = fabs(Ue[i * 4 + s] - ub[s]);
        if (a > dv[s]) dv[s] = a;
      }
    const double rho_lo = ub[0] - lam * dv[0];
    if (rho_lo >= eps_r) {
      const double m_hi = sqrt(ub[1] * ub[1] + ub[2] * ub[2]) + lam * sqrt(dv[1] * dv[1] + dv[2] * dv[2]);
      if (g1 * (ub[3] - lam * dv[3] - 0.5 * m_hi * m_hi / rho_lo) >= eps_p) continue;
    }
    const int64_t *fside = c->face_side + e * nface;
    double rmin, pmin;
    probe_minima(c, Ue, ub, 1.0, fside, &rmin, &pmin);
    if (rmin >= eps_r && pmin >= eps_p) continue;
    double theta = 1.0;
    if (rmin < eps_r) {
      const double gap = ub[0] - rmin;
      theta = gap <= 0.0 ? 0.0 : (ub[0] - eps_r) / gap;
      theta = theta < 0.0 ? 0.0 : (theta > 1.0 ? 1.0 : theta);
    }
    double r_, p_hi;
    probe_minima(c, Ue, ub, theta, fside, &r_, &p_hi);
    if (p_hi < eps_p) {
      double lo = 0.0, hi = theta;
      for (int it = 0; it < c->steps; ++it) {
        const double mid = 0.5 * (lo + hi);
        double pm;
        probe_minima(c, Ue, ub, mid, fside, &r_, &pm);
        if (pm >= eps_p)
          lo = mid;
        else
          hi = mid;
      }
      theta = lo;
    }
    for (int i = 0; i < nbf; ++i)
      for (int s = 0; s < 4; ++s) Ue[i * 4 + s] = ub[s] + theta * (Ue[i * 4 + s] - ub[s]);
    ++n_scaled;
  }
  if (counters) {
    counters[0] += n_scaled;
    counters[1] += n_repair;
  }
}

static double rms_weighted(const cpu_case *c, const double *A) {
  const int64_t n = c->n_elem * c->nbf;
  double total = 0.0;
#pragma omp parallel for schedule(static) reduction(+ : total)
  for (int64_t k = 0; k < n; ++k)
    for (int s = 0; s < 4; ++s) {
      const double v = A[k * 4 + s] * c->weight[s];
      total += v * v;
    }
  return sqrt(total / (double)(n * 4));
}

static void local_dt(const cpu_case *c) {
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < c->n_elem; ++e) {
    const double d = c->wave[e] < FLOOR ? FLOOR : c->wave[e];
    c->dt[e] = c->dt_factor * 2.0 * c->elem_area[e] / d;
  }
}

/* out = a U + b (V + dt F), with a = 0 meaning out = V + dt F */
static void combine(const cpu_case *c, const double *U, const double *V, const double *F, double a, double b,
                    double *out) {
  const int m = c->nbf * 4;
#pragma omp parallel for schedule(static)
  for (int64_t e = 0; e < c->n_elem; ++e) {
    const double d = c->dt[e];
    for (int i = 0; i < m; ++i) {
      const int64_t k = e * m + i;
      out[k] = a == 0.0 ? V[k] + 1.0 * d * F[k] : a * U[k] + b * (V[k] + d * F[k]);
    }
  }
}

static double rate(const cpu_case *c, const double *U, double *F) {
  edge_pass(c, U);
  element_rate(c, U, F);
  return 0.0;
}

/* Advance n_steps SSP-RK3 (scheme 1) or forward-Euler (scheme 0) steps from U_in into U_out
 * (the reference's NumbaBackend.run); res receives the last step's residual norm. */
int cpu_run(const cpu_case *c, const double *U_in, double *U_out, int n_steps, int scheme, double *res,
            int64_t *counters) {
  if (c->nbf > 64) return -1;
  const int64_t n = c->n_elem * c->nbf * 4;
  double *cur = c->S0, *nxt = c->S1, *U1 = c->S2;
  memcpy(cur, U_in, sizeof(double) * n);
  double r = NAN;
  for (int it = 0; it < n_steps; ++it) {
    rate(c, cur, c->F0);
    local_dt(c);
    r = rms_weighted(c, c->F0);
    if (scheme == 0) {
      combine(c, cur, cur, c->F0, 0.0, 1.0, nxt);
      limit(c, nxt, counters);
    } else {
      combine(c, cur, cur, c->F0, 0.0, 1.0, U1);
      limit(c, U1, counters);
      rate(c, U1, c->F1);
      combine(c, cur, U1, c->F1, 0.75, 0.25, nxt);
      limit(c, nxt, counters);
      rate(c, nxt, c->F2);
      combine(c, cur, nxt, c->F2, 1.0 / 3.0, 2.0 / 3.0, U1);
      limit(c, U1, counters);
      memcpy(nxt, U1, sizeof(double) * n);
    }
    double *t = cur;
    cur = nxt;
    nxt = t;
  }
  memcpy(U_out, cur, sizeof(double) * n);
  if (res) *res = r;
  return 0;
}

/* The residual's rate -M^-1 R and the wave-speed sums (one edge and one element pass). */
int cpu_rate(const cpu_case *c, const double *U, double *out) {
  if (c->nbf > 64) return -1;
  rate(c, U, out);
  return 0;
}

void cpu_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n > 0 ? n : 1);
#else
  (void)n;
#endif
}

int cpu_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
