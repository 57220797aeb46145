"""CPU oracle for the DG residual / limiter / SSP-RK3 path -- TEST INFRASTRUCTURE.

This module is the checker, never the product: only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import it.
The CUDA backend never calls into it and has no CPU fallback.

It restates, in vectorised NumPy, the reference solver's NumPy path:

* primitives with density and pressure floored at 1e-10
  (src/physics/thermo.py:33,46-53) and the projected Euler flux (:73-80);
* Roe with the Harten-Hyman fix (src/physics/fluxes.py:38-103), HLLC with
  Batten's speeds and the optional low-Mach scaling (:106-255), AUSM+-up with
  beta=1/8, alpha=3/16, Kp=0.4, Ku=0.2 (:262-445);
* the slip wall, stagnation inflow and pressure outflow with the optional
  backflow blend (src/physics/boundary.py:20-214);
* the residual R = volume + face terms and the wave-speed sum
  (src/spatial/assembly.py:52-157), the block inverse mass (:160-162);
* the Zhang-Shu positivity limiter: cell-mean repair, 1e-8 margins, closed-form
  density factor, 12-step pressure bisection, probes at the volume points and
  the element's own face points (src/spatial/limiter.py:86-243);
* the local time step and the component-weighted RMS norm
  (src/timestepping/step.py:150-183, src/backends/base.py:42-78), the
  forward-Euler and SSP-RK3 steps (src/backends/base.py:155-179).

One deliberate difference from src/spatial/limiter.py:241-243: elements the
limiter leaves alone are returned untouched, as the reference's compiled path
does (src/backends/_numba_kernels.py:1030-1093), instead of being rebuilt as
``ubar + 1 * (U - ubar)``, which perturbs them by round-off.

Pinned against outputs of the reference itself in ``tests/golden`` (generated
by ``tests/golden/make_golden.py``).
"""

from __future__ import annotations

import numpy as np

FLOOR = 1e-10
INFLOW, OUTFLOW, WALL, AXIS = 1, 2, 3, 4


# ---------------------------------------------------------------- physics
def _abs(x):
    """|x|.  For a complex-step argument x + i h (h tiny), x times the sign of
    its real part: analytic, so the imaginary part carries the derivative of
    |x| (the modulus would drop it).  Real arguments go to numpy.abs."""
    if np.iscomplexobj(x):
        return np.where(np.real(x) < 0.0, -x, x)
    return np.abs(x)


def _sign(x):
    return np.sign(np.real(x))

def primitives(U, g):
    rho = np.maximum(U[..., 0], FLOOR)
    vx = U[..., 1] / rho
    vy = U[..., 2] / rho
    p = np.maximum((g - 1.0) * (U[..., 3] - 0.5 * rho * (vx * vx + vy * vy)), FLOOR)
    return rho, vx, vy, p, (U[..., 3] + p) / rho


def normal_flux(U, nx, ny, g):
    rho, vx, vy, p, H = primitives(U, g)
    vn = vx * nx + vy * ny
    return np.stack([rho * vn, rho * vx * vn + p * nx, rho * vy * vn + p * ny, rho * H * vn], -1)


def euler_flux(U, g):
    rho, vx, vy, p, H = primitives(U, g)
    F = np.stack([rho * vx, rho * vx * vx + p, rho * vx * vy, rho * vx * H], -1)
    G = np.stack([rho * vy, rho * vx * vy, rho * vy * vy + p, rho * vy * H], -1)
    return F, G


def roe(UL, UR, nx, ny, g, efix):
    rL, uL, vL, pL, HL = primitives(UL, g)
    rR, uR, vR, pR, HR = primitives(UR, g)
    FL, FR = normal_flux(UL, nx, ny, g), normal_flux(UR, nx, ny, g)
    sL, sR = np.sqrt(rL), np.sqrt(rR)
    d = sL + sR
    u = (sL * uL + sR * uR) / d
    v = (sL * vL + sR * vR) / d
    H = (sL * HL + sR * HR) / d
    q2 = u * u + v * v
    c = np.sqrt(np.maximum((g - 1.0) * (H - 0.5 * q2), FLOOR))
    vn = u * nx + v * ny
    l1, l2, l3 = _abs(vn + c), _abs(vn - c), _abs(vn)
    smax = np.maximum(l1, l2)
    eps = efix * c
    with np.errstate(divide="ignore", invalid="ignore"):
        l1, l2, l3 = (np.where(lam < eps, (lam * lam + eps * eps) / (2.0 * eps), lam) for lam in (l1, l2, l3))
    dU = UR - UL
    d0, d1, d2, d3 = dU[..., 0], dU[..., 1], dU[..., 2], dU[..., 3]
    G1 = (g - 1.0) * (0.5 * q2 * d0 - u * d1 - v * d2 + d3)
    G2 = -vn * d0 + d1 * nx + d2 * ny
    s1, s2 = 0.5 * (l1 + l2), 0.5 * (l1 - l2)
    C1 = (G1 / (c * c)) * (s1 - l3) + (G2 / c) * s2
    C2 = (G1 / c) * s2 + (s1 - l3) * G2
    diss = np.stack([l3 * d0 + C1, l3 * d1 + C1 * u + C2 * nx, l3 * d2 + C1 * v + C2 * ny, l3 * d3 + C1 * H + C2 * vn], -1)
    return 0.5 * (FL + FR) - 0.5 * diss, smax


def hllc(UL, UR, nx, ny, g, low_mach=0.0):
    rL, uL, vL, pL, HL = primitives(UL, g)
    rR, uR, vR, pR, HR = primitives(UR, g)
    vnL, vnR = uL * nx + vL * ny, uR * nx + vR * ny
    aL = np.sqrt(np.maximum(g * pL / rL, FLOOR))
    aR = np.sqrt(np.maximum(g * pR / rR, FLOOR))
    sL, sR = np.sqrt(rL), np.sqrt(rR)
    d = sL + sR
    u = (sL * uL + sR * uR) / d
    v = (sL * vL + sR * vR) / d
    H = (sL * HL + sR * HR) / d
    vt = u * nx + v * ny
    at = np.sqrt(np.maximum((g - 1.0) * (H - 0.5 * (u * u + v * v)), FLOOR))
    SL = np.minimum(vnL - aL, vt - at)
    SR = np.maximum(vnR + aR, vt + at)
    if low_mach > 0.0:
        mach = np.maximum(_abs(vnL) / aL, _abs(vnR) / aR)
        phi = np.minimum(1.0, mach / low_mach)
        bL, bR = np.minimum(vnL, vt), np.maximum(vnR, vt)
        SL = bL - phi * (bL - SL)
        SR = bR + phi * (SR - bR)
    mL, mR = rL * (SL - vnL), rR * (SR - vnR)
    dm = np.where(_abs(mR - mL) > FLOOR, mR - mL, FLOOR)
    SM = (rR * vnR * (SR - vnR) - rL * vnL * (SL - vnL) + pL - pR) / dm

    def guard(x):
        return np.where(_abs(x) > FLOOR, x, FLOOR)

    def star(U, r, u_, v_, p, vn, S):
        fac = (S - vn) / guard(S - SM)
        rs = r * fac
        us, vs = u_ + (SM - vn) * nx, v_ + (SM - vn) * ny
        Es = U[..., 3] / r + (SM - vn) * (SM + p / guard(r * (S - vn)))
        return np.stack([rs, rs * us, rs * vs, rs * Es], -1)

    FL, FR = normal_flux(UL, nx, ny, g), normal_flux(UR, nx, ny, g)
    FsL = FL + SL[..., None] * (star(UL, rL, uL, vL, pL, vnL, SL) - UL)
    FsR = FR + SR[..., None] * (star(UR, rR, uR, vR, pR, vnR, SR) - UR)
    F = np.where((SL >= 0.0)[..., None], FL, np.where((SR <= 0.0)[..., None], FR, np.where((SM >= 0.0)[..., None], FsL, FsR)))
    return F, np.maximum(_abs(SL), _abs(SR))


_B, _A, _KP, _KU = 0.125, 0.1875, 0.4, 0.2


def ausmup(UL, UR, nx, ny, g):
    rL, uL, vL, pL, _ = primitives(UL, g)
    rR, uR, vR, pR, _ = primitives(UR, g)
    vnL, vnR = uL * nx + vL * ny, uR * nx + vR * ny
    aL, aR = np.sqrt(g * pL / rL), np.sqrt(g * pR / rR)
    ah, rh = 0.5 * (aL + aR), 0.5 * (rL + rR)
    mL, mR = vnL / ah, vnR / ah
    mb2 = 0.5 * (mL * mL + mR * mR)

    def m2(m):
        return 0.25 * (m + 1.0) ** 2, -0.25 * (m - 1.0) ** 2

    pL2, mL2 = m2(mL)
    pR2, mR2 = m2(mR)
    m4p = np.where(_abs(mL) >= 1.0, 0.5 * (mL + _abs(mL)), pL2 * (1.0 - 16.0 * _B * mL2))
    m4m = np.where(_abs(mR) >= 1.0, 0.5 * (mR - _abs(mR)), mR2 * (1.0 + 16.0 * _B * pR2))
    uh = ah * (m4p + m4m) + _KP * np.maximum(1.0 - mb2, 0.0) * (pL - pR) / (rh * ah)
    p5p = np.where(_abs(mL) >= 1.0, 0.5 * (1.0 + _sign(mL)), pL2 * ((2.0 - mL) - 16.0 * _A * mL * mL2))
    p5m = np.where(_abs(mR) >= 1.0, 0.5 * (1.0 - _sign(mR)), mR2 * ((-2.0 - mR) + 16.0 * _A * mR * pR2))
    ph = p5p * pL + p5m * pR + _KU * p5p * p5m * rh * ah * (vnL - vnR)
    PsiL = np.stack([rL, rL * uL, rL * vL, UL[..., 3] + pL], -1)
    PsiR = np.stack([rR, rR * uR, rR * vR, UR[..., 3] + pR], -1)
    F = 0.5 * uh[..., None] * (PsiL + PsiR) - 0.5 * _abs(uh)[..., None] * (PsiR - PsiL)
    z = np.zeros_like(ph)
    F = F + ph[..., None] * np.stack([z, nx + z, ny + z, z], -1)
    return F, np.maximum(_abs(vnL) + aL, _abs(vnR) + aR)


def wall(U, nx, ny, g):
    rho = np.maximum(U[..., 0], FLOOR)
    vx, vy = U[..., 1] / rho, U[..., 2] / rho
    vn = vx * nx + vy * ny
    vt2 = (vx - vn * nx) ** 2 + (vy - vn * ny) ** 2
    pb = np.maximum((g - 1.0) * (U[..., 3] - 0.5 * rho * vt2), FLOOR)
    z = np.zeros_like(pb)
    return np.stack([z, pb * nx, pb * ny, z], -1), np.sqrt(g * pb / rho)


def inflow(U, nx, ny, g, Tt, pt, Rgas, alpha):
    at2 = g * Rgas * Tt
    at = np.sqrt(at2)
    rho_t = g * pt / at2
    rho, vx, vy, p, _ = primitives(U, g)
    a = np.sqrt(g * p / rho)
    Jp = vx * nx + vy * ny + 2.0 * a / (g - 1.0)
    beta = (Jp / at) ** 2
    nd = nx * np.cos(alpha) + ny * np.sin(alpha)
    qa = 0.5 * (g - 1.0) * beta - nd * nd
    qb = -4.0 * nd / (g - 1.0)
    qc = beta - (2.0 / (g - 1.0)) ** 2
    qa = np.where(_abs(qa) < 1e-12, np.where(qa >= 0, 1e-12, -1e-12), qa)
    sq = np.sqrt(np.maximum(qb * qb - 4.0 * qa * qc, 0.0))
    r1, r2 = (-qb + sq) / (2.0 * qa), (-qb - sq) / (2.0 * qa)
    M = np.minimum(np.where(r1 >= 0.0, r1, 1e30), np.where(r2 >= 0.0, r2, 1e30))
    M = np.clip(np.where(M > 0.5e30, 0.0, M), 0.0, 1.0)
    ab = np.sqrt(at2 / (1.0 + 0.5 * (g - 1.0) * M * M))
    vxb, vyb = M * ab * np.cos(alpha), M * ab * np.sin(alpha)
    rhob = rho_t * (1.0 + 0.5 * (g - 1.0) * M * M) ** (-1.0 / (g - 1.0))
    pb = rhob * ab * ab / g
    Hb = at2 / (g - 1.0)
    vnb = vxb * nx + vyb * ny
    F = np.stack([rhob * vnb, rhob * vxb * vnb + pb * nx, rhob * vyb * vnb + pb * ny, rhob * Hb * vnb], -1)
    return F, _abs(vnb) + ab


def outflow(U, nx, ny, g, p_back, rho_t=0.0, p_t=1.0, band=0.05):
    rho, vx, vy, p, _ = primitives(U, g)
    a = np.sqrt(g * p / rho)
    vn = vx * nx + vy * ny
    pb = p_back * np.ones_like(p)
    rhob = rho * (pb / p) ** (1.0 / g)
    ab = np.sqrt(g * pb / rhob)
    vnb = vn + 2.0 / (g - 1.0) * (a - ab)
    vxb = (vx - vn * nx) + vnb * nx
    vyb = (vy - vn * ny) + vnb * ny
    Eb = pb / ((g - 1.0) * rhob) + 0.5 * (vxb * vxb + vyb * vyb)
    Us = np.stack([rhob, rhob * vxb, rhob * vyb, rhob * Eb], -1)
    if rho_t > 0.0:
        rf = rho_t * (pb / p_t) ** (1.0 / g)
        af = np.sqrt(g * pb / rf)
        vnf = vn + 2.0 / (g - 1.0) * (a - af)
        vxf, vyf = vnf * nx, vnf * ny
        Ef = pb / ((g - 1.0) * rf) + 0.5 * (vxf * vxf + vyf * vyf)
        Uf = np.stack([rf, rf * vxf, rf * vyf, rf * Ef], -1)
        t = np.clip((vn / a) / max(band, 1e-12), 0.0, 1.0)[..., None]
        Us = t * Us + (1.0 - t) * Uf
    Ub = np.where((vn / a >= 1.0)[..., None], U, Us)
    F = normal_flux(Ub, nx, ny, g)
    ro, uo, vo, po, _ = primitives(Ub, g)
    return F, _abs(uo * nx + vo * ny) + np.sqrt(g * po / ro)


def interface(flow, UL, UR, nx, ny):
    name = flow.flux
    if name == "roe":
        return roe(UL, UR, nx, ny, flow.gamma, flow.entropy_fix)
    if name == "hllc":
        return hllc(UL, UR, nx, ny, flow.gamma, flow.hllc_low_mach)
    if name == "ausmup":
        return ausmup(UL, UR, nx, ny, flow.gamma)
    raise ValueError(f"unknown flux {name!r}")


# --------------------------------------------------------------- residual
def _face_tables(ops):
    """``(E, nface, nbf, nqf)`` basis of each element on each of its own faces."""
    ed = ops.topology.edges
    nface = ed.face_edge.shape[1]
    return ops.ref.phi_face[ed.face_side, np.arange(nface)[None, :]]


def edge_fluxes(U, ops, flow):
    ed = ops.topology.edges
    pf = ops.ref.phi_face
    ni = ed.n_interior
    nrm = np.asarray(ops.edge_normal)
    UL = np.einsum("kiq,kis->kqs", pf[0][ed.iedge_face[:, 0]], U[ed.iedge_elem[:, 0]])
    UR = np.einsum("kiq,kis->kqs", pf[1][ed.iedge_face[:, 1]], U[ed.iedge_elem[:, 1]])
    F_i, s_i = interface(flow, UL, UR, nrm[:ni, :, 0], nrm[:ni, :, 1])
    Ub = np.einsum("kiq,kis->kqs", pf[0][ed.bedge_face], U[ed.bedge_elem])
    nb = nrm[ni:]
    Fb = np.zeros(Ub.shape, dtype=np.result_type(Ub, nb))
    sb = np.zeros(Ub.shape[:2], dtype=Fb.dtype)
    g = flow.gamma
    for tag, sl in ed.tag_slices.items():
        u, nx, ny = Ub[sl], nb[sl, :, 0], nb[sl, :, 1]
        if tag == INFLOW:
            f, s = inflow(u, nx, ny, g, flow.total_temperature, flow.total_pressure, flow.Rgas, flow.inflow_angle)
        elif tag == OUTFLOW:
            rho_t = flow.stagnation_density if flow.backflow else 0.0
            f, s = outflow(u, nx, ny, g, flow.back_pressure, rho_t, flow.total_pressure)
        else:
            f, s = wall(u, nx, ny, g)
        Fb[sl], sb[sl] = f, s
    return np.concatenate([F_i, Fb]), np.concatenate([s_i, sb])


def residual(U, ops, flow):
    """``(R, wave)`` with ``M dU/dt = -R``.  Complex U (a complex step) is kept complex."""
    U = np.asarray(U)
    if not np.iscomplexobj(U):
        U = U.astype(float)
    F, speed = edge_fluxes(U, ops, flow)
    uq = np.einsum("iq,eis->eqs", ops.ref.phi_vol, U)
    Fx, Fy = euler_flux(uq, flow.gamma)
    R = -(np.einsum("eiq,eqs->eis", ops.grad_x, Fx) + np.einsum("eiq,eqs->eis", ops.grad_y, Fy))
    fw = F * (np.asarray(ops.edge_jac) * ops.ref.w_face[None, :])[..., None]
    fb = _face_tables(ops)
    for f in range(fb.shape[1]):
        R = R + np.einsum("eiq,eqs->eis", fb[:, f], fw[ops.face_edge[:, f]]) * ops.face_sign[:, f][:, None, None]
    wave = (speed.max(axis=1) * ops.edge_length)[ops.face_edge].sum(axis=1)
    return R, wave


def inverse_mass(R, ops):
    return np.einsum("eij,ejs->eis", ops.inv_mass, R)


def rate(U, ops, flow):
    R, wave = residual(U, ops, flow)
    return -inverse_mass(R, ops), wave


# ---------------------------------------------------------------- limiter
def positivity(U, ops, flow, fraction=1e-8, steps=12):
    """Limit ``U``.  Returns ``(U_new, limited_mask, repaired_mask)``."""
    U = np.array(U, dtype=float, copy=True)
    ne = U.shape[0]
    none = np.zeros(ne, bool)
    if ops.ref.order == 0:
        return U, none, none
    g = flow.gamma
    rho_floor = fraction * flow.stagnation_density
    p_floor = fraction * flow.total_pressure
    mw = np.asarray(ops.mean_weights)
    ub = np.einsum("ei,eis->es", mw, U)
    rho_new = np.maximum(ub[:, 0], rho_floor)
    e_min = p_floor / (g - 1.0) + 0.5 * (ub[:, 1] ** 2 + ub[:, 2] ** 2) / rho_new
    rhoE_new = np.maximum(ub[:, 3], e_min)
    repaired = (rho_new != ub[:, 0]) | (rhoE_new != ub[:, 3])
    if repaired.any():
        U[repaired, :, 0] += (rho_new - ub[:, 0])[repaired, None]
        U[repaired, :, 3] += (rhoE_new - ub[:, 3])[repaired, None]
        ub = np.einsum("ei,eis->es", mw, U)
    probes = np.concatenate(
        [np.einsum("iq,eis->eqs", ops.ref.phi_vol, U), np.einsum("efiq,eis->efqs", _face_tables(ops), U).reshape(ne, -1, 4)],
        axis=1,
    )
    pbar = (g - 1.0) * (ub[:, 3] - 0.5 * (ub[:, 1] ** 2 + ub[:, 2] ** 2) / ub[:, 0])
    eps_r = np.maximum(fraction * ub[:, 0], 0.5 * rho_floor)
    eps_p = np.maximum(fraction * pbar, 0.5 * p_floor)

    def pmin(theta, ubar, dev):
        V = ubar[:, None, :] + theta[:, None, None] * dev
        r = np.maximum(V[..., 0], 1e-300)
        return ((g - 1.0) * (V[..., 3] - 0.5 * (V[..., 1] ** 2 + V[..., 2] ** 2) / r)).min(axis=1)

    ones = np.ones(ne)
    bad = (probes[..., 0].min(axis=1) < eps_r) | (pmin(ones, ub, probes - ub[:, None, :]) < eps_p)
    idx = np.flatnonzero(bad)
    if idx.size:
        u, pr = ub[idx], probes[idx]
        dev = pr - u[:, None, :]
        rmin = pr[..., 0].min(axis=1)
        gap = u[:, 0] - rmin
        th_r = np.where(rmin < eps_r[idx], np.clip((u[:, 0] - eps_r[idx]) / np.where(gap > 0.0, gap, 1.0), 0.0, 1.0), 1.0)
        lo, hi = np.zeros_like(th_r), th_r.copy()
        ok_hi = pmin(hi, u, dev) >= eps_p[idx]
        for _ in range(steps):
            mid = 0.5 * (lo + hi)
            good = pmin(mid, u, dev) >= eps_p[idx]
            lo = np.where(good, mid, lo)
            hi = np.where(good, hi, mid)
        th = np.where(ok_hi, th_r, lo)
        U[idx] = u[:, None, :] + th[:, None, None] * (U[idx] - u[:, None, :])
    return U, bad, repaired


# ------------------------------------------------------------- slope limiter
def superbee_pair(a, b):
    """Roe's Superbee in its two-argument form, maxmod(minmod(2a, b), minmod(a, 2b))
    (src/spatial/limiter.py:246-270)."""
    def minmod(x, y):
        return np.where(x * y <= 0.0, 0.0, np.where(_abs(x) < _abs(y), x, y))

    def maxmod(x, y):
        return np.where(x * y <= 0.0, 0.0, np.where(_abs(x) > _abs(y), x, y))

    return maxmod(minmod(2.0 * a, b), minmod(a, 2.0 * b))


def superbee(U, ops, tvb_constant=50.0, tol=1e-12):
    """The Superbee TVB slope limiter (src/spatial/limiter.py:273-405): per element and face the own
    increment d = (face-averaged own trace) - ubar against the jump a = ubar(neighbour) - ubar; a
    face is quiet on a boundary, for |d| <= tol, or below the TVB threshold
    tvb * (A_e / A_total) * max_e |ubar_s|; theta_e = min over faces and components of
    clip(superbee(a, d) / d, 0, 1); U <- ubar + theta (U - ubar).  Returns (U_new, changed mask)."""
    U = np.asarray(U, float)
    if ops.ref.order == 0:
        return U.copy(), np.zeros(U.shape[0], bool)
    ubar = np.einsum("ei,eis->es", np.asarray(ops.mean_weights), U)
    ed = ops.topology.edges
    E = U.shape[0]
    nface = ed.face_edge.shape[1]
    nb = np.repeat(np.arange(E)[:, None], nface, axis=1)
    nb[ed.iedge_elem[:, 0], ed.iedge_face[:, 0]] = ed.iedge_elem[:, 1]
    nb[ed.iedge_elem[:, 1], ed.iedge_face[:, 1]] = ed.iedge_elem[:, 0]
    interior = (nb != np.arange(E)[:, None])[..., None]
    jump = ubar[nb] - ubar[:, None, :]
    w = np.asarray(ops.ref.w_face)
    dev = np.einsum("efiq,q,eis->efs", _face_tables(ops), w, U) / w.sum() - ubar[:, None, :]
    allowed = superbee_pair(jump, dev)
    safe = np.where(np.abs(dev) > tol, dev, 1.0)
    theta_face = np.clip(allowed / safe, 0.0, 1.0)
    area = np.asarray(ops.elem_area)
    share = (area / area.sum())[:, None, None]
    scale = np.abs(ubar).max(axis=0)[None, None, :]
    quiet = (np.abs(dev) <= tol) | ~interior | (np.abs(dev) <= tvb_constant * share * scale)
    theta = np.where(quiet, 1.0, theta_face).min(axis=(1, 2))
    out = ubar[:, None, :] + theta[:, None, None] * (U - ubar[:, None, :])
    return out, np.abs(out - U).max(axis=(1, 2)) > 0.0


# ------------------------------------------------------------------ march
def step_coefficient(order, cfl, scheme):
    table = {"ssprk3": (1.437, 2.337, 2.240), "euler": (1.169, 1.337, 0.775)}[scheme]
    if cfl is None:
        if order < len(table):
            lim = table[order]
        else:
            lim = 0.70 if scheme == "euler" else 1.32 * (2 * order + 1) / (order + 1)
        cfl = 0.7 * lim
    return cfl / (2 * order + 1)


def time_step(wave, ops, order, cfl, scheme, pscale=1.0):
    return pscale * (step_coefficient(order, cfl, scheme) * 2.0 * np.asarray(ops.elem_area) / np.maximum(wave, FLOOR))


def norm(A, flow):
    a_t = flow.stagnation_sound_speed
    w = np.array([1.0, 1.0 / a_t, 1.0 / a_t, 1.0 / a_t**2])
    with np.errstate(over="ignore", invalid="ignore"):
        B = np.asarray(A) * w
        return float(np.sqrt(np.mean(B * B)))


class Stepper:
    """Forward-Euler / SSP-RK3 march with per-stage limiter records."""

    def __init__(self, ops, flow, opts):
        self.ops, self.flow, self.opts = ops, flow, opts
        p = ops.ref.order
        self.scheme = opts.scheme or ("euler" if p < 1 else "ssprk3")
        pc = getattr(opts, "positivity_cfl", 0.0)
        self.pscale = float(pc) if (pc > 0.0 and opts.limiter != "none" and p > 0) else 1.0
        self.stage_masks = []

    def limit(self, U):
        if self.opts.limiter == "none" or self.ops.ref.order == 0:
            self.stage_masks.append(np.zeros(U.shape[0], bool))
            return U
        if self.opts.limiter == "superbee":
            U, _ = superbee(U, self.ops, getattr(self.opts, "tvb_constant", 50.0))
        elif self.opts.limiter != "positivity":
            raise ValueError(f"unknown limiter {self.opts.limiter!r}")
        out, bad, _ = positivity(U, self.ops, self.flow)
        self.stage_masks.append(bad)
        return out

    def step(self, U):
        F0, wave = rate(U, self.ops, self.flow)
        dt = time_step(wave, self.ops, self.ops.ref.order, self.opts.cfl, self.scheme, self.pscale)[:, None, None]
        res = norm(F0, self.flow)
        if self.scheme == "euler":
            return self.limit(U + dt * F0), res
        U1 = self.limit(U + dt * F0)
        F1, _ = rate(U1, self.ops, self.flow)
        U2 = self.limit(0.75 * U + 0.25 * (U1 + dt * F1))
        F2, _ = rate(U2, self.ops, self.flow)
        return self.limit((1.0 / 3.0) * U + (2.0 / 3.0) * (U2 + dt * F2)), res

    def run(self, U, n):
        res = float("nan")
        with np.errstate(over="ignore", invalid="ignore"):
            for _ in range(n):
                U, res = self.step(U)
        return U, res


# ---------------------------------------------------------------- adjoint
# The reference takes its adjoint's derivatives from JAX (src/sensitivity.py:
# 289-460).  Here they come from complex steps through the restatement above:
# f(x + i h) = f(x) + i h f'(x) + O(h^2) for an analytic f, so Im f / h is the
# derivative to round-off with h = 1e-30 (no cancellation, unlike a finite
# difference).  Branches compare real parts, as the reference's do.
H_CS = 1e-30


class _Ops:
    pass


def operators_at(ops, X):
    """The operator fields ``residual`` reads, rebuilt at node coordinates X (real or complex).

    Restates src/spatial/operators.py:238-303 for straight-sided (Q = 1)
    elements: metrics from the vertex map, w det (dphi/dx, dphi/dy), the mass
    matrix and its inverse, the owner's edge tangent, |dX/dsigma|, the normal
    (t_y, -t_x)/|t| and the edge length.
    """
    rd, topo = ops.ref, ops.topology
    X = np.asarray(X)
    Xe = X[topo.elem_nodes]
    x_xi, x_eta = Xe[:, :, 0] @ rd.dgeom_dxi_vol, Xe[:, :, 0] @ rd.dgeom_deta_vol
    y_xi, y_eta = Xe[:, :, 1] @ rd.dgeom_dxi_vol, Xe[:, :, 1] @ rd.dgeom_deta_vol
    det = x_xi * y_eta - x_eta * y_xi
    inv = 1.0 / det
    xi_x, xi_y, eta_x, eta_y = y_eta * inv, -x_eta * inv, -y_xi * inv, x_xi * inv
    wdet = rd.w_vol[None, :] * det
    out = _Ops()
    out.ref, out.topology = rd, topo
    out.grad_x = wdet[:, None, :] * (rd.dphi_dxi_vol[None] * xi_x[:, None, :] + rd.dphi_deta_vol[None] * eta_x[:, None, :])
    out.grad_y = wdet[:, None, :] * (rd.dphi_dxi_vol[None] * xi_y[:, None, :] + rd.dphi_deta_vol[None] * eta_y[:, None, :])
    out.inv_mass = np.linalg.inv(np.einsum("iq,jq,eq->eij", rd.phi_vol, rd.phi_vol, wdet))
    out.elem_area = wdet.sum(axis=1)
    ed = topo.edges
    owner_e = np.concatenate([ed.iedge_elem[:, 0], ed.bedge_elem])
    owner_f = np.concatenate([ed.iedge_face[:, 0], ed.bedge_face])
    t = np.einsum("enq,end->eqd", np.asarray(rd.dgeom_dsigma_face)[owner_f], Xe[owner_e])
    jac = np.sqrt(t[..., 0] ** 2 + t[..., 1] ** 2)
    out.edge_jac = jac
    out.edge_normal = np.stack([t[..., 1], -t[..., 0]], -1) / jac[..., None]
    out.edge_length = (jac * rd.w_face[None, :]).sum(axis=1)
    out.face_edge = ops.face_edge
    out.face_sign = ops.face_sign
    out.n_elem = ops.n_elem
    return out


def state_jacobian(U, ops, flow):
    """dR/dU as a dense (n, n) matrix over the flattened (E, NP, 4) state, by complex steps."""
    U = np.asarray(U, float)
    n = U.size
    J = np.empty((n, n))
    for k in range(n):
        Uc = U.astype(complex).ravel()
        Uc[k] += 1j * H_CS
        J[:, k] = residual(Uc.reshape(U.shape), ops, flow)[0].imag.ravel() / H_CS
    return J


def state_vjp(U, lam, ops, flow, J=None):
    """(dR/dU)^T lam in the (E, NP, 4) layout."""
    J = state_jacobian(U, ops, flow) if J is None else J
    return (J.T @ np.asarray(lam, float).ravel()).reshape(np.shape(U))


def coord_vjp(U, lam, ops, flow):
    """(dR/dX)^T lam as an (N_nodes, 2) array, by one complex step per node coordinate."""
    X = np.asarray(ops.node_coords, float)
    lam = np.asarray(lam, float)
    g = np.zeros_like(X)
    Uc = np.asarray(U, float).astype(complex)
    for a in range(X.shape[0]):
        for d in range(2):
            Xc = X.astype(complex)
            Xc[a, d] += 1j * H_CS
            R = residual(Uc, operators_at(ops, Xc), flow)[0]
            g[a, d] = float(np.sum(lam * R.imag)) / H_CS
    return g


def back_pressure_vjp(U, lam, ops, flow):
    """(dR/dp_back)^T lam by a complex step on the back pressure."""
    import dataclasses

    fc = dataclasses.replace(flow, back_pressure_ratio=flow.back_pressure_ratio + 1j * H_CS / flow.total_pressure)
    R = residual(np.asarray(U, float).astype(complex), ops, fc)[0]
    return float(np.sum(np.asarray(lam, float) * R.imag)) / H_CS


def adjoint_march(U, seed, ops, flow, cfl, n_steps, J=None):
    """n_steps of the adjoint pseudo-time march from lam = 0 (src/sensitivity.py:318-358):
    dlam/dtau = -M^-1 ((dR/dU)^T lam - seed), classical RK4, dt frozen from the
    converged state with the SSP-RK3 coefficient at cfl."""
    U = np.asarray(U, float)
    J = state_jacobian(U, ops, flow) if J is None else J
    seed = np.asarray(seed, float)
    _, wave = residual(U, ops, flow)
    dt = time_step(wave, ops, ops.ref.order, cfl, "ssprk3")[:, None, None]

    def rate(lam):
        return -inverse_mass(state_vjp(U, lam, ops, flow, J) - seed, ops)

    lam = np.zeros_like(seed)
    for _ in range(n_steps):
        f0 = rate(lam)
        f1 = rate(lam + 0.5 * dt * f0)
        f2 = rate(lam + 0.5 * dt * f1)
        f3 = rate(lam + dt * f2)
        lam = lam + dt / 6.0 * (f0 + 2.0 * f1 + 2.0 * f2 + f3)
    return lam
