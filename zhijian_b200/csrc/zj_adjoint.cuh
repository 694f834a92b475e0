// zj_adjoint.cuh -- local vector-Jacobian products of the physics-mode
// residual's pointwise functions, FP64:
//   euler_flux_vjp   (dF/dU)^T Fbar + (dG/dU)^T Gbar, closed form
//   viscous_vjp      transposed viscous flux w.r.t. the state and the
//                    conservative gradients, closed form (reverse sweep of
//                    phys::viscous_flux)
//   riemann_vjp      transposed common flux w.r.t. both states: the Roe
//                    solver by its reverse sweep (roe_vjp), Rusanov and HLLC
//                    column by column from tangent evaluations on dual
//                    numbers (zj_dual.cuh)
//   ghost_vjp        transposed ghost state w.r.t. the interior trace, from
//                    dual-number tangents
// The dual-number columns transpose exactly the arithmetic the forward
// kernels run, branches and floors included; the reverse sweeps follow the
// same branch conventions (a floor passes the derivative when it keeps the
// value, |x| has slope +1 at 0).
#pragma once

#include <cuda_runtime.h>

#include "zj_device.cuh"
#include "zj_dual.cuh"
#include "zj_physics.cuh"

namespace zj {
namespace adj {

using namespace dev;

// ub += (dF/du)^T Fb + (dG/du)^T Gb for the Euler fluxes of euler_flux.
__device__ __forceinline__ void euler_flux_vjp(const double* s, double g, const double* Fb,
                                               const double* Gb, double* ub) {
    const double ir = rcp_any(s[0]);
    const double u = s[1] * ir, v = s[2] * ir, E = s[3];
    const double c = g - 1.0;
    const double p = c * s[0] * (E * ir - 0.5 * (u * u + v * v));
    double mb = Fb[0], nb = Gb[0], Eb = 0.0, pb = 0.0, ubar = 0.0, vbar = 0.0;
    // F1 = m u + p, F2 = m v, F3 = (E + p) u
    mb += Fb[1] * u; ubar += Fb[1] * s[1]; pb += Fb[1];
    mb += Fb[2] * v; vbar += Fb[2] * s[1];
    Eb += Fb[3] * u; pb += Fb[3] * u; ubar += Fb[3] * (E + p);
    // G1 = n u, G2 = n v + p, G3 = (E + p) v
    nb += Gb[1] * u; ubar += Gb[1] * s[2];
    nb += Gb[2] * v; vbar += Gb[2] * s[2]; pb += Gb[2];
    Eb += Gb[3] * v; pb += Gb[3] * v; vbar += Gb[3] * (E + p);
    // p = c (E - (m^2 + n^2) / (2 rho))
    double rb = pb * c * 0.5 * (u * u + v * v);
    mb -= pb * c * u;
    nb -= pb * c * v;
    Eb += pb * c;
    // u = m / rho, v = n / rho
    mb += ubar * ir; rb -= ubar * u * ir;
    nb += vbar * ir; rb -= vbar * v * ir;
    ub[0] += rb; ub[1] += mb; ub[2] += nb; ub[3] += Eb;
}

// Reverse sweep of phys::viscous_flux: given Fvb, Gvb (components 1..3; the
// mass components of the viscous flux are zero), adds the adjoints of the
// state s and of the gradients dx = dU/dx, dy = dU/dy into sb, dxb, dyb.
// Returns Fvb . Fv + Gvb . Gv: the viscous flux is proportional to 1/Re, so
// minus this over Re is the flux adjoint's Reynolds-number derivative.
__device__ __forceinline__ double viscous_vjp(const double* s, const double* dx, const double* dy,
                                            double g, double Re, double Pr, const double* Fvb,
                                            const double* Gvb, double* sb, double* dxb,
                                            double* dyb) {
    // forward recomputation (the operations of phys::viscous_flux)
    const double ir = rcp_any(s[0]);
    const double u = s[1] * ir, v = s[2] * ir;
    const double dudx = (dx[1] - u * dx[0]) * ir, dudy = (dy[1] - u * dy[0]) * ir;
    const double dvdx = (dx[2] - v * dx[0]) * ir, dvdy = (dy[2] - v * dy[0]) * ir;
    const double c = g - 1.0;
    const double q2 = u * u + v * v;
    const double p = c * s[0] * (s[3] * ir - 0.5 * q2);
    const double Tm = p * ir;
    const double dpdx = c * (dx[3] - 0.5 * dx[0] * q2 - s[0] * (u * dudx + v * dvdx));
    const double dpdy = c * (dy[3] - 0.5 * dy[0] * q2 - s[0] * (u * dudy + v * dvdy));
    const double dTdx = (dpdx - Tm * dx[0]) * ir, dTdy = (dpdy - Tm * dy[0]) * ir;
    const double mu = zj_pow07(Tm) / Re;
    const double kc = g / (c * Pr);
    const double k = mu * kc;
    const double div = dudx + dvdy, lam = (-2.0 / 3.0) * mu;
    const double txx = 2.0 * mu * dudx + lam * div, tyy = 2.0 * mu * dvdy + lam * div;
    const double txy = mu * (dudy + dvdx);
    // reverse
    const double txxb = Fvb[1] + Fvb[3] * u;
    const double txyb = Fvb[2] + Fvb[3] * v + Gvb[1] + Gvb[3] * u;
    const double tyyb = Gvb[2] + Gvb[3] * v;
    double ubar = Fvb[3] * txx + Gvb[3] * txy;
    double vbar = Fvb[3] * txy + Gvb[3] * tyy;
    const double kb = Fvb[3] * dTdx + Gvb[3] * dTdy;
    const double dTdxb = Fvb[3] * k, dTdyb = Gvb[3] * k;
    double mub = 0.0, lamb = 0.0, divb = 0.0;
    double dudxb = 0.0, dudyb = 0.0, dvdxb = 0.0, dvdyb = 0.0;
    mub += txxb * 2.0 * dudx; dudxb += txxb * 2.0 * mu; lamb += txxb * div; divb += txxb * lam;
    mub += tyyb * 2.0 * dvdy; dvdyb += tyyb * 2.0 * mu; lamb += tyyb * div; divb += tyyb * lam;
    mub += txyb * (dudy + dvdx); dudyb += txyb * mu; dvdxb += txyb * mu;
    mub += lamb * (-2.0 / 3.0);
    dudxb += divb; dvdyb += divb;
    mub += kb * kc;
    double Tmb = (Tm != 0.0) ? mub * 0.7 * mu / Tm : 0.0;
    double irb = 0.0;
    double dpdxb = dTdxb * ir, dpdyb = dTdyb * ir;
    Tmb -= dTdxb * dx[0] * ir + dTdyb * dy[0] * ir;
    dxb[0] -= dTdxb * Tm * ir;
    dyb[0] -= dTdyb * Tm * ir;
    irb += dTdxb * (dpdx - Tm * dx[0]) + dTdyb * (dpdy - Tm * dy[0]);
    double q2b = 0.0, s0b = 0.0;
    // dpdx = c (dx3 - dx0 q2 / 2 - s0 (u dudx + v dvdx))
    dxb[3] += c * dpdxb;
    dxb[0] -= 0.5 * c * q2 * dpdxb;
    q2b -= 0.5 * c * dx[0] * dpdxb;
    s0b -= c * (u * dudx + v * dvdx) * dpdxb;
    ubar -= c * s[0] * dudx * dpdxb; dudxb -= c * s[0] * u * dpdxb;
    vbar -= c * s[0] * dvdx * dpdxb; dvdxb -= c * s[0] * v * dpdxb;
    dyb[3] += c * dpdyb;
    dyb[0] -= 0.5 * c * q2 * dpdyb;
    q2b -= 0.5 * c * dy[0] * dpdyb;
    s0b -= c * (u * dudy + v * dvdy) * dpdyb;
    ubar -= c * s[0] * dudy * dpdyb; dudyb -= c * s[0] * u * dpdyb;
    vbar -= c * s[0] * dvdy * dpdyb; dvdyb -= c * s[0] * v * dpdyb;
    // Tm = p ir
    const double pb = Tmb * ir;
    irb += Tmb * p;
    // p = c s0 (s3 ir - q2/2)
    s0b += pb * c * (s[3] * ir - 0.5 * q2);
    sb[3] += pb * c * s[0] * ir;
    irb += pb * c * s[0] * s[3];
    q2b -= 0.5 * pb * c * s[0];
    ubar += 2.0 * u * q2b;
    vbar += 2.0 * v * q2b;
    // velocity gradients
    dxb[1] += dudxb * ir; ubar -= dudxb * dx[0] * ir; dxb[0] -= dudxb * u * ir; irb += dudxb * (dx[1] - u * dx[0]);
    dyb[1] += dudyb * ir; ubar -= dudyb * dy[0] * ir; dyb[0] -= dudyb * u * ir; irb += dudyb * (dy[1] - u * dy[0]);
    dxb[2] += dvdxb * ir; vbar -= dvdxb * dx[0] * ir; dxb[0] -= dvdxb * v * ir; irb += dvdxb * (dx[2] - v * dx[0]);
    dyb[2] += dvdyb * ir; vbar -= dvdyb * dy[0] * ir; dyb[0] -= dvdyb * v * ir; irb += dvdyb * (dy[2] - v * dy[0]);
    // u = s1 ir, v = s2 ir, ir = 1/s0
    sb[1] += ubar * ir; irb += ubar * s[1];
    sb[2] += vbar * ir; irb += vbar * s[2];
    s0b -= irb * ir * ir;
    sb[0] += s0b;
    return Fvb[1] * txx + Fvb[2] * txy + Fvb[3] * (u * txx + v * txy + k * dTdx) +
           Gvb[1] * txy + Gvb[2] * tyy + Gvb[3] * (u * txy + v * tyy + k * dTdy);
}

// Reverse of phys::pressure: Ub += pb dp/dU, p = (g-1)(U3 - (U1^2+U2^2)/(2 U0)).
__device__ __forceinline__ void pressure_vjp(const double* U, double g, double pb, double* Ub) {
    const double ir = rcp_any(U[0]);
    const double u = U[1] * ir, v = U[2] * ir, c = g - 1.0;
    Ub[0] += pb * c * 0.5 * (u * u + v * v);
    Ub[1] -= pb * c * u;
    Ub[2] -= pb * c * v;
    Ub[3] += pb * c;
}

// Reverse of phys::flux_normal(U, praw, n): adds into Ub and returns praw's
// adjoint.  Floors pass the derivative when the value is kept (the dual
// numbers' max convention).
__device__ __forceinline__ double flux_normal_vjp(const double* U, double praw, double nx, double ny,
                                                  const double* Fb, double* Ub) {
    const double rho = fmax(U[0], 1e-10);
    const double ir = rcp_any(rho);
    const double u = U[1] * ir, v = U[2] * ir;
    const double p = fmax(praw, 1e-10);
    const double H = U[3] + praw;
    const double vn = u * nx + v * ny;
    double rhob = Fb[0] * vn + Fb[1] * u * vn + Fb[2] * v * vn;
    double vnb = Fb[0] * rho + Fb[1] * rho * u + Fb[2] * rho * v + Fb[3] * H;
    double ub = Fb[1] * rho * vn + vnb * nx;
    double vb = Fb[2] * rho * vn + vnb * ny;
    const double pb = Fb[1] * nx + Fb[2] * ny;
    const double Hb = Fb[3] * vn;
    Ub[3] += Hb;
    double prawb = Hb + ((praw >= 1e-10) ? pb : 0.0);
    Ub[1] += ub * ir;
    Ub[2] += vb * ir;
    const double irb = ub * U[1] + vb * U[2];
    rhob -= irb * ir * ir;
    if (U[0] >= 1e-10) Ub[0] += rhob;
    (void)p;
    return prawb;
}

// Reverse sweep of phys::riemann_roe (Harten's entropy fix included): adds
// (dFc/dUL)^T Fb into ULb and (dFc/dUR)^T Fb into URb.
__device__ __forceinline__ void roe_vjp(const double* UL, const double* UR, double nx, double ny,
                                        double g, const double* Fb, double* ULb, double* URb) {
    // forward recomputation
    const double rhoL = fmax(UL[0], 1e-10), rhoR = fmax(UR[0], 1e-10);
    const double irL = rcp_any(rhoL), irR = rcp_any(rhoR);
    const double uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    const double pL = phys::pressure(UL, g), pR = phys::pressure(UR, g);
    const double HL = (UL[3] + pL) * irL, HR = (UR[3] + pR) * irR;
    const double sL = zj_sqrt(rhoL), sR = zj_sqrt(rhoR);
    const double ssum = sL + sR;
    const double iden = rcp_any(fmax(ssum, 1e-10));
    const double rhoRoe = sL * sR;
    const double uRoe = (sL * uL + sR * uR) * iden, vRoe = (sL * vL + sR * vR) * iden;
    const double HRoe = (sL * HL + sR * HR) * iden;
    const double vnRoe = uRoe * nx + vRoe * ny, qsq = uRoe * uRoe + vRoe * vRoe;
    const double carg = (g - 1.0) * (HRoe - 0.5 * qsq);
    const double c = zj_sqrt(fmax(carg, 1e-10));
    const double l1o = fabs(vnRoe - c), l2 = fabs(vnRoe), l4o = fabs(vnRoe + c);
    const double eps = 0.1 * c;
    const bool fix1 = l1o < eps, fix4 = l4o < eps;
    const double l1 = fix1 ? (l1o * l1o + eps * eps) * rcp_any(2.0 * eps) : l1o;
    const double l4 = fix4 ? (l4o * l4o + eps * eps) * rcp_any(2.0 * eps) : l4o;
    const double drho = rhoR - rhoL, du = uR - uL, dv = vR - vL, dp = pR - pL;
    const double dvn = du * nx + dv * ny;
    const double c2 = c * c;
    const double ics = rcp_any(fmax(c2, 1e-10));
    const double a1 = (dp - rhoRoe * c * dvn) * (0.5 * ics);
    const double a2 = drho - dp * ics;
    const double a3 = rhoRoe * (dv * nx - du * ny);
    const double a4 = (dp + rhoRoe * c * dvn) * (0.5 * ics);
    const double tx = -ny, ty = nx;
    const double w1 = l1 * a1, w2 = l2 * a2, w3 = l2 * a3, w4 = l4 * a4;
    // reverse: F = (FL + FR)/2 - dF/2
    double flb[4], dFb[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) { flb[v] = 0.5 * Fb[v]; dFb[v] = -0.5 * Fb[v]; }
    double pLb = flux_normal_vjp(UL, pL, nx, ny, flb, ULb);
    double pRb = flux_normal_vjp(UR, pR, nx, ny, flb, URb);
    const double w1b = dFb[0] + dFb[1] * (uRoe - c * nx) + dFb[2] * (vRoe - c * ny) + dFb[3] * (HRoe - c * vnRoe);
    const double w2b = dFb[0] + dFb[1] * uRoe + dFb[2] * vRoe + dFb[3] * 0.5 * qsq;
    const double w3b = dFb[1] * tx + dFb[2] * ty + dFb[3] * (uRoe * tx + vRoe * ty);
    const double w4b = dFb[0] + dFb[1] * (uRoe + c * nx) + dFb[2] * (vRoe + c * ny) + dFb[3] * (HRoe + c * vnRoe);
    const double wsum = w1 + w2 + w4;
    double uRoeb = dFb[1] * wsum + dFb[3] * w3 * tx;
    double vRoeb = dFb[2] * wsum + dFb[3] * w3 * ty;
    double cb = (w4 - w1) * (dFb[1] * nx + dFb[2] * ny + dFb[3] * vnRoe);
    double HRoeb = dFb[3] * (w1 + w4);
    double vnRoeb = dFb[3] * c * (w4 - w1);
    double qsqb = dFb[3] * 0.5 * w2;
    double l1b = w1b * a1, l4b = w4b * a4;
    const double l2b = w2b * a2 + w3b * a3;
    const double a1b = w1b * l1, a2b = w2b * l2, a3b = w3b * l2, a4b = w4b * l4;
    double dpb = 0.0, rhoRoeb = 0.0, dvnb = 0.0, icsb = 0.0, drhob = 0.0, dub = 0.0, dvb = 0.0;
    // a4, a3, a2, a1
    dpb += a4b * 0.5 * ics; rhoRoeb += a4b * 0.5 * ics * c * dvn; cb += a4b * 0.5 * ics * rhoRoe * dvn;
    dvnb += a4b * 0.5 * ics * rhoRoe * c; icsb += a4b * 0.5 * (dp + rhoRoe * c * dvn);
    rhoRoeb += a3b * (dv * nx - du * ny); dvb += a3b * rhoRoe * nx; dub -= a3b * rhoRoe * ny;
    drhob += a2b; dpb -= a2b * ics; icsb -= a2b * dp;
    dpb += a1b * 0.5 * ics; rhoRoeb -= a1b * 0.5 * ics * c * dvn; cb -= a1b * 0.5 * ics * rhoRoe * dvn;
    dvnb -= a1b * 0.5 * ics * rhoRoe * c; icsb += a1b * 0.5 * (dp - rhoRoe * c * dvn);
    if (c2 >= 1e-10) cb -= icsb * ics * ics * 2.0 * c;
    dub += dvnb * nx; dvb += dvnb * ny;
    pRb += dpb; pLb -= dpb;
    double uLb = -dub, uRb = dub, vLb = -dvb, vRb = dvb, rhoLb = -drhob, rhoRb = drhob;
    // entropy fix: l = (lo^2 + eps^2) / (2 eps)
    double epsb = 0.0, l1ob = l1b, l4ob = l4b;
    if (fix4) { l4ob = l4b * l4o / eps; epsb += l4b * (0.5 - l4o * l4o / (2.0 * eps * eps)); }
    if (fix1) { l1ob = l1b * l1o / eps; epsb += l1b * (0.5 - l1o * l1o / (2.0 * eps * eps)); }
    cb += 0.1 * epsb;
    const double s4 = (vnRoe + c < 0.0) ? -1.0 : 1.0;
    const double s2 = (vnRoe < 0.0) ? -1.0 : 1.0;
    const double s1 = (vnRoe - c < 0.0) ? -1.0 : 1.0;
    vnRoeb += l4ob * s4 + l2b * s2 + l1ob * s1;
    cb += l4ob * s4 - l1ob * s1;
    // c = sqrt(max(carg, 1e-10))
    if (carg >= 1e-10 && c > 0.0) {
        const double cargb = cb * 0.5 / c;
        HRoeb += cargb * (g - 1.0);
        qsqb -= cargb * (g - 1.0) * 0.5;
    }
    uRoeb += 2.0 * uRoe * qsqb + vnRoeb * nx;
    vRoeb += 2.0 * vRoe * qsqb + vnRoeb * ny;
    // Roe averages
    double sLb = (uRoeb * uL + vRoeb * vL + HRoeb * HL) * iden;
    double sRb = (uRoeb * uR + vRoeb * vR + HRoeb * HR) * iden;
    uLb += uRoeb * sL * iden; uRb += uRoeb * sR * iden;
    vLb += vRoeb * sL * iden; vRb += vRoeb * sR * iden;
    const double HLb = HRoeb * sL * iden, HRb = HRoeb * sR * iden;
    const double idenb = uRoeb * (sL * uL + sR * uR) + vRoeb * (sL * vL + sR * vR) + HRoeb * (sL * HL + sR * HR);
    sLb += rhoRoeb * sR; sRb += rhoRoeb * sL;
    if (ssum >= 1e-10) { const double t = -idenb * iden * iden; sLb += t; sRb += t; }
    if (sL > 0.0) rhoLb += sLb * 0.5 / sL;
    if (sR > 0.0) rhoRb += sRb * 0.5 / sR;
    // H = (U3 + p) ir
    ULb[3] += HLb * irL; pLb += HLb * irL; double irLb = HLb * (UL[3] + pL);
    URb[3] += HRb * irR; pRb += HRb * irR; double irRb = HRb * (UR[3] + pR);
    pressure_vjp(UL, g, pLb, ULb);
    pressure_vjp(UR, g, pRb, URb);
    // velocities and floored densities
    ULb[1] += uLb * irL; ULb[2] += vLb * irL; irLb += uLb * UL[1] + vLb * UL[2];
    URb[1] += uRb * irR; URb[2] += vRb * irR; irRb += uRb * UR[1] + vRb * UR[2];
    rhoLb -= irLb * irL * irL;
    rhoRb -= irRb * irR * irR;
    if (UL[0] >= 1e-10) ULb[0] += rhoLb;
    if (UR[0] >= 1e-10) URb[0] += rhoRb;
}

// (dFc/dUL)^T Fb into ULb, (dFc/dUR)^T Fb into URb (accumulated): the Roe
// solver by its reverse sweep, the others by eight tangent evaluations on
// dual numbers.
template <int RIEM>
__device__ __forceinline__ void riemann_vjp(const double* UL, const double* UR, double nx, double ny,
                                            double g, const double* Fb, double* ULb, double* URb) {
    if constexpr (RIEM == ZJ_RIEMANN_ROE) {
        roe_vjp(UL, UR, nx, ny, g, Fb, ULb, URb);
    } else {
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
        Dual L[4], R[4], F[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            L[v] = Dual(UL[v], (k == v) ? 1.0 : 0.0);
            R[v] = Dual(UR[v], (k == 4 + v) ? 1.0 : 0.0);
        }
        phys::riemann<RIEM>(L, R, Dual(nx), Dual(ny), Dual(g), F);
        const double t = Fb[0] * F[0].d + Fb[1] * F[1].d + Fb[2] * F[2].d + Fb[3] * F[3].d;
        if (k < 4) ULb[k] += t;
        else URb[k - 4] += t;
    }
    }
}

// (dGhost/dUi)^T Gb into Uib (accumulated): four tangent evaluations of the
// ghost state on dual numbers.
__device__ __forceinline__ void ghost_vjp(const double* Ui, double nx, double ny, int bct,
                                          const double* bcd, double g, const double* Gb,
                                          double* Uib) {
    Dual bd[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) bd[i] = Dual(bcd[i]);
#pragma unroll 1
    for (int k = 0; k < 4; ++k) {
        Dual Ud[4], Gd[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) Ud[v] = Dual(Ui[v], (k == v) ? 1.0 : 0.0);
        phys::ghost_phys(Ud, Dual(nx), Dual(ny), bct, bd, Dual(g), Gd);
        Uib[k] += Gb[0] * Gd[0].d + Gb[1] * Gd[1].d + Gb[2] * Gd[2].d + Gb[3] * Gd[3].d;
    }
}

}  // namespace adj
}  // namespace zj
