// zj_physics.cuh -- device physics of the physics-mode residual kernels:
// ideal-gas relations, the reference's Riemann solvers and ghost states, and
// the viscous flux.
#pragma once

#include <cuda_runtime.h>

#include "zj_device.cuh"
#include "zj_fr.h"
#include "zj_math.h"

namespace zj {
namespace phys {

using namespace dev;

// ------------------------------------------------------------ physics --

// IdealGas::pressure (euler.hpp:16-23)
__device__ __forceinline__ double pressure(const double* U, double g) {
    const double ir = rcp_any(U[0]);
    const double u = U[1] * ir, v = U[2] * ir, E = U[3] * ir;
    return (g - 1.0) * U[0] * (E - 0.5 * (u * u + v * v));
}

// IdealGas::soundSpeed (euler.hpp:34-41)
__device__ __forceinline__ double sound_speed(double p_raw, double rho_raw, double g) {
    const double p = fmax(p_raw, 1e-10), rho = fmax(rho_raw, 1e-10);
    return zj_sqrt(g * p * rcp_any(rho));
}

// IdealGas::fluxNormal (euler.hpp:133-147): floored density and pressure,
// total enthalpy from the unfloored pressure.
__device__ __forceinline__ void flux_normal(const double* U, double praw, double nx, double ny,
                                            double* Fn) {
    const double rho = fmax(U[0], 1e-10);
    const double ir = rcp_any(rho);
    const double u = U[1] * ir, v = U[2] * ir;
    const double p = fmax(praw, 1e-10);
    const double H = U[3] + praw;
    const double vn = u * nx + v * ny;
    Fn[0] = rho * vn;
    Fn[1] = rho * u * vn + p * nx;
    Fn[2] = rho * v * vn + p * ny;
    Fn[3] = H * vn;
}

// RiemannSolvers::rusanov (euler.hpp:184-200): s = |u| + c of each side.
__device__ __forceinline__ void riemann_rusanov(const double* UL, const double* UR, double nx,
                                                double ny, double g, double* F) {
    const double pL = pressure(UL, g), pR = pressure(UR, g);
    double FL[4], FR[4];
    flux_normal(UL, pL, nx, ny, FL);
    flux_normal(UR, pR, nx, ny, FR);
    const double irL = rcp_any(UL[0]), irR = rcp_any(UR[0]);
    const double uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    const double sL = zj_sqrt(uL * uL + vL * vL) + sound_speed(pL, UL[0], g);
    const double sR = zj_sqrt(uR * uR + vR * vR) + sound_speed(pR, UR[0], g);
    const double smax = fmax(sL, sR);
#pragma unroll
    for (int i = 0; i < 4; ++i) F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * smax * (UR[i] - UL[i]);
}

// RiemannSolvers::roe with Harten's entropy fix (euler.hpp:204-294).
__device__ __forceinline__ void riemann_roe(const double* UL, const double* UR, double nx,
                                            double ny, double g, double* F) {
    const double rhoL = fmax(UL[0], 1e-10), rhoR = fmax(UR[0], 1e-10);
    const double irL = rcp_any(rhoL), irR = rcp_any(rhoR);
    const double uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    const double pL = pressure(UL, g), pR = pressure(UR, g);
    const double HL = (UL[3] + pL) * irL, HR = (UR[3] + pR) * irR;
    const double sL = zj_sqrt(rhoL), sR = zj_sqrt(rhoR);
    const double iden = rcp_any(fmax(sL + sR, 1e-10));
    const double rhoRoe = sL * sR;
    const double uRoe = (sL * uL + sR * uR) * iden, vRoe = (sL * vL + sR * vR) * iden;
    const double HRoe = (sL * HL + sR * HR) * iden;
    const double vnRoe = uRoe * nx + vRoe * ny, qsq = uRoe * uRoe + vRoe * vRoe;
    const double c = zj_sqrt(fmax((g - 1.0) * (HRoe - 0.5 * qsq), 1e-10));
    double l1 = fabs(vnRoe - c);
    const double l2 = fabs(vnRoe);
    double l4 = fabs(vnRoe + c);
    const double eps = 0.1 * c;
    if (l1 < eps) l1 = (l1 * l1 + eps * eps) * rcp_any(2.0 * eps);
    if (l4 < eps) l4 = (l4 * l4 + eps * eps) * rcp_any(2.0 * eps);
    const double drho = rhoR - rhoL, du = uR - uL, dv = vR - vL;
    const double dp = pR - pL;
    const double dvn = du * nx + dv * ny;
    const double ics = rcp_any(fmax(c * c, 1e-10));
    const double a1 = (dp - rhoRoe * c * dvn) * (0.5 * ics);
    const double a2 = drho - dp * ics;
    const double a3 = rhoRoe * (dv * nx - du * ny);
    const double a4 = (dp + rhoRoe * c * dvn) * (0.5 * ics);
    double FL[4], FR[4];
    flux_normal(UL, pL, nx, ny, FL);
    flux_normal(UR, pR, nx, ny, FR);
    const double tx = -ny, ty = nx;
    const double w1 = l1 * a1, w2 = l2 * a2, w3 = l2 * a3, w4 = l4 * a4;
    const double dF0 = w1 + w2 + w4;
    const double dF1 = w1 * (uRoe - c * nx) + w2 * uRoe + w3 * tx + w4 * (uRoe + c * nx);
    const double dF2 = w1 * (vRoe - c * ny) + w2 * vRoe + w3 * ty + w4 * (vRoe + c * ny);
    const double dF3 = w1 * (HRoe - c * vnRoe) + w2 * 0.5 * qsq + w3 * (uRoe * tx + vRoe * ty) +
                       w4 * (HRoe + c * vnRoe);
    F[0] = 0.5 * (FL[0] + FR[0]) - 0.5 * dF0;
    F[1] = 0.5 * (FL[1] + FR[1]) - 0.5 * dF1;
    F[2] = 0.5 * (FL[2] + FR[2]) - 0.5 * dF2;
    F[3] = 0.5 * (FL[3] + FR[3]) - 0.5 * dF3;
}

__device__ __forceinline__ double away_from_zero(double d) {
    return (fabs(d) < 1e-10) ? ((d >= 0) ? 1e-10 : -1e-10) : d;
}

// RiemannSolvers::hllc (euler.hpp:298-375).
__device__ __forceinline__ void riemann_hllc(const double* UL, const double* UR, double nx,
                                             double ny, double g, double* F) {
    const double rhoL = fmax(UL[0], 1e-10), rhoR = fmax(UR[0], 1e-10);
    const double irL = rcp_any(rhoL), irR = rcp_any(rhoR);
    const double uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    const double pLr = pressure(UL, g), pRr = pressure(UR, g);
    const double pL = fmax(pLr, 1e-10), pR = fmax(pRr, 1e-10);
    const double cL = sound_speed(pLr, UL[0], g), cR = sound_speed(pRr, UR[0], g);
    const double vnL = uL * nx + vL * ny, vnR = uR * nx + vR * ny;
    double ps = 0.5 * (pL + pR) - 0.5 * (vnR - vnL) * 0.5 * (rhoL + rhoR) * 0.5 * (cL + cR);
    ps = fmax(ps, 1e-10);
    const double k = (g + 1.0) / (2.0 * g);
    const double qL = (ps <= pL) ? 1.0 : zj_sqrt(1.0 + k * (ps * rcp_any(pL) - 1.0));
    const double qR = (ps <= pR) ? 1.0 : zj_sqrt(1.0 + k * (ps * rcp_any(pR) - 1.0));
    const double SL = vnL - cL * qL, SR = vnR + cR * qR;
    const double dSM = away_from_zero(rhoL * (SL - vnL) - rhoR * (SR - vnR));
    const double SM = (pR - pL + rhoL * vnL * (SL - vnL) - rhoR * vnR * (SR - vnR)) / dSM;
    // One star-state evaluation for either side of the contact (no divergent
    // call sites): the side is selected, then the same arithmetic runs.
    const bool left = (SM >= 0.0);
    const double* Uk = left ? UL : UR;
    const double rk = left ? rhoL : rhoR, uk = left ? uL : uR, vk = left ? vL : vR;
    const double vnk = left ? vnL : vnR, pk = left ? pL : pR, Sk = left ? SL : SR;
    const double pkr = left ? pLr : pRr;
    const double dK = away_from_zero(Sk - SM);
    const double dvn = away_from_zero(Sk - vnk);
    const double fac = rk * dvn / dK;
    double Us[4];
    Us[0] = fac;
    Us[1] = fac * (uk + (SM - vnk) * nx);
    Us[2] = fac * (vk + (SM - vnk) * ny);
    Us[3] = fac * (Uk[3] / rk + (SM - vnk) * (SM + pk / (rk * dvn)));
    double Fk[4];
    flux_normal(Uk, pkr, nx, ny, Fk);
#pragma unroll
    for (int i = 0; i < 4; ++i) F[i] = Fk[i] + Sk * (Us[i] - Uk[i]);
    if (SL >= 0.0) flux_normal(UL, pLr, nx, ny, F);
    else if (SR <= 0.0) flux_normal(UR, pRr, nx, ny, F);
}

template <int RIEM>
__device__ __forceinline__ void riemann(const double* UL, const double* UR, double nx, double ny,
                                        double g, double* F) {
    if (RIEM == ZJ_RIEMANN_ROE) riemann_roe(UL, UR, nx, ny, g, F);
    else if (RIEM == ZJ_RIEMANN_HLLC) riemann_hllc(UL, UR, nx, ny, g, F);
    else riemann_rusanov(UL, UR, nx, ny, g, F);
}

__device__ __forceinline__ void prim2cons(double rho, double u, double v, double p, double g,
                                          double* U) {
    U[0] = rho; U[1] = rho * u; U[2] = rho * v;
    U[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
}

// BoundaryCondition::ghostState of every class (boundary_condition.hpp:42-311)
// with the parameters createBCFromSpec gives them (boundary_condition.cpp:32-64),
// packed per boundary slot: far-field (rho, u, v, p) at infinity; outflow
// p_static; inflow p_total, T_total, flow direction; wall T_wall (0: adiabatic).
__device__ __forceinline__ void ghost_phys(const double* Ui, double nx, double ny, int bct,
                           const double* __restrict__ bcd, double g, double* Ug) {
    const double rho = Ui[0];
    const double u = Ui[1] / rho, v = Ui[2] / rho;
    const double p = pressure(Ui, g);
    switch (bct) {
        case ZJ_BC_WALL: {
            const double Tw = bcd[0];
            prim2cons(rho, -u, -v, (Tw > 0) ? rho * Tw : p, g, Ug);
            break;
        }
        case ZJ_BC_SLIPWALL: case ZJ_BC_SYMMETRY: {
            const double vn = u * nx + v * ny;
            prim2cons(rho, u - 2.0 * vn * nx, v - 2.0 * vn * ny, p, g, Ug);
            break;
        }
        case ZJ_BC_FARFIELD: {
            const double r_inf = bcd[0], u_inf = bcd[1], v_inf = bcd[2], p_inf = bcd[3];
            double Uinf[4];
            prim2cons(r_inf, u_inf, v_inf, p_inf, g, Uinf);
            const double c_inf = sound_speed(pressure(Uinf, g), Uinf[0], g);
            const double c_i = sound_speed(p, rho, g);
            const double vn_i = u * nx + v * ny, vn_inf = u_inf * nx + v_inf * ny;
            const double Rp = vn_i + 2.0 * c_i / (g - 1.0), Rm = vn_inf - 2.0 * c_inf / (g - 1.0);
            const double vn_b = 0.5 * (Rp + Rm), c_b = 0.25 * (g - 1.0) * (Rp - Rm);
            const bool out = (vn_b >= 0);
            const double vt = out ? (u * (-ny) + v * nx) : (u_inf * (-ny) + v_inf * nx);
            const double s = out ? p / pow(rho, g) : p_inf / pow(r_inf, g);
            const double rb = pow(c_b * c_b / (g * s), 1.0 / (g - 1.0));
            const double pb = rb * c_b * c_b / g;
            prim2cons(rb, vn_b * nx - vt * ny, vn_b * ny + vt * nx, pb, g, Ug);
            break;
        }
        case ZJ_BC_INFLOW: {
            const double pt = bcd[0], Tt = bcd[1], dx = bcd[2], dy = bcd[3];
            double M2 = 2.0 / (g - 1.0) * (pow(p / pt, -(g - 1.0) / g) - 1.0);
            M2 = fmax(M2, 0.0);
            const double Mn = sqrt(M2);
            const double T = Tt / (1.0 + 0.5 * (g - 1.0) * M2);
            const double rb = p / T;
            const double vel = Mn * sqrt(g * p / rb);
            prim2cons(rb, vel * dx, vel * dy, p, g, Ug);
            break;
        }
        case ZJ_BC_OUTFLOW:
            prim2cons(rho, u, v, bcd[0], g, Ug);
            break;
        default:
            Ug[0] = Ui[0]; Ug[1] = Ui[1]; Ug[2] = Ui[2]; Ug[3] = Ui[3];
    }
}

// Viscous flux of the reference's computeViscousFluxSPKernel
// (kernels.cu:742-786): velocity and temperature gradients from the
// conservative gradients dx = dU/dx, dy = dU/dy; mu = T^0.7/Re,
// k = mu gamma / ((gamma-1) Pr); Stokes hypothesis.
__device__ __forceinline__ void viscous_flux(const double* s, const double* dx, const double* dy,
                                             double g, double Re, double Pr, double* Fv,
                                             double* Gv) {
    const double ir = rcp_any(s[0]);
    const double u = s[1] * ir, v = s[2] * ir;
    const double dudx = (dx[1] - u * dx[0]) * ir, dudy = (dy[1] - u * dy[0]) * ir;
    const double dvdx = (dx[2] - v * dx[0]) * ir, dvdy = (dy[2] - v * dy[0]) * ir;
    const double p = (g - 1.0) * s[0] * (s[3] * ir - 0.5 * (u * u + v * v));
    const double T = p * ir;
    const double dpdx = (g - 1.0) * (dx[3] - 0.5 * dx[0] * (u * u + v * v) - s[0] * (u * dudx + v * dvdx));
    const double dpdy = (g - 1.0) * (dy[3] - 0.5 * dy[0] * (u * u + v * v) - s[0] * (u * dudy + v * dvdy));
    const double dTdx = (dpdx - T * dx[0]) * ir, dTdy = (dpdy - T * dy[0]) * ir;
    const double mu = pow(T, 0.7) / Re;
    const double k = mu * g / ((g - 1.0) * Pr);
    const double div = dudx + dvdy, lam = -2.0 / 3.0 * mu;
    const double txx = 2.0 * mu * dudx + lam * div, tyy = 2.0 * mu * dvdy + lam * div;
    const double txy = mu * (dudy + dvdx);
    Fv[0] = 0.0; Fv[1] = txx; Fv[2] = txy; Fv[3] = u * txx + v * txy + k * dTdx;
    Gv[0] = 0.0; Gv[1] = txy; Gv[2] = tyy; Gv[3] = u * txy + v * tyy + k * dTdy;
}

}  // namespace phys
}  // namespace zj
