// zj_physics.cuh -- device physics of the physics-mode residual kernels:
// ideal-gas relations, the reference's Riemann solvers and ghost states, and
// the viscous flux.  Templated on the arithmetic type T: double for the FP64
// path, float for the mixed-precision form.  Both instantiations run the same
// operations in the same order; the FP64 one is the reference-parity path.
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
template <typename T>
__device__ __forceinline__ T pressure(const T* U, T g) {
    const T ir = rcp_any(U[0]);
    const T u = U[1] * ir, v = U[2] * ir, E = U[3] * ir;
    return (g - T(1)) * U[0] * (E - T(0.5) * (u * u + v * v));
}

// The same with ir = 1/U[0] already computed (identical arithmetic).
template <typename T>
__device__ __forceinline__ T pressure_ir(const T* U, T ir, T g) {
    const T u = U[1] * ir, v = U[2] * ir, E = U[3] * ir;
    return (g - T(1)) * U[0] * (E - T(0.5) * (u * u + v * v));
}

// IdealGas::soundSpeed (euler.hpp:34-41)
template <typename T>
__device__ __forceinline__ T sound_speed(T p_raw, T rho_raw, T g) {
    const T p = max_any(p_raw, T(1e-10)), rho = max_any(rho_raw, T(1e-10));
    return sqrt_any(g * p * rcp_any(rho));
}

// IdealGas::fluxNormal (euler.hpp:133-147): floored density and pressure,
// total enthalpy from the unfloored pressure.
template <typename T>
__device__ __forceinline__ void flux_normal(const T* U, T praw, T nx, T ny, T* Fn) {
    const T rho = max_any(U[0], T(1e-10));
    const T ir = rcp_any(rho);
    const T u = U[1] * ir, v = U[2] * ir;
    const T p = max_any(praw, T(1e-10));
    const T H = U[3] + praw;
    const T vn = u * nx + v * ny;
    Fn[0] = rho * vn;
    Fn[1] = rho * u * vn + p * nx;
    Fn[2] = rho * v * vn + p * ny;
    Fn[3] = H * vn;
}

// flux_normal with the floored density rho = max(U[0], 1e-10) and its
// reciprocal ir already computed (identical arithmetic).
template <typename T>
__device__ __forceinline__ void flux_normal_ir(const T* U, T rho, T ir, T praw, T nx, T ny, T* Fn) {
    const T u = U[1] * ir, v = U[2] * ir;
    const T p = max_any(praw, T(1e-10));
    const T H = U[3] + praw;
    const T vn = u * nx + v * ny;
    Fn[0] = rho * vn;
    Fn[1] = rho * u * vn + p * nx;
    Fn[2] = rho * v * vn + p * ny;
    Fn[3] = H * vn;
}

// 1/U[0] given ir = 1/max(U[0], 1e-10): the same value unless the floor
// applied (then computed).
template <typename T>
__device__ __forceinline__ T raw_rcp(const T* U, T ir) {
    T r = ir;
    if (!(U[0] >= T(1e-10))) r = rcp_any(U[0]);
    return r;
}

// RiemannSolvers::rusanov (euler.hpp:184-200): s = |u| + c of each side.
template <typename T>
__device__ __forceinline__ void riemann_rusanov(const T* UL, const T* UR, T nx, T ny, T g, T* F) {
    const T pL = pressure(UL, g), pR = pressure(UR, g);
    T FL[4], FR[4];
    flux_normal(UL, pL, nx, ny, FL);
    flux_normal(UR, pR, nx, ny, FR);
    const T irL = rcp_any(UL[0]), irR = rcp_any(UR[0]);
    const T uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    const T sL = sqrt_any(uL * uL + vL * vL) + sound_speed(pL, UL[0], g);
    const T sR = sqrt_any(uR * uR + vR * vR) + sound_speed(pR, UR[0], g);
    const T smax = max_any(sL, sR);
#pragma unroll
    for (int i = 0; i < 4; ++i) F[i] = T(0.5) * (FL[i] + FR[i]) - T(0.5) * smax * (UR[i] - UL[i]);
}

// RiemannSolvers::roe with Harten's entropy fix (euler.hpp:204-294).
template <typename T>
__device__ __forceinline__ void riemann_roe(const T* UL, const T* UR, T nx, T ny, T g, T* F) {
    const T rhoL = max_any(UL[0], T(1e-10)), rhoR = max_any(UR[0], T(1e-10));
    const T irL = rcp_any(rhoL), irR = rcp_any(rhoR);
    const T uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    // pressure() and flux_normal() take 1/U[0] and 1/max(U[0], 1e-10): the
    // reciprocals above, reused (the same values, each computed once)
    const T pL = pressure_ir(UL, raw_rcp(UL, irL), g), pR = pressure_ir(UR, raw_rcp(UR, irR), g);
    const T HL = (UL[3] + pL) * irL, HR = (UR[3] + pR) * irR;
    const T sL = sqrt_any(rhoL), sR = sqrt_any(rhoR);
    const T iden = rcp_any(max_any(sL + sR, T(1e-10)));
    const T rhoRoe = sL * sR;
    const T uRoe = (sL * uL + sR * uR) * iden, vRoe = (sL * vL + sR * vR) * iden;
    const T HRoe = (sL * HL + sR * HR) * iden;
    const T vnRoe = uRoe * nx + vRoe * ny, qsq = uRoe * uRoe + vRoe * vRoe;
    const T c = sqrt_any(max_any((g - T(1)) * (HRoe - T(0.5) * qsq), T(1e-10)));
    T l1 = abs_any(vnRoe - c);
    const T l2 = abs_any(vnRoe);
    T l4 = abs_any(vnRoe + c);
    const T eps = T(0.1) * c;
    if (l1 < eps) l1 = (l1 * l1 + eps * eps) * rcp_any(T(2) * eps);
    if (l4 < eps) l4 = (l4 * l4 + eps * eps) * rcp_any(T(2) * eps);
    const T drho = rhoR - rhoL, du = uR - uL, dv = vR - vL;
    const T dp = pR - pL;
    const T dvn = du * nx + dv * ny;
    const T ics = rcp_any(max_any(c * c, T(1e-10)));
    const T a1 = (dp - rhoRoe * c * dvn) * (T(0.5) * ics);
    const T a2 = drho - dp * ics;
    const T a3 = rhoRoe * (dv * nx - du * ny);
    const T a4 = (dp + rhoRoe * c * dvn) * (T(0.5) * ics);
    T FL[4], FR[4];
    flux_normal_ir(UL, rhoL, irL, pL, nx, ny, FL);
    flux_normal_ir(UR, rhoR, irR, pR, nx, ny, FR);
    const T tx = -ny, ty = nx;
    const T w1 = l1 * a1, w2 = l2 * a2, w3 = l2 * a3, w4 = l4 * a4;
    const T dF0 = w1 + w2 + w4;
    const T dF1 = w1 * (uRoe - c * nx) + w2 * uRoe + w3 * tx + w4 * (uRoe + c * nx);
    const T dF2 = w1 * (vRoe - c * ny) + w2 * vRoe + w3 * ty + w4 * (vRoe + c * ny);
    const T dF3 = w1 * (HRoe - c * vnRoe) + w2 * T(0.5) * qsq + w3 * (uRoe * tx + vRoe * ty) +
                  w4 * (HRoe + c * vnRoe);
    F[0] = T(0.5) * (FL[0] + FR[0]) - T(0.5) * dF0;
    F[1] = T(0.5) * (FL[1] + FR[1]) - T(0.5) * dF1;
    F[2] = T(0.5) * (FL[2] + FR[2]) - T(0.5) * dF2;
    F[3] = T(0.5) * (FL[3] + FR[3]) - T(0.5) * dF3;
}

template <typename T>
__device__ __forceinline__ T away_from_zero(T d) {
    return (abs_any(d) < T(1e-10)) ? ((d >= T(0)) ? T(1e-10) : T(-1e-10)) : d;
}

// RiemannSolvers::hllc (euler.hpp:298-375).
template <typename T>
__device__ __forceinline__ void riemann_hllc(const T* UL, const T* UR, T nx, T ny, T g, T* F) {
    const T rhoL = max_any(UL[0], T(1e-10)), rhoR = max_any(UR[0], T(1e-10));
    const T irL = rcp_any(rhoL), irR = rcp_any(rhoR);
    const T uL = UL[1] * irL, vL = UL[2] * irL, uR = UR[1] * irR, vR = UR[2] * irR;
    const T pLr = pressure(UL, g), pRr = pressure(UR, g);
    const T pL = max_any(pLr, T(1e-10)), pR = max_any(pRr, T(1e-10));
    const T cL = sound_speed(pLr, UL[0], g), cR = sound_speed(pRr, UR[0], g);
    const T vnL = uL * nx + vL * ny, vnR = uR * nx + vR * ny;
    T ps = T(0.5) * (pL + pR) - T(0.5) * (vnR - vnL) * T(0.5) * (rhoL + rhoR) * T(0.5) * (cL + cR);
    ps = max_any(ps, T(1e-10));
    const T k = div_any(g + T(1), T(2) * g);
    const T qL = (ps <= pL) ? T(1) : sqrt_any(T(1) + k * (ps * rcp_any(pL) - T(1)));
    const T qR = (ps <= pR) ? T(1) : sqrt_any(T(1) + k * (ps * rcp_any(pR) - T(1)));
    const T SL = vnL - cL * qL, SR = vnR + cR * qR;
    const T dSM = away_from_zero(rhoL * (SL - vnL) - rhoR * (SR - vnR));
    const T SM = div_any(pR - pL + rhoL * vnL * (SL - vnL) - rhoR * vnR * (SR - vnR), dSM);
    // One star-state evaluation for either side of the contact (no divergent
    // call sites): the side is selected, then the same arithmetic runs.
    const bool left = (SM >= T(0));
    const T* Uk = left ? UL : UR;
    const T rk = left ? rhoL : rhoR, uk = left ? uL : uR, vk = left ? vL : vR;
    const T vnk = left ? vnL : vnR, pk = left ? pL : pR, Sk = left ? SL : SR;
    const T pkr = left ? pLr : pRr;
    const T dK = away_from_zero(Sk - SM);
    const T dvn = away_from_zero(Sk - vnk);
    const T fac = div_any(rk * dvn, dK);
    T Us[4];
    Us[0] = fac;
    Us[1] = fac * (uk + (SM - vnk) * nx);
    Us[2] = fac * (vk + (SM - vnk) * ny);
    Us[3] = fac * (div_any(Uk[3], rk) + (SM - vnk) * (SM + div_any(pk, rk * dvn)));
    T Fk[4];
    flux_normal(Uk, pkr, nx, ny, Fk);
#pragma unroll
    for (int i = 0; i < 4; ++i) F[i] = Fk[i] + Sk * (Us[i] - Uk[i]);
    if (SL >= T(0)) flux_normal(UL, pLr, nx, ny, F);
    else if (SR <= T(0)) flux_normal(UR, pRr, nx, ny, F);
}

template <int RIEM, typename T>
__device__ __forceinline__ void riemann(const T* UL, const T* UR, T nx, T ny, T g, T* F) {
    if (RIEM == ZJ_RIEMANN_ROE) riemann_roe(UL, UR, nx, ny, g, F);
    else if (RIEM == ZJ_RIEMANN_HLLC) riemann_hllc(UL, UR, nx, ny, g, F);
    else riemann_rusanov(UL, UR, nx, ny, g, F);
}

template <typename T>
__device__ __forceinline__ void prim2cons(T rho, T u, T v, T p, T g, T* U) {
    U[0] = rho; U[1] = rho * u; U[2] = rho * v;
    U[3] = div_any(p, g - T(1)) + T(0.5) * rho * (u * u + v * v);
}

// BoundaryCondition::ghostState of every class (boundary_condition.hpp:42-311)
// with the parameters createBCFromSpec gives them (boundary_condition.cpp:32-64),
// packed per boundary slot: far-field (rho, u, v, p) at infinity; outflow
// p_static; inflow p_total, T_total, flow direction; wall T_wall (0: adiabatic).
template <typename T>
__device__ __forceinline__ void ghost_phys(const T* Ui, T nx, T ny, int bct,
                                           const T* __restrict__ bcd, T g, T* Ug) {
    const T rho = Ui[0];
    const T u = div_any(Ui[1], rho), v = div_any(Ui[2], rho);
    const T p = pressure(Ui, g);
    switch (bct) {
        case ZJ_BC_WALL: {
            const T Tw = bcd[0];
            prim2cons(rho, -u, -v, (Tw > T(0)) ? rho * Tw : p, g, Ug);
            break;
        }
        case ZJ_BC_SLIPWALL: case ZJ_BC_SYMMETRY: {
            const T vn = u * nx + v * ny;
            prim2cons(rho, u - T(2) * vn * nx, v - T(2) * vn * ny, p, g, Ug);
            break;
        }
        case ZJ_BC_FARFIELD: {
            const T r_inf = bcd[0], u_inf = bcd[1], v_inf = bcd[2], p_inf = bcd[3];
            T Uinf[4];
            prim2cons(r_inf, u_inf, v_inf, p_inf, g, Uinf);
            const T c_inf = sound_speed(pressure(Uinf, g), Uinf[0], g);
            const T c_i = sound_speed(p, rho, g);
            const T vn_i = u * nx + v * ny, vn_inf = u_inf * nx + v_inf * ny;
            const T Rp = vn_i + div_any(T(2) * c_i, g - T(1)), Rm = vn_inf - div_any(T(2) * c_inf, g - T(1));
            const T vn_b = T(0.5) * (Rp + Rm), c_b = T(0.25) * (g - T(1)) * (Rp - Rm);
            const bool out = (vn_b >= T(0));
            const T vt = out ? (u * (-ny) + v * nx) : (u_inf * (-ny) + v_inf * nx);
            const T s = out ? div_any(p, pow_any(rho, g)) : div_any(p_inf, pow_any(r_inf, g));
            const T rb = pow_any(div_any(c_b * c_b, g * s), div_any(T(1), g - T(1)));
            const T pb = div_any(rb * c_b * c_b, g);
            prim2cons(rb, vn_b * nx - vt * ny, vn_b * ny + vt * nx, pb, g, Ug);
            break;
        }
        case ZJ_BC_INFLOW: {
            const T pt = bcd[0], Tt = bcd[1], dx = bcd[2], dy = bcd[3];
            T M2 = div_any(T(2), g - T(1)) * (pow_any(div_any(p, pt), div_any(-(g - T(1)), g)) - T(1));
            M2 = max_any(M2, T(0));
            const T Mn = sqrt_ieee(M2);
            const T Tb = div_any(Tt, T(1) + T(0.5) * (g - T(1)) * M2);
            const T rb = div_any(p, Tb);
            const T vel = Mn * sqrt_ieee(div_any(g * p, rb));
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
template <typename T>
__device__ __forceinline__ void viscous_flux(const T* s, const T* dx, const T* dy, T g, T Re,
                                             T Pr, T* Fv, T* Gv) {
    const T ir = rcp_any(s[0]);
    const T u = s[1] * ir, v = s[2] * ir;
    const T dudx = (dx[1] - u * dx[0]) * ir, dudy = (dy[1] - u * dy[0]) * ir;
    const T dvdx = (dx[2] - v * dx[0]) * ir, dvdy = (dy[2] - v * dy[0]) * ir;
    const T p = (g - T(1)) * s[0] * (s[3] * ir - T(0.5) * (u * u + v * v));
    const T Tm = p * ir;
    const T dpdx = (g - T(1)) * (dx[3] - T(0.5) * dx[0] * (u * u + v * v) - s[0] * (u * dudx + v * dvdx));
    const T dpdy = (g - T(1)) * (dy[3] - T(0.5) * dy[0] * (u * u + v * v) - s[0] * (u * dudy + v * dvdy));
    const T dTdx = (dpdx - Tm * dx[0]) * ir, dTdy = (dpdy - Tm * dy[0]) * ir;
    const T mu = div_any(visc_pow(Tm), Re);
    const T k = div_any(mu * g, (g - T(1)) * Pr);
    const T div = dudx + dvdy, lam = T(-2.0 / 3.0) * mu;
    const T txx = T(2) * mu * dudx + lam * div, tyy = T(2) * mu * dvdy + lam * div;
    const T txy = mu * (dudy + dvdx);
    Fv[0] = T(0); Fv[1] = txx; Fv[2] = txy; Fv[3] = u * txx + v * txy + k * dTdx;
    Gv[0] = T(0); Gv[1] = txy; Gv[2] = tyy; Gv[3] = u * txy + v * tyy + k * dTdy;
}

// viscous_flux with ir = 1/s[0] supplied and the law's two divisions taken
// as products with iRe = 1/Re and kfac = gamma/((gamma-1) Pr), computed once
// per thread (each within 2 ulp of the divided form).
template <typename T>
__device__ __forceinline__ void viscous_flux_f(const T* s, T ir, const T* dx, const T* dy, T g, T iRe,
                                               T kfac, T* Fv, T* Gv) {
    const T u = s[1] * ir, v = s[2] * ir;
    const T dudx = (dx[1] - u * dx[0]) * ir, dudy = (dy[1] - u * dy[0]) * ir;
    const T dvdx = (dx[2] - v * dx[0]) * ir, dvdy = (dy[2] - v * dy[0]) * ir;
    const T p = (g - T(1)) * s[0] * (s[3] * ir - T(0.5) * (u * u + v * v));
    const T Tm = p * ir;
    const T dpdx = (g - T(1)) * (dx[3] - T(0.5) * dx[0] * (u * u + v * v) - s[0] * (u * dudx + v * dvdx));
    const T dpdy = (g - T(1)) * (dy[3] - T(0.5) * dy[0] * (u * u + v * v) - s[0] * (u * dudy + v * dvdy));
    const T dTdx = (dpdx - Tm * dx[0]) * ir, dTdy = (dpdy - Tm * dy[0]) * ir;
    const T mu = visc_pow(Tm) * iRe;
    const T k = mu * kfac;
    const T div = dudx + dvdy, lam = T(-2.0 / 3.0) * mu;
    const T txx = T(2) * mu * dudx + lam * div, tyy = T(2) * mu * dvdy + lam * div;
    const T txy = mu * (dudy + dvdx);
    Fv[0] = T(0); Fv[1] = txx; Fv[2] = txy; Fv[3] = u * txx + v * txy + k * dTdx;
    Gv[0] = T(0); Gv[1] = txy; Gv[2] = tyy; Gv[3] = u * txy + v * tyy + k * dTdy;
}

// Neumann data of the walls imposed on the common normal viscous flux Fvn of
// a boundary face (the gradient there is the interior one,
// BoundaryCondition::ghostGradient, boundary_condition.hpp:25-31): a slip or
// symmetry wall carries no shear stress and no heat flux (only tau_nn n
// remains; its energy work vanishes with u.n = 0), an adiabatic no-slip wall
// (T_wall = 0) no heat flux (its velocity is zero, so the energy flux is the
// heat flux).  These are the conditions the reference's wall classes state
// (boundary_condition.hpp:60-67, 146-155).  With the interior gradient and no
// such data the face adds u q to the discrete energy (BR1, sign-indefinite),
// which grows at the corners of slip-walled boxes.  The map is a symmetric
// projection: its transpose is itself.
template <typename T>
__device__ __forceinline__ void wall_viscous_closure(int bc_type, bool adiabatic, T nx, T ny, T* Fvn) {
    if (bc_type == ZJ_BC_SLIPWALL || bc_type == ZJ_BC_SYMMETRY) {
        const T tnn = Fvn[1] * nx + Fvn[2] * ny;
        Fvn[1] = tnn * nx;
        Fvn[2] = tnn * ny;
        Fvn[3] = T(0);
    } else if (bc_type == ZJ_BC_WALL && adiabatic) {
        Fvn[3] = T(0);
    }
}

// The closure of boundary face r (no-op elsewhere, partition interfaces
// included); bc is the face data table.
template <typename T, typename B>
__device__ __forceinline__ void boundary_viscous_closure(const EdgeRec& r, const B* bc, T nx, T ny, T* Fvn) {
    if ((r.flags & (kEdgeBoundary | kEdgeInterface)) != kEdgeBoundary) return;
    const int bt = edge_bc_type(r.flags);
    const bool adiabatic = bt == ZJ_BC_WALL && !(bc[(long long)r.nbr_edge * 8] > B(0));
    wall_viscous_closure(bt, adiabatic, nx, ny, Fvn);
}

}  // namespace phys
}  // namespace zj
