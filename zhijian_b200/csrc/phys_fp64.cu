// phys_fp64.cu -- FP64 residual and SSP-RK3 stage kernels of the conservative
// FR scheme the parameters ask for ("physics mode", compat off).
//
//   R = -(1/J) [ D_xi F~ + D_eta G~
//                + g_R'(xi) dF_1 - g_L'(xi) dF_3 + g_R'(eta) dF_2 - g_L'(eta) dF_0 ]
//   F~ = J (xi_x F + xi_y G),  G~ = J (eta_x F + eta_y G)
//   dF_e = s_e (n_out . F_common) - (extrapolated transformed flux . n_ref_out)
// with s_e = L_e/2 the edge Jacobian of a straight edge, g_L, g_R the VCJH
// correction functions of the flux type (Vincent, Castonguay & Jameson 2011),
// the common flux from the reference's Rusanov/Roe/HLLC
// (include/physics/euler.hpp:184-375) evaluated once per face point from the
// left element's side, and the ghost states of
// include/bc/boundary_condition.hpp:42-311.  No positivity clamps.
//
// Same CTA organisation as the compat kernel (compat_fp64.cu): phase A loads
// and transformed fluxes, B interface terms, C divergence + correction + RK
// update, D traces of the new state.
#include <cuda_runtime.h>

#include "zj_device.cuh"
#include "zj_kernels.h"
#include "zj_math.h"

namespace zj {
namespace {

using namespace dev;

#ifndef ZJ_PHYS_MIN_BLOCKS
#define ZJ_PHYS_MIN_BLOCKS 3
#endif

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
__device__ void ghost_phys(const double* Ui, double nx, double ny, int bct,
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

// -------------------------------------------------------------- kernels --

template <int P, int RIEM>
__global__ void __launch_bounds__(Shape<P>::THREADS, ZJ_PHYS_MIN_BLOCKS)
k_phys_stage(const StageArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS, DS = S::DS;
    __shared__ double sOps[S::NOPS];
    __shared__ __align__(16) double sF[EB * FS];
    __shared__ __align__(16) double sG[EB * FS];
    __shared__ __align__(16) double sD[EB * DS];
    __shared__ __align__(16) double sU[EB * FS];
    __shared__ double sRed[32];

    const int tid = threadIdx.x;
    for (int i = tid; i < S::NOPS; i += blockDim.x) sOps[i] = a.ops[i];

    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    const bool is_sp = valid && k < NSP;
    const bool is_fp = valid && k < NFT;
    const double g = a.gamma;
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    // ---- A: loads; transformed fluxes into shared memory
    EdgeRec r{-1, 0, kEdgeOrphan, 0};
    double4 nr = make_double4(0.0, 0.0, 0.0, 0.0);
    double qo[4], qn[4] = {0.0, 0.0, 0.0, 0.0}, u[4], Jd = 1.0;
    if (is_fp) {
        r = a.edges[e * 4 + edge];
        const double2 n01 = __ldg(reinterpret_cast<const double2*>(a.enrm + e * 4 + edge));
        const double2 n23 = __ldg(reinterpret_cast<const double2*>(a.enrm + e * 4 + edge) + 1);
        nr = make_double4(n01.x, n01.y, n23.x, n23.y);
        load4_nc(a.Tin + (e * NFT + k) * 4, qo);
    }
    if (is_sp) {
        const long long idx = e * NSP + k;
        load4(a.U + idx * 4, u);
        double ji[4];
        load4_nc(a.Jinv + idx * 4, ji);
        Jd = __ldg(a.J + idx);
        if ((k & 3) == 0 && a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        const double ir = rcp_any(u[0]);
        const double uu = u[1] * ir, vv = u[2] * ir, E = u[3] * ir;
        const double p = (g - 1.0) * u[0] * (E - 0.5 * (uu * uu + vv * vv));
        const double F[4] = {u[1], u[1] * uu + p, u[1] * vv, (u[3] + p) * uu};
        const double G[4] = {u[2], u[2] * uu, u[2] * vv + p, (u[3] + p) * vv};
        double* f = sF + el * FS + j * RS + i;
        double* h = sG + el * FS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            f[v * VS] = Jd * (ji[0] * F[v] + ji[1] * G[v]);
            h[v * VS] = Jd * (ji[2] * F[v] + ji[3] * G[v]);
        }
    }
    // The neighbour's point that coincides with this one: both elements run
    // their shared edge counter-clockwise.
    if (is_fp && !(r.flags & (kEdgeOrphan | kEdgeBoundary)))
        load4_nc(a.Tin + (((long long)r.nbr * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, qn);
    __syncthreads();   // sOps, sF, sG ready

    // ---- B: interface terms.  The common flux is evaluated from the left
    // element's side on both sides of a face (bit-identical on both).
    if (is_fp) {
        double Fd[4] = {0.0, 0.0, 0.0, 0.0};
        if (!(r.flags & kEdgeOrphan)) {
            const double nx = nr.x, ny = nr.y, s = 0.5 * nr.z;
            if (r.flags & kEdgeBoundary)
                ghost_phys(qo, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, g, qn);
            const bool right = (r.flags & kEdgeRight) != 0;
            double UL[4], UR[4], Fc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) { UL[v] = right ? qn[v] : qo[v]; UR[v] = right ? qo[v] : qn[v]; }
            riemann<RIEM>(UL, UR, nx, ny, g, Fc);
            const double ss = right ? -s : s;
            // Extrapolated transformed flux along this element's outward
            // reference normal: +F~ on edge 1, -F~ on edge 3, -G~ on edge 0,
            // +G~ on edge 2.
            const bool along_eta = (edge == 0 || edge == 2);
            double Fn[4];
            trace_point<N1, RS, VS>((along_eta ? sG : sF) + el * FS, sOps + N1 * N1,
                                    sOps + N1 * N1 + N1, edge, fp, Fn);
            const double sgn = (edge == 0 || edge == 3) ? -1.0 : 1.0;
#pragma unroll
            for (int v = 0; v < 4; ++v) Fd[v] = ss * Fc[v] - sgn * Fn[v];
        }
        store4(sD + el * DS + k * 4, Fd);
    }
    __syncthreads();

    // ---- C: divergence, VCJH correction, 1/J, stage update
    double rsq = 0.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        double u0[4];
        if (a.stage >= 2) load4(a.U0 + idx * 4, u0);
        double Di[N1], Dj[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) { Di[m] = sOps[i * N1 + m]; Dj[m] = sOps[j * N1 + m]; }
        const double* gL = sOps + N1 * N1 + 2 * N1;
        const double* gR = gL + N1;
        const double gRi = gR[i], gLi = gL[i], gRj = gR[j], gLj = gL[j];
        const double* f = sF + el * FS;
        const double* h = sG + el * FS;
        const double* d = sD + el * DS;
        double c1[4], c3[4], c2[4], c0[4];
        load4(d + (1 * N1 + j) * 4, c1);
        load4(d + (3 * N1 + (N1 - 1 - j)) * 4, c3);
        load4(d + (2 * N1 + (N1 - 1 - i)) * 4, c2);
        load4(d + (0 * N1 + i) * 4, c0);
        const double iJ = rcp_any(Jd);
        double res[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            double fr[N1];
            load_row<N1>(f + v * VS + j * RS, fr);
            double div = 0.0;
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma(Di[m], fr[m], div);
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma(Dj[m], h[v * VS + m * RS + i], div);
            const double corr = gRi * c1[v] - gLi * c3[v] + gRj * c2[v] - gLj * c0[v];
            res[v] = -(div + corr) * iJ;
        }
        if (a.stage == 0) {
            store4(a.R + idx * 4, res);
#pragma unroll
            for (int v = 0; v < 4; ++v) rsq += res[v] * res[v];
        } else {
            const double dt = *a.dt;
            double uo[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                if (a.stage == 1) uo[v] = u[v] + dt * res[v];
                else if (a.stage == 2) uo[v] = 0.75 * u0[v] + 0.25 * u[v] + 0.25 * dt * res[v];
                else uo[v] = (1.0 / 3.0) * u0[v] + (2.0 / 3.0) * u[v] + (2.0 / 3.0) * dt * res[v];
            }
            store4(a.Uout + idx * 4, uo);
            double* su = sU + el * FS + j * RS + i;
#pragma unroll
            for (int v = 0; v < 4; ++v) su[v * VS] = uo[v];
            if (a.stage == 3) {
#pragma unroll
                for (int v = 0; v < 4; ++v) rsq += res[v] * res[v];
            }
        }
    }
    if (a.stage == 0 || a.stage == 3) {
        const double bs = block_sum(rsq, sRed);
        if (tid == 0) a.partials[blockIdx.x] = bs;
    }
    if (a.stage == 0) return;
    __syncthreads();

    // ---- D: traces of the new state
    if (is_fp) {
        double t[4];
        trace_point<N1, RS, VS>(sU + el * FS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        store4(a.Tout + (e * NFT + k) * 4, t);
    }
}

template <int P, int RIEM>
cudaError_t launch_t(const StageArgs& a, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    static bool carveout_set = false;
    if (!carveout_set) {
        cudaFuncSetAttribute(k_phys_stage<P, RIEM>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        carveout_set = true;
    }
    k_phys_stage<P, RIEM><<<(unsigned)grid, S::THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

template <int P>
cudaError_t launch_p(int riemann, const StageArgs& a, cudaStream_t s) {
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV: return launch_t<P, ZJ_RIEMANN_RUSANOV>(a, s);
        case ZJ_RIEMANN_ROE: return launch_t<P, ZJ_RIEMANN_ROE>(a, s);
        case ZJ_RIEMANN_HLLC: return launch_t<P, ZJ_RIEMANN_HLLC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_phys_stage(int P, int riemann, const StageArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return launch_p<1>(riemann, a, s);
        case 2: return launch_p<2>(riemann, a, s);
        case 3: return launch_p<3>(riemann, a, s);
        case 4: return launch_p<4>(riemann, a, s);
        case 5: return launch_p<5>(riemann, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zj
