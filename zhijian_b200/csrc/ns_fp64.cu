// ns_fp64.cu -- FP64 Navier-Stokes residual and SSP-RK3 stages (physics mode,
// viscous on).  Two launches per residual:
//
//  k_ns_grad   corrected gradient Q = grad U at the solution points and its
//              traces at the flux points (written for the neighbours);
//  k_ns_stage  recomputes Q at the solution points, total flux F - F_v, the
//              common flux = Riemann(U_L, U_R) - F_v(avg U, avg Q).n, FR
//              correction, stage update and traces of the new state.
//
// Gradient: U^C = U^D + (U_c - U^D) g at the edges with the common solution
// U_c = (U_L + U_R)/2 (the ghost state on boundaries), the same VCJH
// correction functions as the flux, chain rule with the pointwise metrics:
//   dU/dxi  = D_xi U  + g_R'(xi) dU_1 + g_L'(xi) dU_3
//   dU/deta = D_eta U + g_L'(eta) dU_0 + g_R'(eta) dU_2,   dU_e = U_c - U_own
//   Q_x = xi_x dU/dxi + eta_x dU/deta,  Q_y = xi_y dU/dxi + eta_y dU/deta.
// Viscous flux: the reference's computeViscousFluxSPKernel law
// (kernels.cu:742-786); common viscous flux: average state and average
// gradients (BR2Scheme::commonFlux, navierstokes.hpp:177-204); boundaries
// copy the interior gradient (BoundaryCondition::ghostGradient).
#include <cuda_runtime.h>

#include "zj_device.cuh"
#include "zj_kernels.h"
#include "zj_math.h"
#include "zj_physics.cuh"

namespace zj {
namespace {

using namespace dev;
using namespace phys;

#ifndef ZJ_NS_MIN_BLOCKS
#define ZJ_NS_MIN_BLOCKS 2        // stage kernel
#endif
#ifndef ZJ_NSG_MIN_BLOCKS
#define ZJ_NSG_MIN_BLOCKS 4       // gradient kernel
#endif

// Corrected gradient at solution point (i, j) of one element: su is the
// element's state in the [var][row][col] shared layout, du its face jumps
// U_c - U_own in the [flux point][var] layout.
template <int N1, int RS, int VS>
__device__ __forceinline__ void corrected_gradient(const double* su, const double* du,
                                                   const double* ops, int i, int j,
                                                   const double* ji, double* Qx, double* Qy) {
    const double* gL = ops + N1 * N1 + 2 * N1;
    const double* gR = gL + N1;
    double Di[N1], Dj[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) { Di[m] = ops[i * N1 + m]; Dj[m] = ops[j * N1 + m]; }
    double d1[4], d3[4], d0[4], d2[4];
    load4(du + (1 * N1 + j) * 4, d1);
    load4(du + (3 * N1 + (N1 - 1 - j)) * 4, d3);
    load4(du + (0 * N1 + i) * 4, d0);
    load4(du + (2 * N1 + (N1 - 1 - i)) * 4, d2);
    const double gRi = gR[i], gLi = gL[i], gRj = gR[j], gLj = gL[j];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        double row[N1];
        load_row<N1>(su + v * VS + j * RS, row);
        double dxi = 0.0, deta = 0.0;
#pragma unroll
        for (int m = 0; m < N1; ++m) {
            dxi = fma(Di[m], row[m], dxi);
            deta = fma(Dj[m], su[v * VS + m * RS + i], deta);
        }
        dxi += gRi * d1[v] + gLi * d3[v];
        deta += gLj * d0[v] + gRj * d2[v];
        Qx[v] = ji[0] * dxi + ji[2] * deta;
        Qy[v] = ji[1] * dxi + ji[3] * deta;
    }
}

// Loads of a flux-point thread: edge record, normal, own trace, the
// neighbour's coinciding trace point or the ghost state.
struct FacePoint {
    EdgeRec r;
    double nx, ny, len;
    double qo[4], qn[4];
};

template <int N1>
__device__ __forceinline__ void load_face_point(const StageArgs& a, long long e, int edge, int fp,
                                                FacePoint& f) {
    constexpr int NFT = 4 * N1;
    f.r = a.edges[e * 4 + edge];
    const double2 n01 = __ldg(reinterpret_cast<const double2*>(a.enrm + e * 4 + edge));
    const double2 n23 = __ldg(reinterpret_cast<const double2*>(a.enrm + e * 4 + edge) + 1);
    f.nx = n01.x; f.ny = n01.y; f.len = n23.x;
    load4_nc(a.Tin + (e * NFT + edge * N1 + fp) * 4, f.qo);
    f.qn[0] = f.qo[0]; f.qn[1] = f.qo[1]; f.qn[2] = f.qo[2]; f.qn[3] = f.qo[3];
    if (!(f.r.flags & kEdgeOrphan)) {
        // interior: the neighbour's coinciding point; boundary: the ghost row
        // written with the trace (phys_fp64.cu)
        const long long row = (f.r.flags & kEdgeBoundary) ? a.n_elem * 4 + f.r.nbr_edge
                                                          : (long long)f.r.nbr * 4 + f.r.nbr_edge;
        load4_nc(a.Tin + (row * N1 + (N1 - 1 - fp)) * 4, f.qn);
    }
}

template <int P>
__global__ void __launch_bounds__(Shape<P>::THREADS, ZJ_NSG_MIN_BLOCKS)
k_ns_grad(const StageArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS, DS = S::DS;
    constexpr int QS = 8 * VS + (6 - (8 * VS) % 16 + 16) % 16;
    __shared__ double sOps[S::NOPS];
    __shared__ __align__(16) double sU[EB * FS];
    __shared__ __align__(16) double sDU[EB * DS];
    __shared__ __align__(16) double sQ[EB * QS];

    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    double ji[4];
    if (is_sp) {
        const long long idx = e * NSP + k;
        double u[4];
        load4(a.U + idx * 4, u);
        load4_nc(a.Jinv + idx * 4, ji);
        double* su = sU + el * FS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = u[v];
    }
    if (is_fp) {
        FacePoint f;
        load_face_point<N1>(a, e, edge, fp, f);
        double d[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) d[v] = (f.r.flags & kEdgeOrphan) ? 0.0 : 0.5 * (f.qn[v] - f.qo[v]);
        store4(sDU + el * DS + k * 4, d);
    }
    __syncthreads();
    if (is_sp) {
        double Qx[4], Qy[4];
        corrected_gradient<N1, RS, VS>(sU + el * FS, sDU + el * DS, sOps, i, j, ji, Qx, Qy);
        double* sq = sQ + el * QS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) { sq[v * VS] = Qx[v]; sq[(4 + v) * VS] = Qy[v]; }
    }
    __syncthreads();
    if (is_fp) {
        double t[8];
        trace_point<N1, RS, VS>(sQ + el * QS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        trace_point<N1, RS, VS>(sQ + el * QS + 4 * VS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge,
                                fp, t + 4);
        double* o = a.TQout + (e * NFT + k) * 8;
        store4(o, t);
        store4(o + 4, t + 4);
    }
}

template <int P, int RIEM>
__global__ void __launch_bounds__(Shape<P>::THREADS, ZJ_NS_MIN_BLOCKS)
k_ns_stage(const StageArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS, DS = S::DS;
    __shared__ double sOps[S::NOPS];
    __shared__ __align__(16) double sF[EB * FS];
    __shared__ __align__(16) double sG[EB * FS];
    __shared__ __align__(16) double sD[EB * DS];   // face jumps of U, then flux differences
    __shared__ __align__(16) double sU[EB * FS];   // stage state, then the new state
    __shared__ double sRed[32];

    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const double g = a.gamma;
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    // ---- A1: loads, face jumps, stage state into shared memory
    FacePoint f;
    double Qo[8], Qn[8];
    if (is_fp) {
        load_face_point<N1>(a, e, edge, fp, f);
        const double* qt = a.TQ + (e * NFT + k) * 8;
        load4_nc(qt, Qo);
        load4_nc(qt + 4, Qo + 4);
#pragma unroll
        for (int v = 0; v < 8; ++v) Qn[v] = Qo[v];
        if (!(f.r.flags & (kEdgeOrphan | kEdgeBoundary))) {
            const double* qn = a.TQ + (((long long)f.r.nbr * 4 + f.r.nbr_edge) * N1 + (N1 - 1 - fp)) * 8;
            load4_nc(qn, Qn);
            load4_nc(qn + 4, Qn + 4);
        }
        double d[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) d[v] = (f.r.flags & kEdgeOrphan) ? 0.0 : 0.5 * (f.qn[v] - f.qo[v]);
        store4(sD + el * DS + k * 4, d);
    }
    double u[4], ji[4], Jd = 1.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        load4(a.U + idx * 4, u);
        load4_nc(a.Jinv + idx * 4, ji);
        Jd = __ldg(a.J + idx);
        if ((k & 3) == 0 && a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        double* su = sU + el * FS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = u[v];
    }
    __syncthreads();

    // ---- A2: gradient, total transformed fluxes
    if (is_sp) {
        double Qx[4], Qy[4], Fv[4], Gv[4];
        corrected_gradient<N1, RS, VS>(sU + el * FS, sD + el * DS, sOps, i, j, ji, Qx, Qy);
        viscous_flux(u, Qx, Qy, g, a.Re, a.Pr, Fv, Gv);
        const double ir = rcp_any(u[0]);
        const double uu = u[1] * ir, vv = u[2] * ir, E = u[3] * ir;
        const double p = (g - 1.0) * u[0] * (E - 0.5 * (uu * uu + vv * vv));
        const double F[4] = {u[1] - Fv[0], u[1] * uu + p - Fv[1], u[1] * vv - Fv[2], (u[3] + p) * uu - Fv[3]};
        const double G[4] = {u[2] - Gv[0], u[2] * uu - Gv[1], u[2] * vv + p - Gv[2], (u[3] + p) * vv - Gv[3]};
        double* fo = sF + el * FS + j * RS + i;
        double* ho = sG + el * FS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            fo[v * VS] = Jd * (ji[0] * F[v] + ji[1] * G[v]);
            ho[v * VS] = Jd * (ji[2] * F[v] + ji[3] * G[v]);
        }
    }
    __syncthreads();   // face jumps and the stage state in shared memory are dead now

    // ---- B: interface terms, evaluated from the left element's side
    if (is_fp) {
        double Fd[4] = {0.0, 0.0, 0.0, 0.0};
        if (!(f.r.flags & kEdgeOrphan)) {
            const bool right = (f.r.flags & kEdgeRight) != 0;
            double UL[4], UR[4], Fc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) { UL[v] = right ? f.qn[v] : f.qo[v]; UR[v] = right ? f.qo[v] : f.qn[v]; }
            riemann<RIEM>(UL, UR, f.nx, f.ny, g, Fc);
            double Ua[4], dxa[4], dya[4], Fv[4], Gv[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Ua[v] = 0.5 * (UL[v] + UR[v]);
                dxa[v] = 0.5 * (Qo[v] + Qn[v]);
                dya[v] = 0.5 * (Qo[4 + v] + Qn[4 + v]);
            }
            viscous_flux(Ua, dxa, dya, g, a.Re, a.Pr, Fv, Gv);
            const double ss = right ? -0.5 * f.len : 0.5 * f.len;
            const bool along_eta = (edge == 0 || edge == 2);
            double Fn[4];
            trace_point<N1, RS, VS>((along_eta ? sG : sF) + el * FS, sOps + N1 * N1,
                                    sOps + N1 * N1 + N1, edge, fp, Fn);
            const double sgn = (edge == 0 || edge == 3) ? -1.0 : 1.0;
#pragma unroll
            for (int v = 0; v < 4; ++v)
                Fd[v] = ss * (Fc[v] - (Fv[v] * f.nx + Gv[v] * f.ny)) - sgn * Fn[v];
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
        const double* fo = sF + el * FS;
        const double* ho = sG + el * FS;
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
            load_row<N1>(fo + v * VS + j * RS, fr);
            double div = 0.0;
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma(Di[m], fr[m], div);
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma(Dj[m], ho[v * VS + m * RS + i], div);
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
        if (f.r.flags & kEdgeBoundary) {
            double q[4];
            ghost_phys(t, f.nx, f.ny, edge_bc_type(f.r.flags), a.bc + (long long)f.r.nbr_edge * 8, g, q);
            store4(a.Tout + ((a.n_elem * 4 + f.r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, q);
        }
    }
}

template <class K>
void prefer_shared(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
}

template <int P>
cudaError_t grad_t(const StageArgs& a, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    static bool set = false;
    if (!set) { prefer_shared(k_ns_grad<P>); set = true; }
    k_ns_grad<P><<<(unsigned)grid, S::THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

template <int P, int RIEM>
cudaError_t stage_t(const StageArgs& a, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    static bool set = false;
    if (!set) { prefer_shared(k_ns_stage<P, RIEM>); set = true; }
    k_ns_stage<P, RIEM><<<(unsigned)grid, S::THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

template <int P>
cudaError_t stage_p(int riemann, const StageArgs& a, cudaStream_t s) {
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV: return stage_t<P, ZJ_RIEMANN_RUSANOV>(a, s);
        case ZJ_RIEMANN_ROE: return stage_t<P, ZJ_RIEMANN_ROE>(a, s);
        case ZJ_RIEMANN_HLLC: return stage_t<P, ZJ_RIEMANN_HLLC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

cudaError_t launch_ns_grad(int P, const StageArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return grad_t<1>(a, s);
        case 2: return grad_t<2>(a, s);
        case 3: return grad_t<3>(a, s);
        case 4: return grad_t<4>(a, s);
        case 5: return grad_t<5>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_ns_stage(int P, int riemann, const StageArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return stage_p<1>(riemann, a, s);
        case 2: return stage_p<2>(riemann, a, s);
        case 3: return stage_p<3>(riemann, a, s);
        case 4: return stage_p<4>(riemann, a, s);
        case 5: return stage_p<5>(riemann, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zj
