// adjoint.cu -- vector-Jacobian product of the physics-mode residual (FP64):
// W = (dR/dU)^T L, written as the transpose of the forward kernels, pass by
// pass (the forward residual is phys_kernels.cuh / ns_kernels.cuh):
//
//   R = -(1/J) [D_xi F~ + D_eta G~ + g'(xi) dF_1,3 + g'(eta) dF_0,2]
//   dF = s_e Fc(U_L, U_R) - sgn ext(F~ or G~)          (per flux point)
//
// With a = -L/J at the solution points:
//   k_adj_dfbar   dFbar at every flux point = the g' row sums of a along the
//                 point's line (the transposed correction), stored per point;
//   k_adj_euler   F~bar = D_xi^T a - sgn ext^T(dFbar_own), G~bar likewise,
//                 Fbar = J (xi_x F~bar + eta_x G~bar), ..., then
//                 (dF/dU)^T Fbar + (dG/dU)^T Gbar at the solution points; at
//                 the flux points the face's common-flux adjoint
//                 s_e (dFbar_own - dFbar_neighbour) (both elements of a face
//                 use the same Fc, with opposite s_e), transposed through the
//                 Riemann solver and the ghost state into the own trace
//                 adjoint, which L^T carries back to the solution points.
// Navier-Stokes adds the viscous flux at the solution points and faces and the
// corrected gradient Q(U): k_adj_ns runs the steps above plus the transposed
// viscous flux, the gradient traces' L^T, the metric chain rule and D^T, and
// writes the adjoint of the gradient's face jumps dU_e = (U_nbr - U_own)/2;
// k_adj_ns_gather adds the neighbour's share of those jumps to the trace
// adjoint and applies L^T.
//
// Every pass is element-centric: each element gathers what its neighbours
// wrote in the previous pass, nothing is scattered, no atomics.
#include <cuda_runtime.h>

#include "ns_kernels.cuh"
#include "zj_adjoint.cuh"

#ifndef ZJ_ADJ_MIN_BLOCKS
#define ZJ_ADJ_MIN_BLOCKS 3       // Navier-Stokes adjoint kernel (168 registers)
#endif

namespace zj {
namespace {

using namespace dev;

__device__ __forceinline__ long long nbr_row(const EdgeRec& r, long long n_elem) {
    return (r.flags & kEdgeBoundary) ? n_elem * 4 + r.nbr_edge : (long long)r.nbr * 4 + r.nbr_edge;
}

// a = -L/J of one solution point into the [var][row][col] tile.
template <int RS, int VS>
__device__ __forceinline__ void store_a(const AdjArgs& a, long long idx, int i, int j, double* sA) {
    double l[4];
    gload4(a.L + idx * 4, l);
    const double iJ = rcp_any(__ldg(a.J + idx));
#pragma unroll
    for (int v = 0; v < 4; ++v) sA[v * VS + j * RS + i] = -l[v] * iJ;
}

// Transposed divergence and extrapolation at solution point (i, j):
// F~bar = D_xi^T a - Lp(xi_i) dFbar_1[j] + Lm(xi_i) dFbar_3[n1-1-j],
// G~bar = D_eta^T a - Lp(eta_j) dFbar_2[n1-1-i] + Lm(eta_j) dFbar_0[i].
template <int N1, int RS, int VS>
__device__ __forceinline__ void transposed_divergence(const double* sA, const double* sDF,
                                                      const double* ops, int i, int j,
                                                      double* Ftb, double* Gtb) {
    const double* Lm = ops + N1 * N1;
    const double* Lp = Lm + N1;
    double f1[4], f3[4], f2[4], f0[4];
    load4(sDF + (1 * N1 + j) * 4, f1);
    load4(sDF + (3 * N1 + (N1 - 1 - j)) * 4, f3);
    load4(sDF + (2 * N1 + (N1 - 1 - i)) * 4, f2);
    load4(sDF + (0 * N1 + i) * 4, f0);
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        double fx = 0.0, gy = 0.0;
#pragma unroll
        for (int m = 0; m < N1; ++m) {
            fx = fma(ops[m * N1 + i], sA[v * VS + j * RS + m], fx);
            gy = fma(ops[m * N1 + j], sA[v * VS + m * RS + i], gy);
        }
        Ftb[v] = fx - Lp[i] * f1[v] + Lm[i] * f3[v];
        Gtb[v] = gy - Lp[j] * f2[v] + Lm[j] * f0[v];
    }
}

// L^T of the four edges' trace adjoints at solution point (i, j), added to
// out: W values per flux point, flux point k at sT + k * stride.
template <int N1, int W>
__device__ __forceinline__ void transposed_traces(const double* sT, int stride, const double* ops,
                                                  int i, int j, double* out) {
    const double* Lm = ops + N1 * N1;
    const double* Lp = Lm + N1;
    const double* t1 = sT + (1 * N1 + j) * stride;
    const double* t3 = sT + (3 * N1 + (N1 - 1 - j)) * stride;
    const double* t2 = sT + (2 * N1 + (N1 - 1 - i)) * stride;
    const double* t0 = sT + (0 * N1 + i) * stride;
#pragma unroll
    for (int v = 0; v < W; ++v)
        out[v] += Lp[i] * t1[v] + Lm[i] * t3[v] + Lp[j] * t2[v] + Lm[j] * t0[v];
}

// Final value of one solution point: W itself, or the fused stage update.
__device__ __forceinline__ void store_result(const AdjArgs& a, long long idx, const double* w) {
    if (!a.out) {
        gstore4(a.W + idx * 4, w);
        return;
    }
    double r[4], x[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) r[v] = a.cw * w[v];
    if (a.X0) { gload4(a.X0 + idx * 4, x); for (int v = 0; v < 4; ++v) r[v] = fma(a.c0, x[v], r[v]); }
    if (a.X1) { gload4(a.X1 + idx * 4, x); for (int v = 0; v < 4; ++v) r[v] = fma(a.c1, x[v], r[v]); }
    if (a.X2) { gload4(a.X2 + idx * 4, x); for (int v = 0; v < 4; ++v) r[v] = fma(a.c2, x[v], r[v]); }
    gstore4(a.out + idx * 4, r);
}

// ---------------------------------------------------------------- pass A --
template <int P>
__global__ void __launch_bounds__(Shape<P>::THREADS)
k_adj_dfbar(const AdjArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS;
    __shared__ double sW[2 * N1];            // -gL, gR
    __shared__ __align__(16) double sA[EB * FS];
    const int tid = threadIdx.x;
    if (tid < N1) sW[tid] = -a.ops[N1 * N1 + 2 * N1 + tid];
    else if (tid < 2 * N1) sW[tid] = a.ops[N1 * N1 + 3 * N1 + tid - N1];
    pdl_launch_dependents();
    pdl_wait();   // the adjoint input comes from the previous launches
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    if (valid && k < NSP) store_a<RS, VS>(a, e * NSP + k, k % N1, k / N1, sA + el * FS);
    __syncthreads();
    if (valid && k < NFT) {
        const int edge = k / N1, fp = k - edge * N1;
        double t[4];
        trace_point<N1, RS, VS>(sA + el * FS, sW, sW + N1, edge, fp, t);
        gstore4(a.Db + (e * NFT + k) * 4, t);
    }
}

// ---------------------------------------------------------- pass B, Euler --
template <int P, int RIEM>
__global__ void __launch_bounds__(Shape<P>::THREADS)
k_adj_euler(const AdjArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS, DS = S::DS;
    __shared__ double sOps[S::NOPS];
    __shared__ __align__(16) double sA[EB * FS];
    __shared__ __align__(16) double sDF[EB * DS];
    __shared__ __align__(16) double sTb[EB * DS];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // states, traces and adjoints come from the previous launches
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;
    const double g = a.gamma;

    EdgeRec r{-1, 0, kEdgeOrphan, 0};
    double nx = 0.0, ny = 0.0, len = 0.0, qo[4], qn[4], dfn[4] = {0.0, 0.0, 0.0, 0.0};
    if (is_fp) {
        r = a.edges[e * 4 + edge];
        double n[3];
        load_normal(a.enrm + e * 4 + edge, n);
        nx = n[0]; ny = n[1]; len = n[2];
        gload4(a.T + (e * NFT + k) * 4, qo);
        double df[4];
        gload4(a.Db + (e * NFT + k) * 4, df);
        store4(sDF + el * DS + k * 4, df);
        if (!(r.flags & kEdgeOrphan)) gload4(a.T + (nbr_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
        if (!(r.flags & (kEdgeOrphan | kEdgeBoundary)))
            gload4(a.Db + (((long long)r.nbr * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, dfn);
    }
    double u[4], ji[4], Jd = 1.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        gload4(a.U + idx * 4, u);
        gload4(a.Jinv + idx * 4, ji);
        Jd = __ldg(a.J + idx);
        store_a<RS, VS>(a, idx, i, j, sA + el * FS);
    }
    __syncthreads();

    double ub[4] = {0.0, 0.0, 0.0, 0.0};
    if (is_sp) {
        double Ftb[4], Gtb[4], Fb[4], Gb[4];
        transposed_divergence<N1, RS, VS>(sA + el * FS, sDF + el * DS, sOps, i, j, Ftb, Gtb);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Fb[v] = Jd * (ji[0] * Ftb[v] + ji[2] * Gtb[v]);
            Gb[v] = Jd * (ji[1] * Ftb[v] + ji[3] * Gtb[v]);
        }
        adj::euler_flux_vjp(u, g, Fb, Gb, ub);
    }
    if (is_fp) {
        double tb[4] = {0.0, 0.0, 0.0, 0.0};
        if (!(r.flags & kEdgeOrphan)) {
            const bool right = (r.flags & kEdgeRight) != 0;
            const double ss = right ? -0.5 * len : 0.5 * len;
            double Fcb[4], ULb[4] = {0.0, 0.0, 0.0, 0.0}, URb[4] = {0.0, 0.0, 0.0, 0.0};
            const double* df = sDF + el * DS + k * 4;
#pragma unroll
            for (int v = 0; v < 4; ++v) Fcb[v] = ss * (df[v] - dfn[v]);
            adj::riemann_vjp<RIEM>(right ? qn : qo, right ? qo : qn, nx, ny, g, Fcb, ULb, URb);
#pragma unroll
            for (int v = 0; v < 4; ++v) tb[v] = right ? URb[v] : ULb[v];
            if (r.flags & kEdgeBoundary)
                adj::ghost_vjp(qo, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, g,
                               URb, tb);
        }
        store4(sTb + el * DS + k * 4, tb);
    }
    __syncthreads();
    if (is_sp) {
        transposed_traces<N1, 4>(sTb + el * DS, 4, sOps, i, j, ub);
        store_result(a, e * NSP + k, ub);
    }
}

// ---------------------------------------------------- pass B, Navier-Stokes --
template <int P, int RIEM>
__global__ void __launch_bounds__(Shape<P, 2>::THREADS, ZJ_ADJ_MIN_BLOCKS * kCtaScale)
k_adj_ns(const AdjArgs a) {
    using S = Shape<P, 2>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS, DS = S::DS;
    __shared__ double sOps[S::NOPS];
    __shared__ __align__(16) double sA[EB * FS];      // a, then dxi-bar
    __shared__ __align__(16) double sU[EB * FS];      // stage state, then deta-bar
    __shared__ __align__(16) double sD[EB * DS];      // face jumps of U
    __shared__ __align__(16) double sDF[EB * DS];     // own dFbar
    __shared__ __align__(16) double sTQ[EB * 2 * DS]; // own gradient-trace adjoint
    __shared__ double sRed[32];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // states, traces and adjoints come from the previous launches
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;
    const double g = a.gamma, Re = a.Re, Pr = a.Pr;

    // ---- 1: loads
    EdgeRec r{-1, 0, kEdgeOrphan, 0};
    double nx = 0.0, ny = 0.0, len = 0.0, qo[4], qn[4], dfn[4] = {0.0, 0.0, 0.0, 0.0};
    double Qo[8], Qn[8];
    if (is_fp) {
        r = a.edges[e * 4 + edge];
        double n[3];
        load_normal(a.enrm + e * 4 + edge, n);
        nx = n[0]; ny = n[1]; len = n[2];
        gload4(a.T + (e * NFT + k) * 4, qo);
#pragma unroll
        for (int v = 0; v < 4; ++v) qn[v] = qo[v];
        double df[4];
        gload4(a.Db + (e * NFT + k) * 4, df);
        store4(sDF + el * DS + k * 4, df);
        const double* qt = a.TQ + (e * NFT + k) * 8;
        gload4(qt, Qo);
        gload4(qt + 4, Qo + 4);
#pragma unroll
        for (int v = 0; v < 8; ++v) Qn[v] = Qo[v];
        if (!(r.flags & kEdgeOrphan)) gload4(a.T + (nbr_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
        if (!(r.flags & (kEdgeOrphan | kEdgeBoundary))) {
            const long long nrow = ((long long)r.nbr * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp);
            gload4(a.Db + nrow * 4, dfn);
            gload4(a.TQ + nrow * 8, Qn);
            gload4(a.TQ + nrow * 8 + 4, Qn + 4);
        }
        double d[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) d[v] = (r.flags & kEdgeOrphan) ? 0.0 : 0.5 * (qn[v] - qo[v]);
        store4(sD + el * DS + k * 4, d);
    }
    double u[4], ji[4], Jd = 1.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        gload4(a.U + idx * 4, u);
        gload4(a.Jinv + idx * 4, ji);
        Jd = __ldg(a.J + idx);
        store_a<RS, VS>(a, idx, i, j, sA + el * FS);
#pragma unroll
        for (int v = 0; v < 4; ++v) sU[el * FS + v * VS + j * RS + i] = u[v];
    }
    __syncthreads();

    // ---- 2: transposed fluxes at the solution points; face adjoints
    double re_acc = 0.0;     // L . dR/dRe of this thread's viscous fluxes
    double ub[4] = {0.0, 0.0, 0.0, 0.0}, Qxb[4] = {0.0, 0.0, 0.0, 0.0}, Qyb[4] = {0.0, 0.0, 0.0, 0.0};
    if (is_sp) {
        double Qx[4], Qy[4];
        corrected_gradient<N1, RS, VS>(sU + el * FS, sD + el * DS, sOps, i, j, ji, Qx, Qy);
        double Ftb[4], Gtb[4], Fb[4], Gb[4], mFb[4], mGb[4];
        transposed_divergence<N1, RS, VS>(sA + el * FS, sDF + el * DS, sOps, i, j, Ftb, Gtb);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Fb[v] = Jd * (ji[0] * Ftb[v] + ji[2] * Gtb[v]);
            Gb[v] = Jd * (ji[1] * Ftb[v] + ji[3] * Gtb[v]);
            mFb[v] = -Fb[v];
            mGb[v] = -Gb[v];
        }
        adj::euler_flux_vjp(u, g, Fb, Gb, ub);
        re_acc -= adj::viscous_vjp(u, Qx, Qy, g, Re, Pr, mFb, mGb, ub, Qxb, Qyb) / Re;
    }
    double tb[4] = {0.0, 0.0, 0.0, 0.0};
    if (is_fp) {
        double tq[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (!(r.flags & kEdgeOrphan)) {
            const bool right = (r.flags & kEdgeRight) != 0;
            const bool bnd = (r.flags & kEdgeBoundary) != 0;
            const double ss = right ? -0.5 * len : 0.5 * len;
            double Fcb[4], ULb[4] = {0.0, 0.0, 0.0, 0.0}, URb[4] = {0.0, 0.0, 0.0, 0.0};
            const double* df = sDF + el * DS + k * 4;
#pragma unroll
            for (int v = 0; v < 4; ++v) Fcb[v] = ss * (df[v] - dfn[v]);
            const double* UL = right ? qn : qo;
            const double* UR = right ? qo : qn;
            adj::riemann_vjp<RIEM>(UL, UR, nx, ny, g, Fcb, ULb, URb);
            // common viscous flux F_v(avg U, avg Q).n enters with a minus sign
            // (through the walls' closure, a symmetric projection)
            double Ua[4], dxa[4], dya[4], Fvb[4], Gvb[4], Fnb[4];
            double Uab[4] = {0.0, 0.0, 0.0, 0.0}, dxb[4] = {0.0, 0.0, 0.0, 0.0}, dyb[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int v = 0; v < 4; ++v) Fnb[v] = Fcb[v];
            boundary_viscous_closure(r, a.bc, nx, ny, Fnb);
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Ua[v] = 0.5 * (UL[v] + UR[v]);
                dxa[v] = 0.5 * (Qo[v] + Qn[v]);
                dya[v] = 0.5 * (Qo[4 + v] + Qn[4 + v]);
                Fvb[v] = -Fnb[v] * nx;
                Gvb[v] = -Fnb[v] * ny;
            }
            const double dv = adj::viscous_vjp(Ua, dxa, dya, g, Re, Pr, Fvb, Gvb, Uab, dxb, dyb);
            if (!right) re_acc -= dv / Re;   // once per face: on its left element
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                ULb[v] += 0.5 * Uab[v];
                URb[v] += 0.5 * Uab[v];
                // own gradient trace: half of the average, all of it on a
                // boundary (the ghost gradient is the interior one)
                tq[v] = (bnd ? 1.0 : 0.5) * dxb[v];
                tq[4 + v] = (bnd ? 1.0 : 0.5) * dyb[v];
                tb[v] = right ? URb[v] : ULb[v];
            }
            if (bnd)
                adj::ghost_vjp(qo, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, g,
                               URb, tb);
        }
        store4(sTQ + el * 2 * DS + k * 8, tq);
        store4(sTQ + el * 2 * DS + k * 8 + 4, tq + 4);
    }
    if (a.re_part) {
        const double bs = block_sum(re_acc, sRed);
        if (tid == 0) a.re_part[blockIdx.x] = bs;
    }
    __syncthreads();   // sA, sU, sD free from here

    // ---- 3: gradient adjoint at the solution points (sA, sU reused)
    if (is_sp) {
        transposed_traces<N1, 4>(sTQ + el * 2 * DS, 8, sOps, i, j, Qxb);
        transposed_traces<N1, 4>(sTQ + el * 2 * DS + 4, 8, sOps, i, j, Qyb);
        double* dxi = sA + el * FS;
        double* deta = sU + el * FS;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            dxi[v * VS + j * RS + i] = ji[0] * Qxb[v] + ji[1] * Qyb[v];
            deta[v * VS + j * RS + i] = ji[2] * Qxb[v] + ji[3] * Qyb[v];
        }
    }
    __syncthreads();

    // ---- 4: D^T of the gradient; adjoint of the gradient's face jumps
    if (is_sp) {
        const double* dxi = sA + el * FS;
        const double* deta = sU + el * FS;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            double acc = 0.0;
#pragma unroll
            for (int m = 0; m < N1; ++m) {
                acc = fma(sOps[m * N1 + i], dxi[v * VS + j * RS + m], acc);
                acc = fma(sOps[m * N1 + j], deta[v * VS + m * RS + i], acc);
            }
            ub[v] += acc;
        }
        gstore4(a.W + (e * NSP + k) * 4, ub);
    }
    if (is_fp) {
        const double* gL = sOps + N1 * N1 + 2 * N1;
        const double* gR = gL + N1;
        const bool along_eta = (edge == 0 || edge == 2);
        double dub[4];
        trace_point<N1, RS, VS>((along_eta ? sU : sA) + el * FS, gL, gR, edge, fp, dub);
        if (r.flags & kEdgeOrphan) {
#pragma unroll
            for (int v = 0; v < 4; ++v) dub[v] = 0.0;
        }
        // dU_e = (U_nbr - U_own)/2 with U_nbr the neighbour's trace or the
        // ghost state of the own trace
#pragma unroll
        for (int v = 0; v < 4; ++v) tb[v] -= 0.5 * dub[v];
        if (r.flags & kEdgeBoundary) {
            double hb[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) hb[v] = 0.5 * dub[v];
            adj::ghost_vjp(qo, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, g,
                           hb, tb);
        }
        gstore4(a.Tb + (e * NFT + k) * 4, tb);
        gstore4(a.DUb + (e * NFT + k) * 4, dub);
    }
}

// ------------------------------------------------- pass C, Navier-Stokes --
template <int P>
__global__ void __launch_bounds__(Shape<P>::THREADS)
k_adj_ns_gather(const AdjArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int DS = S::DS;
    __shared__ double sOps[S::NOPS];
    __shared__ __align__(16) double sTb[EB * DS];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // states, traces and adjoints come from the previous launches
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    if (valid && k < NFT) {
        const int edge = k / N1, fp = k - edge * N1;
        double tb[4];
        gload4(a.Tb + (e * NFT + k) * 4, tb);
        const EdgeRec r = a.edges[e * 4 + edge];
        if (!(r.flags & (kEdgeOrphan | kEdgeBoundary))) {
            double dn[4];
            gload4(a.DUb + (((long long)r.nbr * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, dn);
#pragma unroll
            for (int v = 0; v < 4; ++v) tb[v] += 0.5 * dn[v];
        }
        store4(sTb + el * DS + k * 4, tb);
    }
    __syncthreads();
    if (valid && k < NSP) {
        double w[4];
        gload4(a.W + (e * NSP + k) * 4, w);
        transposed_traces<N1, 4>(sTb + el * DS, 4, sOps, k % N1, k / N1, w);
        store_result(a, e * NSP + k, w);
    }
}

template <int P>
cudaError_t dfbar_t(const AdjArgs& a, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    return launch_programmatic(k_adj_dfbar<P>, (unsigned)grid, S::THREADS, s, a);
}

template <int P, int RIEM>
cudaError_t euler_t(const AdjArgs& a, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    return launch_programmatic(k_adj_euler<P, RIEM>, (unsigned)grid, S::THREADS, s, a);
}

template <int P, int RIEM>
cudaError_t ns_t(const AdjArgs& a, cudaStream_t s) {
    using S = Shape<P, 2>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    cudaError_t e = launch_programmatic(k_adj_ns<P, RIEM>, (unsigned)grid, S::THREADS, s, a);
    if (e != cudaSuccess) return e;
    using S1 = Shape<P>;
    const long long g1 = (a.n_elem + S1::EB - 1) / S1::EB;
    return launch_programmatic(k_adj_ns_gather<P>, (unsigned)g1, S1::THREADS, s, a);
}

template <int P>
cudaError_t adj_p(int riemann, bool viscous, const AdjArgs& a, cudaStream_t s) {
    cudaError_t e = dfbar_t<P>(a, s);
    if (e != cudaSuccess) return e;
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV:
            return viscous ? ns_t<P, ZJ_RIEMANN_RUSANOV>(a, s) : euler_t<P, ZJ_RIEMANN_RUSANOV>(a, s);
        case ZJ_RIEMANN_ROE:
            return viscous ? ns_t<P, ZJ_RIEMANN_ROE>(a, s) : euler_t<P, ZJ_RIEMANN_ROE>(a, s);
        case ZJ_RIEMANN_HLLC:
            return viscous ? ns_t<P, ZJ_RIEMANN_HLLC>(a, s) : euler_t<P, ZJ_RIEMANN_HLLC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

int adj_ns_grid(int P, long long n_elem) {
    int eb = 1;
    switch (P) {
        case 1: eb = Shape<1, 2>::EB; break;
        case 2: eb = Shape<2, 2>::EB; break;
        case 3: eb = Shape<3, 2>::EB; break;
        case 4: eb = Shape<4, 2>::EB; break;
        case 5: eb = Shape<5, 2>::EB; break;
        default: return 0;
    }
    return (int)((n_elem + eb - 1) / eb);
}

cudaError_t launch_rhs_vjp(int P, int riemann, bool viscous, const AdjArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return adj_p<1>(riemann, viscous, a, s);
        case 2: return adj_p<2>(riemann, viscous, a, s);
        case 3: return adj_p<3>(riemann, viscous, a, s);
        case 4: return adj_p<4>(riemann, viscous, a, s);
        case 5: return adj_p<5>(riemann, viscous, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zj
