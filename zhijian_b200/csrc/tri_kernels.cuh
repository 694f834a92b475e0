// tri_kernels.cuh -- residual / SSP-RK3 stage kernels of straight-sided
// triangles (physics mode), Euler and Navier-Stokes, templated on the
// arithmetic type like the quad kernels (double: FP64; float: the
// mixed-precision form with the per-element reference state).
//
// A triangle holds nt = (P+1)(P+2)/2 solution points in the first nt of its
// (P+1)^2 state slots and 3 (P+1) flux points in edges 0..2 of its trace rows
// (the layout the quads use, so faces between triangles and quads need no
// special case).  With the operators of tri_setup.cpp:
//   R_n = -(1/J) [ sum_k Dr_nk F~_k + Ds_nk G~_k + sum_q Phi_nq dF_q ],
//   dF_q = s_f F_common . n - (sum_k L_qk F~_k, sum_k L_qk G~_k) . n^_f,
// s_f = |edge| / |reference edge| (2, 2 sqrt 2, 2), n^_f the reference edge's
// unit outward normal.  Navier-Stokes: the corrected gradient
//   dU/dr = sum_k Dr_nk U_k + sum_q Phi_nq n^x_q dU_q,
//   dU/ds = sum_k Ds_nk U_k + sum_q Phi_nq n^y_q dU_q,  dU_q = (U_nbr - U_own)/2,
// chain rule with the constant metrics, and the quads' viscous law and
// common viscous flux.  The kernels visit the triangles through an element
// list; phases as the quad kernels (loads and fluxes, faces, divergence +
// correction + stage, traces and ghost rows).
#pragma once

#include "ns_kernels.cuh"

#ifndef ZJ_TRI_MIN_BLOCKS
#define ZJ_TRI_MIN_BLOCKS 2       // FP64 stage kernel (128 registers; viscous: spills of 16-36 B)
#endif
#ifndef ZJ_TRI32_MIN_BLOCKS
#define ZJ_TRI32_MIN_BLOCKS 3     // precision-form stage kernel (80 registers)
#endif

namespace zj {
namespace {

template <typename T> struct TriMinBlocks { static constexpr int stage = ZJ_TRI_MIN_BLOCKS; };
template <> struct TriMinBlocks<float> { static constexpr int stage = ZJ_TRI32_MIN_BLOCKS; };

template <int P, typename T>
struct TriShape {
    static constexpr int N1 = P + 1;
    static constexpr int NT = (P + 1) * (P + 2) / 2;   // solution points
    static constexpr int NSP = N1 * N1;                // state slots per element
    static constexpr int NFT = 3 * N1;                 // flux points
    static constexpr int TPE = NT > NFT ? NT : NFT;
    static constexpr int EB = (256 / TPE / EbDiv<T>::value) > 0 ? (256 / TPE / EbDiv<T>::value) : 1;
    static constexpr int THREADS = EB * TPE;
    static constexpr int NOPS = 2 * NT * NT + 2 * NT * NFT;   // Dr, Ds, L, Phi
    static constexpr int FS = NT + ((NT & 1) ? 1 : 0);        // one variable's field
    static constexpr int ES = 4 * FS + 2;                     // element stride of a 4-variable field
    static constexpr int DS = 4 * NFT + (sizeof(T) == 8 ? 2 : 4);
};

// reference-edge unit outward normals and lengths
__device__ __forceinline__ double tri_nref_x(int f) { return f == 1 ? 0.70710678118654752440 : (f == 2 ? -1.0 : 0.0); }
__device__ __forceinline__ double tri_nref_y(int f) { return f == 0 ? -1.0 : (f == 1 ? 0.70710678118654752440 : 0.0); }
__device__ __forceinline__ double tri_ref_len(int f) { return f == 1 ? 2.82842712474619009760 : 2.0; }

// Interpolation of a [var][NT] field (stride FS) to flux point q.
template <int NT, int FS, typename T>
__device__ __forceinline__ void tri_interp(const T* fld, const T* Lrow, T* out) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        T t = T(0);
#pragma unroll
        for (int k = 0; k < NT; ++k) t = fma_any(Lrow[k], fld[v * FS + k], t);
        out[v] = t;
    }
}

// Corrected reference gradient at solution point n from the state field su
// ([var][NT]) and the face jumps du ([q][var]).
template <int NT, int NFT, int FS, typename T>
__device__ __forceinline__ void tri_gradient(const T* su, const T* du, const T* Dr, const T* Ds,
                                             const T* Phi, int n, const T* ji, T* Qx, T* Qy) {
    T dr[4] = {T(0), T(0), T(0), T(0)}, ds[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
    for (int k = 0; k < NT; ++k) {
        const T a = Dr[n * NT + k], b = Ds[n * NT + k];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            dr[v] = fma_any(a, su[v * FS + k], dr[v]);
            ds[v] = fma_any(b, su[v * FS + k], ds[v]);
        }
    }
#pragma unroll
    for (int q = 0; q < NFT; ++q) {
        const int f = q / (NFT / 3);
        const T ph = Phi[n * NFT + q];
        const T px = ph * T(tri_nref_x(f)), py = ph * T(tri_nref_y(f));
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            dr[v] = fma_any(px, du[q * 4 + v], dr[v]);
            ds[v] = fma_any(py, du[q * 4 + v], ds[v]);
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        Qx[v] = ji[0] * dr[v] + ji[2] * ds[v];
        Qy[v] = ji[1] * dr[v] + ji[3] * ds[v];
    }
}

template <int P, typename T>
struct TriLayout {
    using S = TriShape<P, T>;
    // offsets in the operator tile
    static constexpr int DR = 0, DSo = S::NT * S::NT, L = 2 * S::NT * S::NT, PHI = L + S::NFT * S::NT;
};

// Element of thread group el in this CTA, or -1.
__device__ __forceinline__ long long tri_element(const int32_t* elist, long long n_list, int EB, int el) {
    const long long g = (long long)blockIdx.x * EB + el;
    return (g < n_list) ? (long long)elist[g] : -1;
}

// ---------------------------------------------------------------- traces --
template <int P, typename T>
__global__ void __launch_bounds__(TriShape<P, T>::THREADS)
k_tri_traces(const StageArgsT<T> a, const int32_t* __restrict__ elist, long long n_list) {
    using S = TriShape<P, T>;
    using Lo = TriLayout<P, T>;
    constexpr int N1 = S::N1, NT = S::NT, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int FS = S::FS, ES = S::ES;
    __shared__ T sOps[S::NOPS];
    __shared__ __align__(16) T sU[EB * ES];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (el < EB) ? tri_element(elist, n_list, EB, el) : -1;
    const bool valid = e >= 0;
    constexpr bool kRef = UsesRef<T>::value;
    T ue[4] = {T(0), T(0), T(0), T(0)};
    if (kRef && valid) load_state(a.U + e * NSP * 4, ue);
    if (valid && k < NT) {
        double u[4];
        T w[4];
        stage_state(a, e * NSP + k, u, w);
        if constexpr (kRef) state_minus_ref(u, ue, w);
#pragma unroll
        for (int v = 0; v < 4; ++v) sU[el * ES + v * FS + k] = w[v];
    }
    __syncthreads();
    if (valid && k < NFT) {
        const int edge = k / N1, fp = k - edge * N1;
        T t[4];
        tri_interp<NT, FS>(sU + el * ES, sOps + Lo::L + k * NT, t);
        if constexpr (kRef) {
#pragma unroll
            for (int v = 0; v < 4; ++v) t[v] += ue[v];
        }
        gstore4(a.Tout + (e * 4 * N1 + k) * 4, t);
        const EdgeRec r = a.edges[e * 4 + edge];
        if (r.flags & kEdgeBoundary) {
            T n[3];
            load_normal(a.enrm + e * 4 + edge, n);
            store_ghost<N1>(a, r, n[0], n[1], fp, t);
        }
    }
}

// ------------------------------------------------------- gradient (NS) --
template <int P, typename T>
__global__ void __launch_bounds__(TriShape<P, T>::THREADS)
k_tri_grad(const StageArgsT<T> a, const int32_t* __restrict__ elist, long long n_list) {
    using S = TriShape<P, T>;
    using Lo = TriLayout<P, T>;
    constexpr int N1 = S::N1, NT = S::NT, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int FS = S::FS, ES = S::ES, DS = S::DS;
    __shared__ T sOps[S::NOPS];
    __shared__ __align__(16) T sU[EB * ES];
    __shared__ __align__(16) T sDU[EB * DS];
    __shared__ __align__(16) T sQ[EB * 2 * ES];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous launches
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (el < EB) ? tri_element(elist, n_list, EB, el) : -1;
    const bool valid = e >= 0;
    const bool is_sp = valid && k < NT, is_fp = valid && k < NFT;
    const int edge = k / N1, fp = k - edge * N1;
    constexpr bool kRef = UsesRef<T>::value;
    T ji[4];
    if (is_sp) {
        const long long idx = e * NSP + k;
        double ud[4];
        T u[4];
        stage_state(a, idx, ud, u);
        if constexpr (kRef) {
            T ue[4];
            load_state(a.U + e * NSP * 4, ue);
            state_minus_ref(ud, ue, u);
        }
        load4_nc(a.Jinv + idx * 4, ji);
#pragma unroll
        for (int v = 0; v < 4; ++v) sU[el * ES + v * FS + k] = u[v];
    }
    if (is_fp) {
        const EdgeRec r = a.edges[e * 4 + edge];
        T qo[4], qn[4];
        load4_nc(a.Tin + (e * 4 * N1 + k) * 4, qo);
        T d[4] = {T(0), T(0), T(0), T(0)};
        if (!(r.flags & kEdgeOrphan)) {
            load4_nc(a.Tin + (neighbour_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
#pragma unroll
            for (int v = 0; v < 4; ++v) d[v] = T(0.5) * (qn[v] - qo[v]);
        }
        store4(sDU + el * DS + k * 4, d);
    }
    __syncthreads();
    if (is_sp) {
        T Qx[4], Qy[4];
        tri_gradient<NT, NFT, FS>(sU + el * ES, sDU + el * DS, sOps + Lo::DR, sOps + Lo::DSo, sOps + Lo::PHI, k,
                                  ji, Qx, Qy);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            sQ[el * 2 * ES + v * FS + k] = Qx[v];
            sQ[el * 2 * ES + ES + v * FS + k] = Qy[v];
        }
    }
    __syncthreads();
    if (is_fp) {
        T t[8];
        tri_interp<NT, FS>(sQ + el * 2 * ES, sOps + Lo::L + k * NT, t);
        tri_interp<NT, FS>(sQ + el * 2 * ES + ES, sOps + Lo::L + k * NT, t + 4);
        T* o = a.TQout + (e * 4 * N1 + k) * 8;
        gstore8(o, t);
    }
}

// ----------------------------------------------------------------- stage --
template <int P, int RIEM, bool VISC, typename T>
__global__ void __launch_bounds__(TriShape<P, T>::THREADS, TriMinBlocks<T>::stage)
k_tri_stage(const StageArgsT<T> a, const int32_t* __restrict__ elist, long long n_list) {
    using S = TriShape<P, T>;
    using Lo = TriLayout<P, T>;
    constexpr int N1 = S::N1, NT = S::NT, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int FS = S::FS, ES = S::ES, DS = S::DS;
    __shared__ T sOps[S::NOPS];
    __shared__ __align__(16) T sF[EB * ES];
    __shared__ __align__(16) T sG[EB * ES];
    __shared__ __align__(16) T sD[EB * DS];    // face jumps of U (NS), then flux differences
    __shared__ __align__(16) T sU[EB * ES];    // stage state (NS), then the new state
    __shared__ double sRed[32];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous launches
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (el < EB) ? tri_element(elist, n_list, EB, el) : -1;
    const bool valid = e >= 0;
    const bool is_sp = valid && k < NT, is_fp = valid && k < NFT;
    const int edge = k / N1, fp = k - edge * N1;
    const T g = T(a.gamma), Re = reynolds(a), Pr = T(a.Pr);
    constexpr bool kRef = UsesRef<T>::value;

    // ---- A1: loads
    T ue[4] = {T(0), T(0), T(0), T(0)};
    if (kRef && valid) load_state(a.U + e * NSP * 4, ue);
    EdgeRec r{-1, 0, kEdgeOrphan, 0};
    T nr[3] = {T(0), T(0), T(0)}, qo[4], qn[4] = {T(0), T(0), T(0), T(0)};
    T Qo[8], Qn[8];
    if (is_fp) {
        r = a.edges[e * 4 + edge];
        load_normal(a.enrm + e * 4 + edge, nr);
        load4_nc(a.Tin + (e * 4 * N1 + k) * 4, qo);
#pragma unroll
        for (int v = 0; v < 4; ++v) qn[v] = qo[v];
        if (!(r.flags & kEdgeOrphan)) load4_nc(a.Tin + (neighbour_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
        if constexpr (VISC) {
            const T* qt = a.TQ + (e * 4 * N1 + k) * 8;
            gload8_nc(qt, Qo);
#pragma unroll
            for (int v = 0; v < 8; ++v) Qn[v] = Qo[v];
            if (!(r.flags & (kEdgeOrphan | kEdgeBoundary))) {
                const T* q2 = a.TQ + (((long long)r.nbr * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 8;
                gload8_nc(q2, Qn);
            }
            T d[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) d[v] = (r.flags & kEdgeOrphan) ? T(0) : T(0.5) * (qn[v] - qo[v]);
            store4(sD + el * DS + k * 4, d);
        }
    }
    T u[4], ji[4], Jd = T(1);
    if (is_sp) {
        const long long idx = e * NSP + k;
        double ud[4];
        stage_state(a, idx, ud, u);
        load4_nc(a.Jinv + idx * 4, ji);
        Jd = ldg_any(a.J + idx);
        if (a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        if constexpr (VISC) {
            T w[4];
            if constexpr (kRef) state_minus_ref(ud, ue, w);
            else {
#pragma unroll
                for (int v = 0; v < 4; ++v) w[v] = u[v];
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) sU[el * ES + v * FS + k] = w[v];
        }
    }
    if constexpr (VISC) __syncthreads();

    // ---- A2: transformed fluxes
    if (is_sp) {
        T F[4], G[4];
        euler_flux(u, g, F, G);
        if constexpr (kRef) {
            T Fe[4], Ge[4];
            euler_flux(ue, g, Fe, Ge);
#pragma unroll
            for (int v = 0; v < 4; ++v) { F[v] -= Fe[v]; G[v] -= Ge[v]; }
        }
        if constexpr (VISC) {
            T Qx[4], Qy[4], Fv[4], Gv[4];
            tri_gradient<NT, NFT, FS>(sU + el * ES, sD + el * DS, sOps + Lo::DR, sOps + Lo::DSo, sOps + Lo::PHI,
                                      k, ji, Qx, Qy);
            viscous_flux(u, Qx, Qy, g, Re, Pr, Fv, Gv);
#pragma unroll
            for (int v = 0; v < 4; ++v) { F[v] -= Fv[v]; G[v] -= Gv[v]; }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            sF[el * ES + v * FS + k] = Jd * (ji[0] * F[v] + ji[1] * G[v]);
            sG[el * ES + v * FS + k] = Jd * (ji[2] * F[v] + ji[3] * G[v]);
        }
    }
    __syncthreads();

    // ---- B: interface terms
    if (is_fp) {
        T Fd[4] = {T(0), T(0), T(0), T(0)};
        if (!(r.flags & kEdgeOrphan)) {
            const bool right = (r.flags & kEdgeRight) != 0;
            T UL[4], UR[4], Fc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) { UL[v] = right ? qn[v] : qo[v]; UR[v] = right ? qo[v] : qn[v]; }
            riemann<RIEM>(UL, UR, nr[0], nr[1], g, Fc);
            if constexpr (kRef) {
                T Fe[4];
                ref_flux_n(ue, g, nr[0], nr[1], Fe);
#pragma unroll
                for (int v = 0; v < 4; ++v) Fc[v] -= Fe[v];
            }
            if constexpr (VISC) {
                T Ua[4], dxa[4], dya[4], Fv[4], Gv[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) {
                    Ua[v] = T(0.5) * (UL[v] + UR[v]);
                    dxa[v] = T(0.5) * (Qo[v] + Qn[v]);
                    dya[v] = T(0.5) * (Qo[4 + v] + Qn[4 + v]);
                }
                viscous_flux(Ua, dxa, dya, g, Re, Pr, Fv, Gv);
                T Fvn[4];
#pragma unroll
                for (int v = 0; v < 4; ++v) Fvn[v] = Fv[v] * nr[0] + Gv[v] * nr[1];
                boundary_viscous_closure(r, a.bc, nr[0], nr[1], Fvn);
#pragma unroll
                for (int v = 0; v < 4; ++v) Fc[v] -= Fvn[v];
            }
            const T sf = nr[2] * T(1.0 / tri_ref_len(edge));
            const T ss = right ? -sf : sf;
            T fx[4], gy[4];
            tri_interp<NT, FS>(sF + el * ES, sOps + Lo::L + k * NT, fx);
            tri_interp<NT, FS>(sG + el * ES, sOps + Lo::L + k * NT, gy);
            const T nx = T(tri_nref_x(edge)), ny = T(tri_nref_y(edge));
#pragma unroll
            for (int v = 0; v < 4; ++v) Fd[v] = ss * Fc[v] - (fx[v] * nx + gy[v] * ny);
        }
        store4(sD + el * DS + k * 4, Fd);   // (NS: the jumps were consumed in A2)
    }
    __syncthreads();

    // ---- C: divergence, correction, 1/J, stage update
    double rsq = 0.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        double u0[4];
        if (a.stage >= 2) gload4(a.U0 + idx * 4, u0);
        T div[4] = {T(0), T(0), T(0), T(0)};
        const T* Dr = sOps + Lo::DR + k * NT;
        const T* Dsr = sOps + Lo::DSo + k * NT;
#pragma unroll
        for (int m = 0; m < NT; ++m) {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                div[v] = fma_any(Dr[m], sF[el * ES + v * FS + m], div[v]);
                div[v] = fma_any(Dsr[m], sG[el * ES + v * FS + m], div[v]);
            }
        }
        const T* Ph = sOps + Lo::PHI + k * NFT;
#pragma unroll
        for (int q = 0; q < NFT; ++q) {
            T d[4];
            load4(sD + el * DS + q * 4, d);
#pragma unroll
            for (int v = 0; v < 4; ++v) div[v] = fma_any(Ph[q], d[v], div[v]);
        }
        const T iJ = rcp_any(Jd);
        T res[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) res[v] = -div[v] * iJ;
        if (a.stage == 0) {
            store_residual(a, idx, res, rsq);
        } else {
            double us[4];
            gload4(a.U + idx * 4, us);
            double uo[4];
            rk_update(a.stage, *a.dt, us, u0, res, uo);
            gstore4(a.Uout + idx * 4, uo);
            T un[4];
            if constexpr (kRef) state_minus_ref(uo, ue, un);
            else {
#pragma unroll
                for (int v = 0; v < 4; ++v) un[v] = T(uo[v]);
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) sU[el * ES + v * FS + k] = un[v];
            if (a.stage == 3) {
#pragma unroll
                for (int v = 0; v < 4; ++v) rsq += double(res[v]) * double(res[v]);
            }
        }
    }
    if (a.stage == 0 || a.stage == 3) {
        const double bs = block_sum(rsq, sRed);
        if (tid == 0) a.partials[blockIdx.x] = bs;
    }
    if (a.stage == 0) return;
    __syncthreads();

    // ---- D: traces of the new state and ghost rows
    if (is_fp) {
        T t[4];
        tri_interp<NT, FS>(sU + el * ES, sOps + Lo::L + k * NT, t);
        if constexpr (kRef) {
#pragma unroll
            for (int v = 0; v < 4; ++v) t[v] += ue[v];
        }
        gstore4(a.Tout + (e * 4 * N1 + k) * 4, t);
        if (r.flags & kEdgeBoundary) store_ghost<N1>(a, r, nr[0], nr[1], fp, t);
    }
}

template <int P, typename T>
cudaError_t tri_traces_t(const StageArgsT<T>& a, const int32_t* elist, long long n, cudaStream_t s) {
    using S = TriShape<P, T>;
    const long long grid = (n + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    k_tri_traces<P, T><<<(unsigned)grid, S::THREADS, 0, s>>>(a, elist, n);
    return cudaGetLastError();
}

template <int P, typename T>
cudaError_t tri_grad_t(const StageArgsT<T>& a, const int32_t* elist, long long n, cudaStream_t s) {
    using S = TriShape<P, T>;
    const long long grid = (n + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    return launch_programmatic(k_tri_grad<P, T>, (unsigned)grid, S::THREADS, s, a, elist, n);
}

template <int P, int RIEM, bool VISC, typename T>
cudaError_t tri_stage_t(const StageArgsT<T>& a, const int32_t* elist, long long n, cudaStream_t s) {
    using S = TriShape<P, T>;
    const long long grid = (n + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    return launch_programmatic(k_tri_stage<P, RIEM, VISC, T>, (unsigned)grid, S::THREADS, s, a, elist, n);
}

template <int P, bool VISC, typename T>
cudaError_t tri_stage_r(int riemann, const StageArgsT<T>& a, const int32_t* elist, long long n, cudaStream_t s) {
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV: return tri_stage_t<P, ZJ_RIEMANN_RUSANOV, VISC>(a, elist, n, s);
        case ZJ_RIEMANN_ROE: return tri_stage_t<P, ZJ_RIEMANN_ROE, VISC>(a, elist, n, s);
        case ZJ_RIEMANN_HLLC: return tri_stage_t<P, ZJ_RIEMANN_HLLC, VISC>(a, elist, n, s);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t tri_dispatch(int what, int P, int riemann, bool visc, const StageArgsT<T>& a, const int32_t* elist,
                         long long n, cudaStream_t s) {
#define ZJ_TRI_CASE(PP)                                                                        \
    case PP:                                                                                   \
        if (what == 0) return tri_traces_t<PP>(a, elist, n, s);                                \
        if (what == 1) return tri_grad_t<PP>(a, elist, n, s);                                  \
        return visc ? tri_stage_r<PP, true>(riemann, a, elist, n, s)                           \
                    : tri_stage_r<PP, false>(riemann, a, elist, n, s);
    switch (P) {
        ZJ_TRI_CASE(1)
        ZJ_TRI_CASE(2)
        ZJ_TRI_CASE(3)
        ZJ_TRI_CASE(4)
        ZJ_TRI_CASE(5)
        default: return cudaErrorInvalidValue;
    }
#undef ZJ_TRI_CASE
}

template <int P>
int tri_grid_t(long long n) { return (int)((n + TriShape<P, double>::EB - 1) / TriShape<P, double>::EB); }

}  // namespace
}  // namespace zj
