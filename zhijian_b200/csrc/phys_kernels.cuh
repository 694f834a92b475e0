// phys_kernels.cuh -- residual and SSP-RK3 stage kernels of the conservative
// FR scheme the parameters ask for ("physics mode", compat off, inviscid).
// Instantiated for T = double by phys_fp64.cu (the reference-parity path) and
// for T = float by phys_fp32.cu (the mixed-precision form: FP32 fluxes, faces,
// operator products, traces and metrics; FP64 state, RK accumulation and
// norm partials).
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
#pragma once

#include <cuda_runtime.h>

#include "zj_device.cuh"
#include "zj_kernels.h"
#include "zj_math.h"
#include "zj_physics.cuh"

#ifndef ZJ_PHYS_MIN_BLOCKS
#define ZJ_PHYS_MIN_BLOCKS 3      // FP64 stage kernel
#endif
#ifndef ZJ_PHYS32_MIN_BLOCKS
#define ZJ_PHYS32_MIN_BLOCKS 4    // mixed-precision stage kernel
#endif

namespace zj {
namespace {

using namespace dev;
using namespace phys;

// Per-element strides of the shared tiles.  Double tiles (two 4-byte banks
// per value): [var][row][col] fields at 6 mod 16 doubles and the
// [flux point][var] tile at 2 mod 16 (Shape).  Float tiles: every stride a
// multiple of 4 floats (16-byte rows) and congruent mod 32 to the threads per
// element (rounded up to a multiple of 4), so the elements that share a warp
// start on disjoint banks.
template <int P, typename T>
struct Tiles {
    using S = Shape<P, EbDiv<T>::value>;
    static constexpr int pad32(int base) {
        return base + ((((S::TPE + 3) & ~3) % 32) - base % 32 + 64) % 32;
    }
    static constexpr bool kD = sizeof(T) == 8;
    static constexpr int FS = kD ? S::FS : pad32(4 * S::VS);         // one field of 4 vars
    static constexpr int DS = kD ? S::DS : pad32(4 * S::NFT);        // flux-point tile
    static constexpr int QS = kD ? 8 * S::VS + (6 - (8 * S::VS) % 16 + 16) % 16
                                 : pad32(8 * S::VS);                 // gradient field
    static_assert(kD || (FS % 4 == 0 && DS % 4 == 0 && QS % 4 == 0), "16-byte float rows");
};

// Element of thread group el of this CTA: through the element list of a
// mesh with several element kinds, else the CTA's contiguous block.
template <typename T>
__device__ __forceinline__ long long block_element(const StageArgsT<T>& a, int EB, int el, bool& valid) {
    const long long g = (long long)blockIdx.x * EB + el;
    if (a.elist) {
        valid = (el < EB) && (g < a.n_list);
        return valid ? (long long)a.elist[g] : 0;
    }
    valid = (el < EB) && (g < a.n_elem);
    return g;
}

// Normal record of flux point fp on edge `edge` of element e: one per edge on
// straight-sided meshes, one per flux point on curved ones (a.nrm_pp).
template <int N1, typename T>
__device__ __forceinline__ const typename Vec4Of<T>::type* normal_rec(const StageArgsT<T>& a, long long e,
                                                                     int edge, int fp) {
    const long long r = e * 4 + edge;
    return a.enrm + (a.nrm_pp ? r * N1 + fp : r);
}

// Boundary ghost states live in extra rows of every trace buffer, after the
// E*4 element edges: row E*4 + slot of boundary slot `slot`, stored at the
// mirrored point n1-1-fp, so a boundary edge loads its ghost exactly like an
// interior edge loads its neighbour (index (row*n1 + n1-1-fp)).  They are
// written where the trace itself is produced, which keeps the ghost-state
// arithmetic (pow, branches per boundary class) out of the face phases.
__device__ __forceinline__ long long neighbour_row(const EdgeRec& r, long long n_elem) {
    return (r.flags & kEdgeBoundary) ? n_elem * 4 + r.nbr_edge : (long long)r.nbr * 4 + r.nbr_edge;
}

// A boundary edge whose ghost row the traces' kernel writes from its
// boundary condition (a partition's interface rows come from the exchange).
__device__ __forceinline__ bool boundary_condition_edge(const EdgeRec& r) {
    return (r.flags & (kEdgeBoundary | kEdgeInterface)) == kEdgeBoundary;
}
// An edge whose neighbour's gradient trace is read (interior edges and
// partition interfaces; a boundary copies the interior gradient).
__device__ __forceinline__ bool has_neighbour_gradient(const EdgeRec& r) {
    return !(r.flags & kEdgeOrphan) && (!(r.flags & kEdgeBoundary) || (r.flags & kEdgeInterface));
}

template <int N1, typename T>
__device__ __forceinline__ void store_ghost(const StageArgsT<T>& a, const EdgeRec& r, T nx, T ny,
                                            int fp, const T* t) {
    T q[4];
    ghost_phys(t, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, T(a.gamma), q);
    gstore4(a.Tout + ((a.n_elem * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, q);
}

// Conserved state of one solution point in the arithmetic type.
template <typename T>
__device__ __forceinline__ void load_state(const double* p, T* u) {
    double d[4];
    gload4(p, d);
#pragma unroll
    for (int v = 0; v < 4; ++v) u[v] = T(d[v]);
}

// Stage state of one solution point: FP64 copy in ud, arithmetic copy in u
// (with the input tangent for the dual-number instantiation).
template <typename T>
__device__ __forceinline__ void stage_state(const StageArgsT<T>& a, long long idx, double* ud, T* u) {
    gload4(a.U + idx * 4, ud);
    if constexpr (IsDual<T>::value) {
        double t[4];
        gload4(a.dU + idx * 4, t);
#pragma unroll
        for (int v = 0; v < 4; ++v) u[v] = Dual(ud[v], t[v]);
    } else {
#pragma unroll
        for (int v = 0; v < 4; ++v) u[v] = T(ud[v]);
    }
}

// Stage-0 output: the FP64 residual (and its tangent for duals); adds the
// residual's squares to rsq.
template <typename T>
__device__ __forceinline__ void store_residual(const StageArgsT<T>& a, long long idx, const T* res,
                                               double& rsq) {
    double rd[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) { rd[v] = double(res[v]); rsq += rd[v] * rd[v]; }
    gstore4(a.R + idx * 4, rd);
    if constexpr (IsDual<T>::value) {
        double td[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) td[v] = res[v].d;
        gstore4(a.dR + idx * 4, td);
    }
}

template <typename T>
__device__ __forceinline__ T reynolds(const StageArgsT<T>& a) {
    if constexpr (IsDual<T>::value) return Dual(a.Re, a.dRe);
    else return T(a.Re);
}

// 1/Re (with its tangent -dRe/Re^2 for duals) and gamma/((gamma-1) Pr),
// read from the launch arguments where they are used.
template <typename T>
__device__ __forceinline__ T inv_reynolds(const StageArgsT<T>& a) {
    if constexpr (IsDual<T>::value) return Dual(a.iRe, -a.dRe * a.iRe * a.iRe);
    else return T(a.iRe);
}

// SSP-RK3 stage update in FP64 from the stage state us, the base state u0
// and the residual res of the arithmetic type.
template <typename T>
__device__ __forceinline__ void rk_update(int stage, double dt, const double* us, const double* u0,
                                          const T* res, double* uo) {
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double r = double(res[v]);
        if (stage == 1) uo[v] = us[v] + dt * r;
        else if (stage == 2) uo[v] = 0.75 * u0[v] + 0.25 * us[v] + 0.25 * dt * r;
        else uo[v] = (1.0 / 3.0) * u0[v] + (2.0 / 3.0) * us[v] + (2.0 / 3.0) * dt * r;
    }
}

// The mixed-precision form runs its FP32 arithmetic on differences from a
// per-element reference state U_e (the element's first solution point,
// rounded to FP32, so exactly representable): the fluxes enter the operator
// products as F(U) - F(U_e), the states as U - U_e (formed in FP64), traces
// are U_e + L (U - U_e), and the common flux is taken minus F(U_e).n.  In
// exact arithmetic the constant flux F(U_e) contributes nothing to an
// element's residual (metric identity of the straight-sided element, shared
// D/L rows reproducing constants, s_e n = transformed normal on a straight
// edge), so the dropped part is exact; what it removes is the FP32 rounding
// of the weights and metrics multiplied by the large constant part of U and
// F, which is a smooth function of the state and would otherwise accumulate
// step after step.  The FP64 path keeps the plain form.
template <typename T>
struct UsesRef { static constexpr bool value = sizeof(T) == 4; };

template <typename T>
__device__ __forceinline__ void euler_flux(const T* u, T g, T* F, T* G) {
    const T ir = rcp_any(u[0]);
    const T uu = u[1] * ir, vv = u[2] * ir, E = u[3] * ir;
    const T p = (g - T(1)) * u[0] * (E - T(0.5) * (uu * uu + vv * vv));
    F[0] = u[1]; F[1] = u[1] * uu + p; F[2] = u[1] * vv; F[3] = (u[3] + p) * uu;
    G[0] = u[2]; G[1] = u[2] * uu; G[2] = u[2] * vv + p; G[3] = (u[3] + p) * vv;
}

// euler_flux with ir = 1/u[0] supplied (identical arithmetic).
template <typename T>
__device__ __forceinline__ void euler_flux_ir(const T* u, T ir, T g, T* F, T* G) {
    const T uu = u[1] * ir, vv = u[2] * ir, E = u[3] * ir;
    const T p = (g - T(1)) * u[0] * (E - T(0.5) * (uu * uu + vv * vv));
    F[0] = u[1]; F[1] = u[1] * uu + p; F[2] = u[1] * vv; F[3] = (u[3] + p) * uu;
    G[0] = u[2]; G[1] = u[2] * uu; G[2] = u[2] * vv + p; G[3] = (u[3] + p) * vv;
}

// F(U_e).n of a reference state.
template <typename T>
__device__ __forceinline__ void ref_flux_n(const T* ue, T g, T nx, T ny, T* Fn) {
    T F[4], G[4];
    euler_flux(ue, g, F, G);
#pragma unroll
    for (int v = 0; v < 4; ++v) Fn[v] = F[v] * nx + G[v] * ny;
}

// Stage state minus the reference, formed in FP64 and rounded once.
template <typename T>
__device__ __forceinline__ void state_minus_ref(const double* U, const T* ue, T* du) {
#pragma unroll
    for (int v = 0; v < 4; ++v) du[v] = T(U[v] - double(ue[v]));
}

template <typename T> struct PhysMinBlocks;
template <> struct PhysMinBlocks<double> { static constexpr int value = ZJ_PHYS_MIN_BLOCKS * kCtaScale; };
template <> struct PhysMinBlocks<float> { static constexpr int value = ZJ_PHYS32_MIN_BLOCKS * kCtaScale; };
template <> struct PhysMinBlocks<Dual> { static constexpr int value = 1; };

template <int P, int RIEM, typename T>
__global__ void __launch_bounds__(Shape<P, EbDiv<T>::value>::THREADS, PhysMinBlocks<T>::value)
k_phys_stage(const StageArgsT<T> a) {
    using S = Shape<P, EbDiv<T>::value>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = Tiles<P, T>::FS, DS = Tiles<P, T>::DS;
    __shared__ T sOps[S::NOPS];
    __shared__ __align__(16) T sF[EB * FS];
    __shared__ __align__(16) T sG[EB * FS];
    __shared__ __align__(16) T sD[EB * DS];
    __shared__ __align__(16) T sU[EB * FS];
    __shared__ double sRed[32];

    const int tid = threadIdx.x;
    for (int i = tid; i < S::NOPS; i += blockDim.x) sOps[i] = a.ops[i];
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous stage

    const int el = tid / TPE, k = tid - el * TPE;
    bool valid;
    const long long e = block_element(a, EB, el, valid);
    const bool is_sp = valid && k < NSP;
    const bool is_fp = valid && k < NFT;
    const T g = T(a.gamma);
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    // ---- A: loads; transformed fluxes into shared memory
    constexpr bool kRef = UsesRef<T>::value;
    EdgeRec r{-1, 0, kEdgeOrphan, 0};
    T nr[3] = {T(0), T(0), T(0)};
    T qo[4], qn[4] = {T(0), T(0), T(0), T(0)}, u[4], Jd = T(1);
    T ue[4] = {T(0), T(0), T(0), T(0)};   // reference state (mixed form)
    if (kRef && valid) load_state(a.U + e * NSP * 4, ue);
    if (is_fp) {
        r = a.edges[e * 4 + edge];
        load_normal(normal_rec<N1>(a, e, edge, fp), nr);
        load4_nc(a.Tin + (e * NFT + k) * 4, qo);
    }
    if (is_sp) {
        const long long idx = e * NSP + k;
        double ud[4];
        stage_state(a, idx, ud, u);
        T ji[4];
        load4_nc(a.Jinv + idx * 4, ji);
        Jd = ldg_any(a.J + idx);
        if ((k & 3) == 0 && a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        T F[4], G[4];
        euler_flux(u, g, F, G);
        if constexpr (kRef) {
            T Fe[4], Ge[4];
            euler_flux(ue, g, Fe, Ge);
#pragma unroll
            for (int v = 0; v < 4; ++v) { F[v] -= Fe[v]; G[v] -= Ge[v]; }
        }
        T* f = sF + el * FS + j * RS + i;
        T* h = sG + el * FS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            f[v * VS] = Jd * (ji[0] * F[v] + ji[1] * G[v]);
            h[v * VS] = Jd * (ji[2] * F[v] + ji[3] * G[v]);
        }
    }
    // The neighbour's point that coincides with this one: both elements run
    // their shared edge counter-clockwise.
    if (is_fp && !(r.flags & kEdgeOrphan))
        load4_nc(a.Tin + (neighbour_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
    __syncthreads();   // sOps, sF, sG ready

    // ---- B: interface terms.  The common flux is evaluated from the left
    // element's side on both sides of a face (bit-identical on both).
    if (is_fp) {
        T Fd[4] = {T(0), T(0), T(0), T(0)};
        if (!(r.flags & kEdgeOrphan)) {
            const T nx = nr[0], ny = nr[1], s = T(0.5) * nr[2];
            const bool right = (r.flags & kEdgeRight) != 0;
            T UL[4], UR[4], Fc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) { UL[v] = right ? qn[v] : qo[v]; UR[v] = right ? qo[v] : qn[v]; }
            riemann<RIEM>(UL, UR, nx, ny, g, Fc);
            if constexpr (kRef) {
                T Fe[4];
                ref_flux_n(ue, g, nx, ny, Fe);
#pragma unroll
                for (int v = 0; v < 4; ++v) Fc[v] -= Fe[v];
            }
            const T ss = right ? -s : s;
            // Extrapolated transformed flux along this element's outward
            // reference normal: +F~ on edge 1, -F~ on edge 3, -G~ on edge 0,
            // +G~ on edge 2.
            const bool along_eta = (edge == 0 || edge == 2);
            T Fn[4];
            trace_point<N1, RS, VS>((along_eta ? sG : sF) + el * FS, sOps + N1 * N1,
                                    sOps + N1 * N1 + N1, edge, fp, Fn);
            const T sgn = (edge == 0 || edge == 3) ? T(-1) : T(1);
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
        if (a.stage >= 2) gload4(a.U0 + idx * 4, u0);
        T Di[N1], Dj[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) { Di[m] = sOps[i * N1 + m]; Dj[m] = sOps[j * N1 + m]; }
        const T* gL = sOps + N1 * N1 + 2 * N1;
        const T* gR = gL + N1;
        const T gRi = gR[i], gLi = gL[i], gRj = gR[j], gLj = gL[j];
        const T* f = sF + el * FS;
        const T* h = sG + el * FS;
        const T* d = sD + el * DS;
        T c1[4], c3[4], c2[4], c0[4];
        load4(d + (1 * N1 + j) * 4, c1);
        load4(d + (3 * N1 + (N1 - 1 - j)) * 4, c3);
        load4(d + (2 * N1 + (N1 - 1 - i)) * 4, c2);
        load4(d + (0 * N1 + i) * 4, c0);
        const T iJ = rcp_any(Jd);
        T res[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            T fr[N1];
            load_row<N1>(f + v * VS + j * RS, fr);
            T div = T(0);
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma_any(Di[m], fr[m], div);
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma_any(Dj[m], h[v * VS + m * RS + i], div);
            const T corr = gRi * c1[v] - gLi * c3[v] + gRj * c2[v] - gLj * c0[v];
            res[v] = -(div + corr) * iJ;
        }
        if (a.stage == 0) {
            store_residual(a, idx, res, rsq);
        } else {
            // The FP64 stage state: the registers of the FP64 path, a reload
            // (L1/L2-resident) for the mixed form.
            double us[4];
            if constexpr (sizeof(T) == 8) {
#pragma unroll
                for (int v = 0; v < 4; ++v) us[v] = double(u[v]);
            } else {
                gload4(a.U + idx * 4, us);
            }
            double uo[4];
            rk_update(a.stage, *a.dt, us, u0, res, uo);
            gstore4(a.Uout + idx * 4, uo);
            T* su = sU + el * FS + j * RS + i;
            T un[4];
            if constexpr (kRef) state_minus_ref(uo, ue, un);
            else {
#pragma unroll
                for (int v = 0; v < 4; ++v) un[v] = T(uo[v]);
            }
#pragma unroll
            for (int v = 0; v < 4; ++v) su[v * VS] = un[v];
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

    // ---- D: traces of the new state
    if (is_fp) {
        T t[4];
        trace_point<N1, RS, VS>(sU + el * FS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        if constexpr (kRef) {
#pragma unroll
            for (int v = 0; v < 4; ++v) t[v] += ue[v];
        }
        gstore4(a.Tout + (e * NFT + k) * 4, t);
        if (boundary_condition_edge(r)) store_ghost<N1>(a, r, nr[0], nr[1], fp, t);
    }
}

// Traces (and boundary ghost rows) of a state that did not come out of a
// stage launch.  a.U: state, a.Tout: trace buffer.
template <int P, typename T>
__global__ void __launch_bounds__(Shape<P, EbDiv<T>::value>::THREADS)
k_phys_traces(const StageArgsT<T> a) {
    using S = Shape<P, EbDiv<T>::value>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = Tiles<P, T>::FS;
    __shared__ T sOps[S::NOPS];
    __shared__ __align__(16) T sU[EB * FS];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    const int el = tid / TPE, k = tid - el * TPE;
    bool valid;
    const long long e = block_element(a, EB, el, valid);
    constexpr bool kRef = UsesRef<T>::value;
    T ue[4] = {T(0), T(0), T(0), T(0)};
    if (kRef && valid) load_state(a.U + e * NSP * 4, ue);
    if (valid && k < NSP) {
        double u[4];
        T w[4];
        stage_state(a, e * NSP + k, u, w);
        T* su = sU + el * FS + (k / N1) * RS + (k % N1);
        if constexpr (kRef) state_minus_ref(u, ue, w);
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = w[v];
    }
    __syncthreads();
    if (valid && k < NFT) {
        const int edge = k / N1, fp = k - edge * N1;
        T t[4];
        trace_point<N1, RS, VS>(sU + el * FS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        if constexpr (kRef) {
#pragma unroll
            for (int v = 0; v < 4; ++v) t[v] += ue[v];
        }
        gstore4(a.Tout + (e * NFT + k) * 4, t);
        const EdgeRec r = a.edges[e * 4 + edge];
        if (boundary_condition_edge(r)) {
            T n[3];
            load_normal(normal_rec<N1>(a, e, edge, fp), n);
            store_ghost<N1>(a, r, n[0], n[1], fp, t);
        }
    }
}

template <class K>
void prefer_shared(K kernel) {
    cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                         cudaSharedmemCarveoutMaxShared);
}

template <int P, int RIEM, typename T>
cudaError_t phys_stage_t(const StageArgsT<T>& a, cudaStream_t s) {
    using S = Shape<P, EbDiv<T>::value>;
    const long long grid = ((a.elist ? a.n_list : a.n_elem) + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    static bool carveout_set = false;
    if (!carveout_set) { prefer_shared(k_phys_stage<P, RIEM, T>); carveout_set = true; }
    return launch_programmatic(k_phys_stage<P, RIEM, T>, (unsigned)grid, S::THREADS, s, a);
}

template <int P, typename T>
cudaError_t phys_stage_p(int riemann, const StageArgsT<T>& a, cudaStream_t s) {
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV: return phys_stage_t<P, ZJ_RIEMANN_RUSANOV>(a, s);
        case ZJ_RIEMANN_ROE: return phys_stage_t<P, ZJ_RIEMANN_ROE>(a, s);
        case ZJ_RIEMANN_HLLC: return phys_stage_t<P, ZJ_RIEMANN_HLLC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int P, typename T>
cudaError_t phys_traces_t(const StageArgsT<T>& a, cudaStream_t s) {
    using S = Shape<P, EbDiv<T>::value>;
    const long long grid = ((a.elist ? a.n_list : a.n_elem) + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    k_phys_traces<P, T><<<(unsigned)grid, S::THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

template <typename T>
cudaError_t phys_traces_dispatch(int P, const StageArgsT<T>& a, cudaStream_t s) {
    switch (P) {
        case 1: return phys_traces_t<1>(a, s);
        case 2: return phys_traces_t<2>(a, s);
        case 3: return phys_traces_t<3>(a, s);
        case 4: return phys_traces_t<4>(a, s);
        case 5: return phys_traces_t<5>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t phys_stage_dispatch(int P, int riemann, const StageArgsT<T>& a, cudaStream_t s) {
    switch (P) {
        case 1: return phys_stage_p<1>(riemann, a, s);
        case 2: return phys_stage_p<2>(riemann, a, s);
        case 3: return phys_stage_p<3>(riemann, a, s);
        case 4: return phys_stage_p<4>(riemann, a, s);
        case 5: return phys_stage_p<5>(riemann, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace
}  // namespace zj
