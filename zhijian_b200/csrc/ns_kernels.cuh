// ns_kernels.cuh -- Navier-Stokes residual and SSP-RK3 stages (physics mode,
// viscous on), templated on the arithmetic type T: double in ns_fp64.cu (the
// reference-parity path), float in ns_fp32.cu (the mixed-precision form; the
// state, the RK accumulation and the norm partials stay FP64).  Two launches
// per residual:
//
//  k_ns_grad_lines (float, double; k_ns_grad for dual numbers)
//              corrected gradient Q = grad U at the solution points and its
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
// copy the interior gradient (BoundaryCondition::ghostGradient) and walls
// impose their Neumann data on the common flux (wall_viscous_closure).
#pragma once

#include <cuda_runtime.h>

#include "zj_device.cuh"
#include "zj_kernels.h"
#include "zj_math.h"
#include "zj_physics.cuh"
#include "phys_kernels.cuh"

// Resident CTAs per SM the launch bounds ask for, counted in CTAs of 128
// threads (other CTA sizes scale them).
#ifndef ZJ_NS_MIN_BLOCKS
#define ZJ_NS_MIN_BLOCKS 5        // FP64 stage kernel (96 registers)
#endif
#ifndef ZJ_NSG_MIN_BLOCKS
#define ZJ_NSG_MIN_BLOCKS 8       // FP64 point-per-thread gradient kernel
#endif
#ifndef ZJ_NS32_MIN_BLOCKS
#define ZJ_NS32_MIN_BLOCKS 10     // mixed-precision stage kernel (48 registers)
#endif
#ifndef ZJ_NSG32_MIN_BLOCKS
#define ZJ_NSG32_MIN_BLOCKS 12    // mixed-precision point-per-thread gradient kernel
#endif
#ifndef ZJ_NS_MIN_BLOCKS_HI
#define ZJ_NS_MIN_BLOCKS_HI 4     // FP64 stage kernel at P5 (fewer spills)
#endif
#ifndef ZJ_NS32_MIN_BLOCKS_HI
#define ZJ_NS32_MIN_BLOCKS_HI 8   // mixed-precision stage kernel at P5
#endif
#ifndef ZJ_NSL_MIN_BLOCKS
#define ZJ_NSL_MIN_BLOCKS 5       // FP64 gradient kernel by lines (96 registers)
#endif
#ifndef ZJ_NSL_MIN_BLOCKS_HI
#define ZJ_NSL_MIN_BLOCKS_HI 4    // the same from P4 up (no spills)
#endif
#ifndef ZJ_NSL32_MIN_BLOCKS
#define ZJ_NSL32_MIN_BLOCKS 8     // mixed-precision gradient kernel by lines (64 registers)
#endif
#ifndef ZJ_NSL32_MIN_BLOCKS_HI
#define ZJ_NSL32_MIN_BLOCKS_HI 6  // the same from P4 up (no spills)
#endif

namespace zj {
namespace {

using namespace dev;
using namespace phys;

template <typename T, int P> struct NSMinBlocks;
constexpr int per_cta(int blocks128) { return blocks128 * 128 / kCtaThreads > 0 ? blocks128 * 128 / kCtaThreads : 1; }
template <int P> struct NSMinBlocks<double, P> {
    static constexpr int stage = per_cta(P <= 4 ? ZJ_NS_MIN_BLOCKS : ZJ_NS_MIN_BLOCKS_HI);
    static constexpr int grad = per_cta(ZJ_NSG_MIN_BLOCKS);
};
template <int P> struct NSMinBlocks<float, P> {
    static constexpr int stage = per_cta(P <= 4 ? ZJ_NS32_MIN_BLOCKS : ZJ_NS32_MIN_BLOCKS_HI);
    static constexpr int grad = per_cta(ZJ_NSG32_MIN_BLOCKS);
};
template <int P> struct NSMinBlocks<Dual, P> { static constexpr int stage = 1, grad = 1; };

// Corrected gradient at solution point (i, j) of one element: su is the
// element's state in the [var][row][col] shared layout, du its face jumps
// U_c - U_own in the [flux point][var] layout.
template <int N1, int RS, int VS, typename T>
__device__ __forceinline__ void corrected_gradient(const T* su, const T* du, const T* ops, int i,
                                                   int j, const T* ji, T* Qx, T* Qy) {
    const T* gL = ops + N1 * N1 + 2 * N1;
    const T* gR = gL + N1;
    T Di[N1], Dj[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) { Di[m] = ops[i * N1 + m]; Dj[m] = ops[j * N1 + m]; }
    T d1[4], d3[4], d0[4], d2[4];
    load4(du + (1 * N1 + j) * 4, d1);
    load4(du + (3 * N1 + (N1 - 1 - j)) * 4, d3);
    load4(du + (0 * N1 + i) * 4, d0);
    load4(du + (2 * N1 + (N1 - 1 - i)) * 4, d2);
    const T gRi = gR[i], gLi = gL[i], gRj = gR[j], gLj = gL[j];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        T row[N1];
        load_row<N1>(su + v * VS + j * RS, row);
        T dxi = T(0), deta = T(0);
#pragma unroll
        for (int m = 0; m < N1; ++m) {
            dxi = fma_any(Di[m], row[m], dxi);
            deta = fma_any(Dj[m], su[v * VS + m * RS + i], deta);
        }
        dxi += gRi * d1[v] + gLi * d3[v];
        deta += gLj * d0[v] + gRj * d2[v];
        Qx[v] = ji[0] * dxi + ji[2] * deta;
        Qy[v] = ji[1] * dxi + ji[3] * deta;
    }
}

// The same gradient with the element's tile also held transposed (sut:
// [var][xi][eta]), so the eta-line of point (i, j) is a row: vector loads
// instead of N1 strided ones; the sums run in the same order.
template <int N1, int RS, int VS, typename T>
__device__ __forceinline__ void corrected_gradient_tr(const T* su, const T* sut, const T* du, const T* ops,
                                                      int i, int j, const T* ji, T* Qx, T* Qy) {
    const T* gL = ops + N1 * N1 + 2 * N1;
    const T* gR = gL + N1;
    T Di[N1], Dj[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) { Di[m] = ops[i * N1 + m]; Dj[m] = ops[j * N1 + m]; }
    T d1[4], d3[4], d0[4], d2[4];
    load4(du + (1 * N1 + j) * 4, d1);
    load4(du + (3 * N1 + (N1 - 1 - j)) * 4, d3);
    load4(du + (0 * N1 + i) * 4, d0);
    load4(du + (2 * N1 + (N1 - 1 - i)) * 4, d2);
    const T gRi = gR[i], gLi = gL[i], gRj = gR[j], gLj = gL[j];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        T row[N1], col[N1];
        load_row<N1>(su + v * VS + j * RS, row);
        load_row<N1>(sut + v * VS + i * RS, col);
        T dxi = T(0), deta = T(0);
#pragma unroll
        for (int m = 0; m < N1; ++m) {
            dxi = fma_any(Di[m], row[m], dxi);
            deta = fma_any(Dj[m], col[m], deta);
        }
        dxi += gRi * d1[v] + gLi * d3[v];
        deta += gLj * d0[v] + gRj * d2[v];
        Qx[v] = ji[0] * dxi + ji[2] * deta;
        Qy[v] = ji[1] * dxi + ji[3] * deta;
    }
}

// Loads of a flux-point thread: edge record, normal, own trace, the
// neighbour's coinciding trace point or the ghost state.
template <typename T>
struct FacePoint {
    EdgeRec r;
    T nx, ny, len;
    T qo[4], qn[4];
};

template <int N1, typename T>
__device__ __forceinline__ void load_face_point(const StageArgsT<T>& a, long long e, int edge, int fp,
                                                FacePoint<T>& f) {
    constexpr int NFT = 4 * N1;
    f.r = a.edges[e * 4 + edge];
    T n[3];
    load_normal(normal_rec<N1>(a, e, edge, fp), n);
    f.nx = n[0]; f.ny = n[1]; f.len = n[2];
    load4_nc(a.Tin + (e * NFT + edge * N1 + fp) * 4, f.qo);
    f.qn[0] = f.qo[0]; f.qn[1] = f.qo[1]; f.qn[2] = f.qo[2]; f.qn[3] = f.qo[3];
    if (!(f.r.flags & kEdgeOrphan)) {
        // interior: the neighbour's coinciding point; boundary: the ghost row
        // written with the trace
        load4_nc(a.Tin + (neighbour_row(f.r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, f.qn);
    }
}

template <int P, typename T>
__global__ void __launch_bounds__(Shape<P, EbDiv<T>::value>::THREADS, NSMinBlocks<T, P>::grad)
k_ns_grad(const StageArgsT<T> a) {
    using S = Shape<P, EbDiv<T>::value>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = Tiles<P, T>::FS, DS = Tiles<P, T>::DS;
    constexpr int QS = Tiles<P, T>::QS;
    __shared__ T sOps[S::NOPS];
    __shared__ __align__(16) T sU[EB * FS];
    __shared__ __align__(16) T sUt[EB * FS];   // the same tile transposed
    __shared__ __align__(16) T sDU[EB * DS];
    __shared__ __align__(16) T sQ[EB * QS];

    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous stage
    const int el = tid / TPE, k = tid - el * TPE;
    bool valid;
    const long long e = block_element(a, EB, el, valid);
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    constexpr bool kRef = UsesRef<T>::value;
    T ji[4];
    if (is_sp) {
        const long long idx = e * NSP + k;
        T u[4];
        if constexpr (kRef) {
            // D (U - U_e): the reference drops out of the derivative exactly
            double ud[4];
            T ue[4];
            gload4(a.U + idx * 4, ud);
            load_state(a.U + e * NSP * 4, ue);
            state_minus_ref(ud, ue, u);
        } else {
            double ud[4];
            stage_state(a, idx, ud, u);
        }
        load4_nc(a.Jinv + idx * 4, ji);
        T* su = sU + el * FS + j * RS + i;
        T* sut = sUt + el * FS + i * RS + j;
#pragma unroll
        for (int v = 0; v < 4; ++v) { su[v * VS] = u[v]; sut[v * VS] = u[v]; }
    }
    if (is_fp) {
        FacePoint<T> f;
        load_face_point<N1>(a, e, edge, fp, f);
        T d[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) d[v] = (f.r.flags & kEdgeOrphan) ? T(0) : T(0.5) * (f.qn[v] - f.qo[v]);
        store4(sDU + el * DS + k * 4, d);
    }
    __syncthreads();
    if (is_sp) {
        T Qx[4], Qy[4];
        corrected_gradient_tr<N1, RS, VS>(sU + el * FS, sUt + el * FS, sDU + el * DS, sOps, i, j, ji, Qx, Qy);
        T* sq = sQ + el * QS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) { sq[v * VS] = Qx[v]; sq[(4 + v) * VS] = Qy[v]; }
    }
    __syncthreads();
    if (is_fp) {
        T t[8];
        trace_point<N1, RS, VS>(sQ + el * QS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        trace_point<N1, RS, VS>(sQ + el * QS + 4 * VS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge,
                                fp, t + 4);
        T* o = a.TQout + (e * NFT + k) * 8;
        gstore8(o, t);
    }
}

// ---- gradient by lines (float and double)
//
// 2 N1 threads per element: one per row j (an xi-line of solution points
// (0..N1-1, j)) and one per column i (an eta-line (i, 0..N1-1)).  The CTA
// first stages its elements' states into shared memory with 16-byte cp.async
// copies (each 16-byte piece fetched once), while every line thread loads the
// traces at its line's two end points (its own and the neighbour's).  A line thread then takes the corrected derivative along its
// line in registers (row: dU/dxi with the jumps of edges 1 and 3; column:
// dU/deta with those of edges 0 and 2) and swaps derivatives with the
// crossing lines through one shared tile.  It forms Q = (xi_x dU/dxi + eta_x
// dU/deta, xi_y dU/dxi + eta_y dU/deta) at its N1 points and the traces of Q
// at its two end points (row j: edge 1 point j with l(+1), edge 3 point
// N1-1-j with l(-1); column i: edge 0 point i with l(-1), edge 2 point
// N1-1-i with l(+1)).  Every sum is corrected_gradient_tr's and
// trace_point's, term for term in the same order, so the traces equal
// k_ns_grad's.
//
// Rows and columns run the same instruction stream (the role only selects
// strides, edges and weights) and fill separate warps at P3.  The derivative
// tile holds point (a = xi index, b = eta index) at a*(N1+1) + b; the staged
// rows are padded by 16 bytes; the element strides spread both access
// patterns over the banks.
template <int P, typename T>
struct LineShape {
    static constexpr int N1 = P + 1, NSP = N1 * N1, NFT = 4 * N1;
    static constexpr int EB = kCtaThreads / (2 * N1);   // elements per CTA
    static constexpr int THREADS = EB * 2 * N1;
    static constexpr int NOPS = N1 * N1 + 4 * N1;
    // derivative tile: [el][role][var][a*R + b]
    static constexpr int R = N1 + 1;
    static constexpr int VB = N1 * R;
    static constexpr int MOD = sizeof(T) == 8 ? 16 : 32;
    static constexpr int ES = 8 * VB + ((4 - (8 * VB) % MOD) + MOD) % MOD;
    // staged states (doubles): [el][b][a*4 + v], rows padded by 16 bytes, the
    // element stride 64 bytes past a multiple of 128
    static constexpr int RU = N1 * 4 + 2;
    static constexpr int EU = N1 * RU + ((8 - (N1 * RU) % 16) + 16) % 16;
    // dynamic shared memory layout (byte offsets, 16-byte aligned); the
    // metrics are read directly (one 16- or 32-byte load a point), which
    // measured faster than staging them with the states
    static constexpr size_t OFF_U = 0;
    static constexpr size_t OFF_D = OFF_U + sizeof(double) * EB * EU;
    static constexpr size_t OFF_OPS = OFF_D + ((sizeof(T) * EB * ES + 15) & ~size_t(15));
    static constexpr size_t SMEM = OFF_OPS + ((sizeof(T) * NOPS + 15) & ~size_t(15));
    static_assert(OFF_D % 16 == 0 && OFF_OPS % 16 == 0, "16-byte aligned regions");
    // A line thread holds a line's states and derivatives: twice the values
    // of a point thread, at half the threads per element.
    // (the counts are per 128 threads; other CTA sizes scale them)
    static constexpr int MIN_BLOCKS_128 =
        sizeof(T) == 8 ? (P <= 3 ? ZJ_NSL_MIN_BLOCKS : ZJ_NSL_MIN_BLOCKS_HI)
                       : (P <= 3 ? ZJ_NSL32_MIN_BLOCKS : ZJ_NSL32_MIN_BLOCKS_HI);
    static constexpr int MIN_BLOCKS = MIN_BLOCKS_128 * 128 / kCtaThreads > 0 ? MIN_BLOCKS_128 * 128 / kCtaThreads : 1;
};

// 16-byte asynchronous global -> shared copy (cp.async, cached in L2 only),
// and the wait for all of this thread's copies.
__device__ __forceinline__ void cp_async16(void* sdst, const void* gsrc) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(sdst));
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

template <int P, typename T>
__global__ void __launch_bounds__(LineShape<P, T>::THREADS, LineShape<P, T>::MIN_BLOCKS)
k_ns_grad_lines(const StageArgsT<T> a) {
    using L = LineShape<P, T>;
    constexpr int N1 = L::N1, NSP = L::NSP, NFT = L::NFT, EB = L::EB, R = L::R, VB = L::VB, ES = L::ES;
    constexpr int RU = L::RU, EU = L::EU;
    extern __shared__ __align__(16) unsigned char smem[];
    double* sU = reinterpret_cast<double*>(smem + L::OFF_U);
    T* sD = reinterpret_cast<T*>(smem + L::OFF_D);
    T* sOps = reinterpret_cast<T*>(smem + L::OFF_OPS);

    const int tid = threadIdx.x;
    for (int t = tid; t < L::NOPS; t += L::THREADS) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous stage
    for (int c = tid; c < EB * NSP * 2; c += L::THREADS) {
        const int el2 = c / (NSP * 2), r = c - el2 * NSP * 2, p = r >> 1, h = r & 1;
        bool v2;
        const long long e2 = block_element(a, EB, el2, v2);
        if (v2) cp_async16(sU + el2 * EU + (p / N1) * RU + (p % N1) * 4 + h * 2, a.U + (e2 * NSP + p) * 4 + h * 2);
    }
    cp_async_commit();

    const int role = tid / (EB * N1);            // 0: row (xi-line), 1: column (eta-line)
    const int rem = tid - role * EB * N1;
    const int el = rem / N1, line = rem - el * N1;
    bool valid;
    const long long e = block_element(a, EB, el, valid);
    // staged offset of the line's point m: row j -> (m, j), column i -> (i, m)
    const int ubase = role ? line * 4 : line * RU, ustride = role ? RU : 4;
    // derivative-tile offset of point m: (a, b) -> a*R + b
    const int tbase = role ? line * R : line, tstride = role ? 1 : R;
    const int eA = role ? 0 : 1, eB = role ? 2 : 3;
    const int fA = line, fB = N1 - 1 - line;
    constexpr bool kRef = UsesRef<T>::value;

    // jumps U_c - U_own = (U_nbr - U_own)/2 at the line's end points
    T dA[4], dB[4];
    if (valid) {
#pragma unroll
        for (int s2 = 0; s2 < 2; ++s2) {
            const int ed = s2 ? eB : eA, fp = s2 ? fB : fA;
            const EdgeRec r = a.edges[e * 4 + ed];
            T qo[4], qn[4];
            load4_nc(a.Tin + (e * NFT + ed * N1 + fp) * 4, qo);
#pragma unroll
            for (int v = 0; v < 4; ++v) qn[v] = qo[v];
            if (!(r.flags & kEdgeOrphan)) load4_nc(a.Tin + (neighbour_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
            T* d = s2 ? dB : dA;
#pragma unroll
            for (int v = 0; v < 4; ++v) d[v] = (r.flags & kEdgeOrphan) ? T(0) : T(0.5) * (qn[v] - qo[v]);
        }
    }
    cp_async_wait_all();
    __syncthreads();   // staged states, operators

    T mine[N1][4];
    if (valid) {
        T u[N1][4];
        const double* su = sU + el * EU;
        T ue[4];
        if constexpr (kRef) {
            double d0[4];
            load4(su, d0);   // the element's first solution point
#pragma unroll
            for (int v = 0; v < 4; ++v) ue[v] = T(d0[v]);
        }
#pragma unroll
        for (int m = 0; m < N1; ++m) {
            double ud[4];
            load4(su + ubase + m * ustride, ud);
            if constexpr (kRef) {
                // D (U - U_e): the reference drops out of the derivative exactly
                state_minus_ref(ud, ue, u[m]);
            } else {
#pragma unroll
                for (int v = 0; v < 4; ++v) u[m][v] = T(ud[v]);
            }
        }
        // corrected derivative along the line: sum_k D[m][k] u_k, then
        // + g1(m) jump_A + g2(m) jump_B (rows: g_R, g_L; columns: g_L, g_R)
        const T* gL = sOps + N1 * N1 + 2 * N1;
        const T* gR = gL + N1;
        const T* g1 = role ? gL : gR;
        const T* g2 = role ? gR : gL;
#pragma unroll
        for (int m = 0; m < N1; ++m) {
            T Dm[N1];
            load_op_row<N1>(sOps, m, Dm);
            const T g1m = g1[m], g2m = g2[m];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                T acc = T(0);
#pragma unroll
                for (int k = 0; k < N1; ++k) acc = fma_any(Dm[k], u[k][v], acc);
                acc += g1m * dA[v] + g2m * dB[v];
                mine[m][v] = acc;
            }
        }
        T* sd = sD + el * ES + role * 4 * VB + tbase;
#pragma unroll
        for (int m = 0; m < N1; ++m)
#pragma unroll
            for (int v = 0; v < 4; ++v) sd[v * VB + m * tstride] = mine[m][v];
    }
    __syncthreads();
    if (!valid) return;

    // Q at the line's points and its traces at the two end points
    const T* WA = sOps + N1 * N1 + (role ? 0 : N1);   // row: l(+1) at edge 1; column: l(-1) at edge 0
    const T* WB = sOps + N1 * N1 + (role ? N1 : 0);   // row: l(-1) at edge 3; column: l(+1) at edge 2
    const T* so = sD + el * ES + (1 - role) * 4 * VB + tbase;
    T tA[8], tB[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) { tA[c] = T(0); tB[c] = T(0); }
#pragma unroll
    for (int m = 0; m < N1; ++m) {
        T ji[4];
        load4_nc(a.Jinv + (e * NSP + (role ? line + m * N1 : line * N1 + m)) * 4, ji);
        const T wa = WA[m], wb = WB[m];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const T other = so[v * VB + m * tstride];
            const T dxi = role ? other : mine[m][v];
            const T deta = role ? mine[m][v] : other;
            const T Qx = ji[0] * dxi + ji[2] * deta;
            const T Qy = ji[1] * dxi + ji[3] * deta;
            tA[v] = fma_any(wa, Qx, tA[v]);
            tA[4 + v] = fma_any(wa, Qy, tA[4 + v]);
            tB[v] = fma_any(wb, Qx, tB[v]);
            tB[4 + v] = fma_any(wb, Qy, tB[4 + v]);
        }
    }
    gstore8(a.TQout + (e * NFT + eA * N1 + fA) * 8, tA);
    gstore8(a.TQout + (e * NFT + eB * N1 + fB) * 8, tB);
}

template <int P, int RIEM, typename T>
__global__ void __launch_bounds__(Shape<P, EbDiv<T>::value>::THREADS, NSMinBlocks<T, P>::stage)
k_ns_stage(const StageArgsT<T> a) {
    using S = Shape<P, EbDiv<T>::value>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = Tiles<P, T>::FS, DS = Tiles<P, T>::DS;
    __shared__ T sOps[S::NOPS];
    // From P4 up the G~ tile is held transposed ([var][xi][eta]), so its
    // eta-lines (divergence, traces of edges 0 and 2) are row loads
    constexpr bool kTrG = P >= 4;
    __shared__ __align__(16) T sF[EB * FS];
    __shared__ __align__(16) T sG[EB * FS];
    __shared__ __align__(16) T sD[EB * DS];   // face jumps of U, then flux differences
    __shared__ __align__(16) T sU[EB * FS];   // stage state, then the new state
    __shared__ double sRed[32];
    // A flux-point thread's face data from the loads to the face phase, parked
    // here (component-major: a warp's accesses fill consecutive banks) so
    // that it holds no registers through the volume phase: own and neighbour
    // traces (4 + 4) and the average gradient trace (8).
    __shared__ T sFP[16 * S::THREADS];

    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    pdl_launch_dependents();
    pdl_wait();   // the gradient traces come from k_ns_grad, the state from the previous stage
    const int el = tid / TPE, k = tid - el * TPE;
    bool valid;
    const long long e = block_element(a, EB, el, valid);
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const T g = T(a.gamma);
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    // ---- A1: loads, face jumps, stage state into shared memory
    FacePoint<T> f;
    T* pk = sFP + tid;   // this thread's parked face data, stride S::THREADS
    if (is_fp) {
        T Qo[8], Qn[8];
        load_face_point<N1>(a, e, edge, fp, f);
        const T* qt = a.TQ + (e * NFT + k) * 8;
        gload8_nc(qt, Qo);
#pragma unroll
        for (int v = 0; v < 8; ++v) Qn[v] = Qo[v];
        if (has_neighbour_gradient(f.r)) {
            const T* qn = a.TQ + (neighbour_row(f.r, a.n_elem) * N1 + (N1 - 1 - fp)) * 8;
            gload8_nc(qn, Qn);
        }
        T d[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) d[v] = (f.r.flags & kEdgeOrphan) ? T(0) : T(0.5) * (f.qn[v] - f.qo[v]);
        store4(sD + el * DS + k * 4, d);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            pk[v * S::THREADS] = f.qo[v];
            pk[(4 + v) * S::THREADS] = f.qn[v];
        }
#pragma unroll
        for (int v = 0; v < 8; ++v) pk[(8 + v) * S::THREADS] = T(0.5) * (Qo[v] + Qn[v]);
    }
    constexpr bool kRef = UsesRef<T>::value;
    T ue[4] = {T(0), T(0), T(0), T(0)};   // reference state (mixed form)
    if (kRef && valid) load_state(a.U + e * NSP * 4, ue);
    T u[4], ji[4], Jd = T(1);
    if (is_sp) {
        const long long idx = e * NSP + k;
        double ud[4];
        stage_state(a, idx, ud, u);
        load4_nc(a.Jinv + idx * 4, ji);
        Jd = ldg_any(a.J + idx);
        if ((k & 3) == 0 && a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        T* su = sU + el * FS + j * RS + i;
        T w[4];
        if constexpr (kRef) state_minus_ref(ud, ue, w);
        else {
#pragma unroll
            for (int v = 0; v < 4; ++v) w[v] = u[v];
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = w[v];
    }
    __syncthreads();

    // ---- A2: gradient, total transformed fluxes
    if (is_sp) {
        T Qx[4], Qy[4], Fv[4], Gv[4];
        corrected_gradient<N1, RS, VS>(sU + el * FS, sD + el * DS, sOps, i, j, ji, Qx, Qy);
        // one reciprocal density for the viscous and the Euler flux
        const T ir = rcp_any(u[0]);
        viscous_flux_f(u, ir, Qx, Qy, g, inv_reynolds(a), T(a.kfac), Fv, Gv);
        T F[4], G[4];
        euler_flux_ir(u, ir, g, F, G);
        if constexpr (kRef) {
            T Fe[4], Ge[4];
            euler_flux(ue, g, Fe, Ge);
#pragma unroll
            for (int v = 0; v < 4; ++v) { F[v] -= Fe[v]; G[v] -= Ge[v]; }
        }
#pragma unroll
        for (int v = 0; v < 4; ++v) { F[v] -= Fv[v]; G[v] -= Gv[v]; }
        T* fo = sF + el * FS + j * RS + i;
        T* ho = sG + el * FS + (kTrG ? i * RS + j : j * RS + i);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            fo[v * VS] = Jd * (ji[0] * F[v] + ji[1] * G[v]);
            ho[v * VS] = Jd * (ji[2] * F[v] + ji[3] * G[v]);
        }
    }
    __syncthreads();   // face jumps and the stage state in shared memory are dead now

    // ---- B: interface terms, evaluated from the left element's side
    if (is_fp) {
        T Fd[4] = {T(0), T(0), T(0), T(0)};
        if (!(f.r.flags & kEdgeOrphan)) {
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                f.qo[v] = pk[v * S::THREADS];
                f.qn[v] = pk[(4 + v) * S::THREADS];
            }
            const bool right = (f.r.flags & kEdgeRight) != 0;
            T UL[4], UR[4], Fc[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) { UL[v] = right ? f.qn[v] : f.qo[v]; UR[v] = right ? f.qo[v] : f.qn[v]; }
            riemann<RIEM>(UL, UR, f.nx, f.ny, g, Fc);
            if constexpr (kRef) {
                T Fe[4];
                ref_flux_n(ue, g, f.nx, f.ny, Fe);
#pragma unroll
                for (int v = 0; v < 4; ++v) Fc[v] -= Fe[v];
            }
            T Ua[4], dxa[4], dya[4], Fv[4], Gv[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) {
                Ua[v] = T(0.5) * (UL[v] + UR[v]);
                dxa[v] = pk[(8 + v) * S::THREADS];
                dya[v] = pk[(12 + v) * S::THREADS];
            }
            viscous_flux_f(Ua, rcp_any(Ua[0]), dxa, dya, g, inv_reynolds(a), T(a.kfac), Fv, Gv);
            T Fvn[4];
#pragma unroll
            for (int v = 0; v < 4; ++v) Fvn[v] = Fv[v] * f.nx + Gv[v] * f.ny;
            boundary_viscous_closure(f.r, a.bc, f.nx, f.ny, Fvn);
            const T ss = right ? T(-0.5) * f.len : T(0.5) * f.len;
            const bool along_eta = (edge == 0 || edge == 2);
            T Fn[4];
            if constexpr (kTrG)
                trace_row<N1, RS, VS>((along_eta ? sG : sF) + el * FS,
                                      (edge == 0 || edge == 3) ? sOps + N1 * N1 : sOps + N1 * N1 + N1,
                                      (edge >= 2) ? (N1 - 1 - fp) : fp, Fn);
            else
                trace_point<N1, RS, VS>((along_eta ? sG : sF) + el * FS, sOps + N1 * N1,
                                        sOps + N1 * N1 + N1, edge, fp, Fn);
            const T sgn = (edge == 0 || edge == 3) ? T(-1) : T(1);
#pragma unroll
            for (int v = 0; v < 4; ++v)
                Fd[v] = ss * (Fc[v] - Fvn[v]) - sgn * Fn[v];
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
        const T* fo = sF + el * FS;
        const T* ho = sG + el * FS;
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
            load_row<N1>(fo + v * VS + j * RS, fr);
            T div = T(0);
#pragma unroll
            for (int m = 0; m < N1; ++m) div = fma_any(Di[m], fr[m], div);
            if constexpr (kTrG) {
                T gc[N1];
                load_row<N1>(ho + v * VS + i * RS, gc);
#pragma unroll
                for (int m = 0; m < N1; ++m) div = fma_any(Dj[m], gc[m], div);
            } else {
#pragma unroll
                for (int m = 0; m < N1; ++m) div = fma_any(Dj[m], ho[v * VS + m * RS + i], div);
            }
            const T corr = gRi * c1[v] - gLi * c3[v] + gRj * c2[v] - gLj * c0[v];
            res[v] = -(div + corr) * iJ;
        }
        if (a.stage == 0) {
            store_residual(a, idx, res, rsq);
        } else {
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
        if (boundary_condition_edge(f.r)) store_ghost<N1>(a, f.r, f.nx, f.ny, fp, t);
    }
}

template <int P, typename T>
cudaError_t ns_grad_t(const StageArgsT<T>& a, cudaStream_t s) {
    if constexpr (!IsDual<T>::value) {
        using L = LineShape<P, T>;
        const long long grid = ((a.elist ? a.n_list : a.n_elem) + L::EB - 1) / L::EB;
        if (grid <= 0) return cudaSuccess;
        static bool set = false;
        if (!set) {
            prefer_shared(k_ns_grad_lines<P, T>);
            cudaFuncSetAttribute(k_ns_grad_lines<P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::SMEM);
            set = true;
        }
        return launch_programmatic_smem(k_ns_grad_lines<P, T>, (unsigned)grid, L::THREADS, L::SMEM, s, a);
    } else {
        using S = Shape<P, EbDiv<T>::value>;
        const long long grid = ((a.elist ? a.n_list : a.n_elem) + S::EB - 1) / S::EB;
        if (grid <= 0) return cudaSuccess;
        static bool set = false;
        if (!set) { prefer_shared(k_ns_grad<P, T>); set = true; }
        return launch_programmatic(k_ns_grad<P, T>, (unsigned)grid, S::THREADS, s, a);
    }
}

template <int P, int RIEM, typename T>
cudaError_t ns_stage_t(const StageArgsT<T>& a, cudaStream_t s) {
    using S = Shape<P, EbDiv<T>::value>;
    const long long grid = ((a.elist ? a.n_list : a.n_elem) + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    static bool set = false;
    if (!set) { prefer_shared(k_ns_stage<P, RIEM, T>); set = true; }
    return launch_programmatic(k_ns_stage<P, RIEM, T>, (unsigned)grid, S::THREADS, s, a);
}

template <int P, typename T>
cudaError_t ns_stage_p(int riemann, const StageArgsT<T>& a, cudaStream_t s) {
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV: return ns_stage_t<P, ZJ_RIEMANN_RUSANOV>(a, s);
        case ZJ_RIEMANN_ROE: return ns_stage_t<P, ZJ_RIEMANN_ROE>(a, s);
        case ZJ_RIEMANN_HLLC: return ns_stage_t<P, ZJ_RIEMANN_HLLC>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t ns_grad_dispatch(int P, const StageArgsT<T>& a, cudaStream_t s) {
    switch (P) {
        case 1: return ns_grad_t<1>(a, s);
        case 2: return ns_grad_t<2>(a, s);
        case 3: return ns_grad_t<3>(a, s);
        case 4: return ns_grad_t<4>(a, s);
        case 5: return ns_grad_t<5>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

template <typename T>
cudaError_t ns_stage_dispatch(int P, int riemann, const StageArgsT<T>& a, cudaStream_t s) {
    switch (P) {
        case 1: return ns_stage_p<1>(riemann, a, s);
        case 2: return ns_stage_p<2>(riemann, a, s);
        case 3: return ns_stage_p<3>(riemann, a, s);
        case 4: return ns_stage_p<4>(riemann, a, s);
        case 5: return ns_stage_p<5>(riemann, a, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace
}  // namespace zj
