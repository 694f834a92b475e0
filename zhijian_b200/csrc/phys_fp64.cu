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
#include "zj_physics.cuh"

namespace zj {
namespace {

using namespace dev;
using namespace phys;

#ifndef ZJ_PHYS_MIN_BLOCKS
#define ZJ_PHYS_MIN_BLOCKS 3
#endif

// -------------------------------------------------------------- kernels --

// Boundary ghost states live in extra rows of every trace buffer, after the
// E*4 element edges: row E*4 + slot of boundary slot `slot`, stored at the
// mirrored point n1-1-fp, so a boundary edge loads its ghost exactly like an
// interior edge loads its neighbour (index (row*n1 + n1-1-fp)).  They are
// written where the trace itself is produced, which keeps the ghost-state
// arithmetic (pow, branches per boundary class) out of the face phases.
__device__ __forceinline__ long long neighbour_row(const EdgeRec& r, long long n_elem) {
    return (r.flags & kEdgeBoundary) ? n_elem * 4 + r.nbr_edge : (long long)r.nbr * 4 + r.nbr_edge;
}

template <int N1>
__device__ __forceinline__ void store_ghost(const StageArgs& a, const EdgeRec& r, double nx, double ny,
                                            int fp, const double* t) {
    double q[4];
    ghost_phys(t, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, a.gamma, q);
    store4(a.Tout + ((a.n_elem * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, q);
}

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
    if (is_fp && !(r.flags & kEdgeOrphan))
        load4_nc(a.Tin + (neighbour_row(r, a.n_elem) * N1 + (N1 - 1 - fp)) * 4, qn);
    __syncthreads();   // sOps, sF, sG ready

    // ---- B: interface terms.  The common flux is evaluated from the left
    // element's side on both sides of a face (bit-identical on both).
    if (is_fp) {
        double Fd[4] = {0.0, 0.0, 0.0, 0.0};
        if (!(r.flags & kEdgeOrphan)) {
            const double nx = nr.x, ny = nr.y, s = 0.5 * nr.z;
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
        if (r.flags & kEdgeBoundary) store_ghost<N1>(a, r, nr.x, nr.y, fp, t);
    }
}

// Traces (and boundary ghost rows) of a state that did not come out of a
// stage launch.  a.U: state, a.Tout: trace buffer.
template <int P>
__global__ void __launch_bounds__(Shape<P>::THREADS)
k_phys_traces(const StageArgs a) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS;
    __shared__ double sOps[S::NOPS];
    __shared__ double sU[EB * FS];
    const int tid = threadIdx.x;
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    if (valid && k < NSP) {
        double u[4];
        load4_nc(a.U + (e * NSP + k) * 4, u);
        double* su = sU + el * FS + (k / N1) * RS + (k % N1);
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = u[v];
    }
    __syncthreads();
    if (valid && k < NFT) {
        const int edge = k / N1, fp = k - edge * N1;
        double t[4];
        trace_point<N1, RS, VS>(sU + el * FS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        store4(a.Tout + (e * NFT + k) * 4, t);
        const EdgeRec r = a.edges[e * 4 + edge];
        if (r.flags & kEdgeBoundary) {
            const double2 n01 = __ldg(reinterpret_cast<const double2*>(a.enrm + e * 4 + edge));
            store_ghost<N1>(a, r, n01.x, n01.y, fp, t);
        }
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

template <int P>
cudaError_t traces_t(const StageArgs& a, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    k_phys_traces<P><<<(unsigned)grid, S::THREADS, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_phys_traces(int P, const StageArgs& a, cudaStream_t s) {
    switch (P) {
        case 1: return traces_t<1>(a, s);
        case 2: return traces_t<2>(a, s);
        case 3: return traces_t<3>(a, s);
        case 4: return traces_t<4>(a, s);
        case 5: return traces_t<5>(a, s);
        default: return cudaErrorInvalidValue;
    }
}

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
