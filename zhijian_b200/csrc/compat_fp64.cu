// compat_fp64.cu -- FP64 residual and SSP-RK3 stage kernels with the
// reference's residual semantics ("compat" mode).
//
// One fused launch per RK stage.  A CTA owns EB consecutive elements; every
// element has TPE threads.  Per stage:
//   A  thread per solution point: load the stage state (32 contiguous bytes
//      per point, coalesced across the warp), Euler fluxes into shared memory.
//   B  thread per flux point: own trace + the neighbour's trace (written by
//      the previous stage), ghost state on boundaries, Rusanov flux and the
//      flux difference of this element's side, into shared memory.
//   C  thread per solution point: sum-factorised divergence, FR correction,
//      SSP-RK3 update and positivity clamp; write the new state.
//   D  thread per flux point: traces of the new state for the next stage.
// The 2D reference operators are Kronecker products of 1D ones with exact
// 0/1 factors, so the sum-factorised sums add the same nonzero terms in the
// same order as the reference's dense loops.
//
// Reference: src/gpu/kernels.cu K1 :30-67, K4 :157-194, K8 :346-450,
// K9 :453-525, K10 :528-701, K13 :813-872, K15 :948-1034, K17 :1245-1295,
// K18 :1297-1349; include/physics/euler.hpp:16-129.
#include <cuda_runtime.h>

#include "zj_kernels.h"
#include "zj_math.h"
#include "zj_device.cuh"

namespace zj {

void pack_ops(const Operators1D& o, std::vector<double>& out) {
    const int n1 = o.n1;
    out.assign(ops_size(n1), 0.0);
    for (int i = 0; i < n1 * n1; ++i) out[i] = o.D1[i];
    for (int j = 0; j < n1; ++j) {
        out[n1 * n1 + j] = o.Lm[j];
        out[n1 * n1 + n1 + j] = o.Lp[j];
        out[n1 * n1 + 2 * n1 + j] = o.gL[j];
        out[n1 * n1 + 3 * n1 + j] = o.gR[j];
    }
}

namespace {

using namespace dev;


// ---------------------------------------------------------------- physics --
//
// The reference divides by rho up to ten times per state; here every state
// takes one reciprocal and multiplies, and reciprocals and square roots come
// from zj_math.h (Newton-Raphson FMA chains, within 2 ulp) instead of the
// long FP64 divide/sqrt sequences.  Each quotient moves by a few ulp; the residual stays within 1e-12
// of the reference's.

// Primitive quantities of one trace state in the form the reference's
// Rusanov flux uses them (kernels.cu:601-630): floored density and pressure,
// velocities, total enthalpy and the wave speed |u| + c.  praw is the
// pressure of IdealGas::pressure (euler.hpp:16-23) from the unfloored
// density, used by the interior flux and the wall ghost states; it differs
// from the floored form only when the trace density is below 1e-10.
struct Prim {
    double q[4];
    double rho, u, v, p, s, H, praw;
};

__device__ __forceinline__ void raw_velocity(const Prim& w, double& u, double& v) {
    if (w.q[0] >= 1e-10) { u = w.u; v = w.v; }
    else { const double ir = 1.0 / w.q[0]; u = w.q[1] * ir; v = w.q[2] * ir; }
}

__device__ __forceinline__ void make_prim(const double* q, double g, Prim& w) {
    w.q[0] = q[0]; w.q[1] = q[1]; w.q[2] = q[2]; w.q[3] = q[3];
    w.rho = fmax(q[0], 1e-10);
    const double ir = rcp_any(w.rho);
    w.u = q[1] * ir;
    w.v = q[2] * ir;
    const double E = q[3] * ir;
    const double pf = (g - 1.0) * w.rho * (E - 0.5 * (w.u * w.u + w.v * w.v));
    if (q[0] >= 1e-10) {
        w.praw = pf;
    } else {
        const double irr = 1.0 / q[0];
        const double ur = q[1] * irr, vr = q[2] * irr;
        w.praw = (g - 1.0) * q[0] * (q[3] * irr - 0.5 * (ur * ur + vr * vr));
    }
    w.p = fmax(pf, 1e-10);
    const double c = zj_sqrt(fmax(g * w.p * ir, 1e-10));
    w.s = zj_sqrt(w.u * w.u + w.v * w.v) + c;
    w.H = E + w.p * ir;
}

// Normal component of the Euler flux (IdealGas::fluxX/fluxY, euler.hpp:101-129).
__device__ __forceinline__ void flux_normal(const Prim& w, double nx, double ny, double* Fn) {
    const double pr = w.praw;
    double u, v;
    raw_velocity(w, u, v);
    Fn[0] = w.q[1] * nx + w.q[2] * ny;
    Fn[1] = (w.q[1] * u + pr) * nx + (w.q[2] * u) * ny;
    Fn[2] = (w.q[1] * v) * nx + (w.q[2] * v + pr) * ny;
    Fn[3] = ((w.q[3] + pr) * u) * nx + ((w.q[3] + pr) * v) * ny;
}

// The reference's hard-coded Rusanov flux with floors (kernels.cu:597-669):
// s_max = max(|u|+c) over both sides, F = (F_L+F_R)/2 - s_max (U_R-U_L)/2,
// NaN/Inf -> 0.  Evaluated for (L, R) = (O, X), or (X, O) when swap: the
// central part and s_max are symmetric and IEEE addition commutes, while
// U_R - U_L only changes sign exactly, so both orders need one code path.
__device__ __forceinline__ void rusanov_pair(const Prim& O, const Prim& X, bool swap, double nx,
                                             double ny, double* F) {
    const double vnO = O.u * nx + O.v * ny, vnX = X.u * nx + X.v * ny;
    const double smax = fmax(O.s, X.s);
    const double FO[4] = {O.rho * vnO, O.rho * O.u * vnO + O.p * nx, O.rho * O.v * vnO + O.p * ny,
                          O.rho * O.H * vnO};
    const double FX[4] = {X.rho * vnX, X.rho * X.u * vnX + X.p * nx, X.rho * X.v * vnX + X.p * ny,
                          X.rho * X.H * vnX};
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double jump = swap ? (O.q[v] - X.q[v]) : (X.q[v] - O.q[v]);
        const double f = 0.5 * (FO[v] + FX[v]) - 0.5 * smax * jump;
        F[v] = isfinite(f) ? f : 0.0;
    }
}

__device__ __forceinline__ void prim2cons(double rho, double u, double v, double p, double g,
                                          double* U) {
    U[0] = rho; U[1] = rho * u; U[2] = rho * v;
    U[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
}

// computeGhostState (kernels.cu:453-525), from the interior primitives.
__device__ void ghost_compat(const Prim& w, double nx, double ny, int bct,
                             const double* __restrict__ bcd, double g, double* Ug) {
    switch (bct) {
        case ZJ_BC_WALL: case ZJ_BC_SLIPWALL: case ZJ_BC_SYMMETRY: {
            double u, v;
            raw_velocity(w, u, v);
            const double vn = u * nx + v * ny;
            prim2cons(w.q[0], u - 2.0 * vn * nx, v - 2.0 * vn * ny, w.praw, g, Ug);
            break;
        }
        case ZJ_BC_FARFIELD: {
            const double rho_inf = bcd[0], u_inf = bcd[1], v_inf = bcd[2], p_inf = bcd[3];
            const double vn_inf = u_inf * nx + v_inf * ny;
            double rb, ub, vb;
            if (vn_inf > 0) { rb = rho_inf; ub = u_inf; vb = v_inf; }
            else { rb = w.rho; ub = w.u; vb = w.v; }
            double pb = 0.5 * (p_inf + w.p);
            rb = fmax(fmin(rb, 100.0), 0.01);
            ub = fmax(fmin(ub, 1000.0), -1000.0);
            vb = fmax(fmin(vb, 1000.0), -1000.0);
            pb = fmax(fmin(pb, 1e7), 1e3);
            prim2cons(rb, ub, vb, pb, g, Ug);
            break;
        }
        case ZJ_BC_OUTFLOW: {
            double u, v;
            raw_velocity(w, u, v);
            prim2cons(w.q[0], u, v, bcd[0], g, Ug);
            break;
        }
        default:
            Ug[0] = w.q[0]; Ug[1] = w.q[1]; Ug[2] = w.q[2]; Ug[3] = w.q[3];
    }
}

// IdealGas::pressure (euler.hpp:16-23)
__device__ __forceinline__ double pressure(const double* U, double g) {
    const double rho = U[0], u = U[1] / rho, v = U[2] / rho, E = U[3] / rho;
    return (g - 1.0) * rho * (E - 0.5 * (u * u + v * v));
}

// enforcePositivityKernel (kernels.cu:1236-1288): gamma fixed at 1.4; the
// clamped density is >= 0.01, so its 1e-10 floor never binds.
__device__ __forceinline__ void positivity(double* U) {
    const double rn = fmax(0.01, fmin(100.0, U[0]));
    const double ir = zj_rcp(rn);   // rn is in [0.01, 100]
    double u = U[1] * ir, v = U[2] * ir;
    const double vm = zj_sqrt(u * u + v * v);
    if (vm > 2000.0) { const double s = 2000.0 / vm; u *= s; v *= s; }
    const double ke = 0.5 * rn * (u * u + v * v);
    double p = (1.4 - 1.0) * (U[3] - ke);
    p = fmax(100.0, fmin(1e8, p));
    U[0] = rn; U[1] = rn * u; U[2] = rn * v; U[3] = p * (1.0 / (1.4 - 1.0)) + ke;
}

// -------------------------------------------------------------- kernels --

// Minimum resident CTAs per SM requested from the register allocator (per
// 256 threads, scaled to the CTA size).
#ifndef ZJ_MIN_BLOCKS
#define ZJ_MIN_BLOCKS 3
#endif
constexpr int kMinBlocks = ZJ_MIN_BLOCKS * kCtaScale;

template <int P>
__global__ void __launch_bounds__(Shape<P>::THREADS, kMinBlocks)
k_compat_stage(const StageArgs a) {
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
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous stage

    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < a.n_elem);
    const bool is_sp = valid && k < NSP;
    const bool is_fp = valid && k < NFT;
    const double g = a.gamma;
    const int edge = k / N1, fp = k - edge * N1;   // flux-point role
    const int i = k % N1, j = k / N1;              // solution-point role (xi, eta)

    // ---- A: independent global loads first; Euler fluxes into shared memory
    EdgeRec r{-1, 0, kEdgeOrphan, 0};
    double2 nr = make_double2(0.0, 0.0);
    double qo[4], qn[4] = {0.0, 0.0, 0.0, 0.0}, u[4];
    if (is_fp) {
        r = a.edges[e * 4 + edge];
        nr = __ldg(reinterpret_cast<const double2*>(a.enrm + e * 4 + edge));
        load4_nc(a.Tin + (e * NFT + k) * 4, qo);
    }
    if (is_sp) {
        const long long idx = e * NSP + k;
        gload4(a.U + idx * 4, u);
        if ((k & 3) == 0) {
            prefetch_l2(a.Jinv + idx * 4);
            if (a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        }
    }
    // Every flux point meets the neighbour's mirrored point N1-1-fp: both
    // elements run their shared edge counter-clockwise (kernels.cu:577).
    if (is_fp && !(r.flags & (kEdgeOrphan | kEdgeBoundary)))
        load4_nc(a.Tin + (((long long)r.nbr * 4 + r.nbr_edge) * N1 + (N1 - 1 - fp)) * 4, qn);
    if (is_sp) {
        const double ir = rcp_any(u[0]);
        const double uu = u[1] * ir, vv = u[2] * ir, E = u[3] * ir;
        const double p = (g - 1.0) * u[0] * (E - 0.5 * (uu * uu + vv * vv));
        double* f = sF + el * FS + j * RS + i;
        double* h = sG + el * FS + j * RS + i;
        f[0] = u[1]; f[VS] = u[1] * uu + p; f[2 * VS] = u[1] * vv; f[3 * VS] = (u[3] + p) * uu;
        h[0] = u[2]; h[VS] = u[2] * uu; h[2 * VS] = u[2] * vv + p; h[3 * VS] = (u[3] + p) * vv;
    }

    // ---- B: common flux of each face point, computed once per side.  A left
    // (or boundary) side owns the slot of its own point; a right side's point
    // fp produces the common flux of slot N1-1-fp (reference pairing: the left
    // trace at fp' with the right trace at N1-1-fp', used by the right side
    // at fp').  Slots hold sigma * Fc, sigma = +1 left, -1 right.
    double sig = 1.0, Fi[4] = {0.0, 0.0, 0.0, 0.0};
    if (is_fp) {
        const double nx = nr.x, ny = nr.y;
        double Fc[4] = {0.0, 0.0, 0.0, 0.0};
        int target = k;
        if (!(r.flags & kEdgeOrphan)) {
            Prim O, X;
            make_prim(qo, g, O);
            if (r.flags & kEdgeBoundary)
                ghost_compat(O, nx, ny, edge_bc_type(r.flags), a.bc + (long long)r.nbr_edge * 8, g, qn);
            make_prim(qn, g, X);
            // Left side: Rusanov(own, neighbour); right side: Rusanov(neighbour, own).
            const bool right = (r.flags & kEdgeRight) != 0;
            rusanov_pair(O, X, right, nx, ny, Fc);
            flux_normal(O, nx, ny, Fi);   // interior flux of this point (kernels.cu:389-424)
            sig = right ? -1.0 : 1.0;
            target = right ? edge * N1 + (N1 - 1 - fp) : k;
        }
        double c[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) c[v] = sig * Fc[v];
        store4(sD + el * DS + target * 4, c);
    }
    __syncthreads();   // sOps, sF, sG, common fluxes ready
    // Flux difference of this point: left Fc - Fi, right -Fc + Fi (kernels.cu:393-424).
    if (is_fp) {
        double* d = sD + el * DS + k * 4;
        double t[4];
        load4(d, t);
#pragma unroll
        for (int v = 0; v < 4; ++v) t[v] = t[v] - sig * Fi[v];
        store4(d, t);
    }
    __syncthreads();

    // ---- C: divergence, correction, stage update
    double rsq = 0.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        double ji[4], u0[4];
        load4_nc(a.Jinv + idx * 4, ji);
        if (a.stage >= 2) gload4(a.U0 + idx * 4, u0);
        double Di[N1], Dj[N1];
#pragma unroll
        for (int m = 0; m < N1; ++m) { Di[m] = sOps[i * N1 + m]; Dj[m] = sOps[j * N1 + m]; }
        const double* gL = sOps + N1 * N1 + 2 * N1;
        const double* gR = gL + N1;
        const double gLj = gL[j], gRi = gR[i], gRj = gR[j], gLi = gL[i];
        const double* f = sF + el * FS;
        const double* h = sG + el * FS;
        const double* d = sD + el * DS;
        double c0[4], c1[4], c2[4], c3[4];
        load4(d + (0 * N1 + i) * 4, c0);
        load4(d + (1 * N1 + j) * 4, c1);
        load4(d + (2 * N1 + i) * 4, c2);
        load4(d + (3 * N1 + j) * 4, c3);
        double res[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            double fr[N1], gr[N1];
            load_row<N1>(f + v * VS + j * RS, fr);
            load_row<N1>(h + v * VS + j * RS, gr);
            double dFdxi = 0.0, dFdeta = 0.0, dGdxi = 0.0, dGdeta = 0.0;
#pragma unroll
            for (int m = 0; m < N1; ++m) {
                dFdxi = fma(Di[m], fr[m], dFdxi);
                dFdeta = fma(Dj[m], f[v * VS + m * RS + i], dFdeta);
                dGdxi = fma(Di[m], gr[m], dGdxi);
                dGdeta = fma(Dj[m], h[v * VS + m * RS + i], dGdeta);
            }
            const double div = (dFdxi * ji[0] + dFdeta * ji[2]) + (dGdxi * ji[1] + dGdeta * ji[3]);
            double rr = -div;
            double corr = 0.0;
            corr += c0[v] * gLj;
            corr += c1[v] * gRi;
            corr += c2[v] * gRj;
            corr += c3[v] * gLi;
            rr -= corr;
            res[v] = rr;
        }
        if (a.stage == 0) {
            gstore4(a.R + idx * 4, res);
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
            positivity(uo);
            gstore4(a.Uout + idx * 4, uo);
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
        gstore4(a.Tout + (e * NFT + k) * 4, t);
    }
}

template <int P>
__global__ void __launch_bounds__(Shape<P>::THREADS)
k_traces(const double* __restrict__ U, double* __restrict__ T, const double* __restrict__ ops,
         long long n_elem) {
    using S = Shape<P>;
    constexpr int N1 = S::N1, NSP = S::NSP, NFT = S::NFT, TPE = S::TPE, EB = S::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = S::FS;
    __shared__ double sOps[S::NOPS];
    __shared__ double sU[EB * FS];
    const int tid = threadIdx.x;
    for (int i = tid; i < S::NOPS; i += blockDim.x) sOps[i] = ops[i];
    const int el = tid / TPE, k = tid - el * TPE;
    const long long e = (long long)blockIdx.x * EB + el;
    const bool valid = (el < EB) && (e < n_elem);
    if (valid && k < NSP) {
        double u[4];
        load4_nc(U + (e * NSP + k) * 4, u);
        double* su = sU + el * FS + (k / N1) * RS + (k % N1);
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = u[v];
    }
    __syncthreads();
    if (valid && k < NFT) {
        const int edge = k / N1, fp = k - edge * N1;
        double t[4];
        trace_point<N1, RS, VS>(sU + el * FS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
        gstore4(T + (e * NFT + k) * 4, t);
    }
}

__global__ void k_reduce_sum(const double* __restrict__ x, int n, double* out) {
    __shared__ double red[32];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += x[i];
    const double t = block_sum(s, red);
    if (threadIdx.x == 0) out[0] = t;
}

__global__ void k_dt_partial(const double* __restrict__ U, const double* __restrict__ h,
                             long long n_states, int n_sp, double g, double cfl, double cf,
                             double* partial, const int8_t* __restrict__ etype, int nt) {
    __shared__ double red[32];
    double m = 1e20;
    for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < n_states;
         s += (long long)gridDim.x * blockDim.x) {
        if (etype && etype[s / n_sp] == ZJ_ELEM_TRI && (int)(s % n_sp) >= nt) continue;   // unused slot
        double q[4];
        load4_nc(U + s * 4, q);
        const double u = q[1] / q[0], v = q[2] / q[0];
        const double vel = sqrt(u * u + v * v);
        const double p = fmax(pressure(q, g), 1e-10), rho = fmax(q[0], 1e-10);
        const double ws = vel + sqrt(g * p / rho);
        const double dl = cfl * h[s / n_sp] / (ws * cf);
        if (dl < m) m = dl;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 1e20;
        for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) r = fmin(r, red[i]);
        partial[blockIdx.x] = r;
    }
}

__global__ void k_min_reduce(const double* __restrict__ x, int n, double* out) {
    __shared__ double red[32];
    double m = 1e20;
    for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmin(m, x[i]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmin(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = 1e20;
        for (int i = 0; i < (int)((blockDim.x + 31) >> 5); ++i) r = fmin(r, red[i]);
        out[0] = r;
    }
}

__global__ void k_check_finite(const double* __restrict__ x, long long n, int* flag) {
    int bad = 0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        if (!isfinite(x[i])) bad = 1;
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

template <int P>
cudaError_t launch_stage_t(const StageArgs& a, cudaStream_t s, int* grid_out) {
    using S = Shape<P>;
    const long long grid = (a.n_elem + S::EB - 1) / S::EB;
    if (grid_out) *grid_out = (int)grid;
    if (grid <= 0) return cudaSuccess;
    // Prefer the largest shared-memory carveout so kMinBlocks CTAs fit per SM.
    static bool carveout_set = false;
    if (!carveout_set) {
        cudaFuncSetAttribute(k_compat_stage<P>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        carveout_set = true;
    }
    return launch_programmatic(k_compat_stage<P>, (unsigned)grid, S::THREADS, s, a);
}

template <int P>
cudaError_t launch_traces_t(const double* U, double* T, const double* ops, long long n, cudaStream_t s) {
    using S = Shape<P>;
    const long long grid = (n + S::EB - 1) / S::EB;
    if (grid <= 0) return cudaSuccess;
    k_traces<P><<<(unsigned)grid, S::THREADS, 0, s>>>(U, T, ops, n);
    return cudaGetLastError();
}

template <int P>
int grid_t(long long n) { return (int)((n + Shape<P>::EB - 1) / Shape<P>::EB); }

}  // namespace

int stage_grid(int P, long long n_elem) {
    switch (P) {
        case 1: return grid_t<1>(n_elem);
        case 2: return grid_t<2>(n_elem);
        case 3: return grid_t<3>(n_elem);
        case 4: return grid_t<4>(n_elem);
        case 5: return grid_t<5>(n_elem);
        default: return 0;
    }
}

cudaError_t launch_compat_stage(int P, const StageArgs& a, cudaStream_t s, int* grid_out) {
    switch (P) {
        case 1: return launch_stage_t<1>(a, s, grid_out);
        case 2: return launch_stage_t<2>(a, s, grid_out);
        case 3: return launch_stage_t<3>(a, s, grid_out);
        case 4: return launch_stage_t<4>(a, s, grid_out);
        case 5: return launch_stage_t<5>(a, s, grid_out);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_traces(int P, const double* U, double* T, const double* ops, long long n,
                          cudaStream_t s) {
    switch (P) {
        case 1: return launch_traces_t<1>(U, T, ops, n, s);
        case 2: return launch_traces_t<2>(U, T, ops, n, s);
        case 3: return launch_traces_t<3>(U, T, ops, n, s);
        case 4: return launch_traces_t<4>(U, T, ops, n, s);
        case 5: return launch_traces_t<5>(U, T, ops, n, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_reduce_sum(const double* partials, int n, double* out, cudaStream_t s) {
    k_reduce_sum<<<1, 1024, 0, s>>>(partials, n, out);
    return cudaGetLastError();
}

cudaError_t launch_compute_dt(const double* U, const double* h, long long n_elem, int n_sp,
                              double gamma, double cfl, int P, double* scratch, int scratch_n,
                              double* out, cudaStream_t s, const int8_t* etype, int nt) {
    const long long n_states = n_elem * n_sp;
    int blocks = (int)((n_states + 255) / 256);
    if (blocks > scratch_n) blocks = scratch_n;
    if (blocks < 1) blocks = 1;
    k_dt_partial<<<blocks, 256, 0, s>>>(U, h, n_states, n_sp, gamma, cfl, 2.0 * P + 1.0, scratch, etype, nt);
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return err;
    k_min_reduce<<<1, 1024, 0, s>>>(scratch, blocks, out);
    return cudaGetLastError();
}

cudaError_t launch_check_finite(const double* x, long long n, int* flag, cudaStream_t s) {
    cudaError_t err = cudaMemsetAsync(flag, 0, sizeof(int), s);
    if (err != cudaSuccess) return err;
    long long blocks = (n + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    if (blocks < 1) blocks = 1;
    k_check_finite<<<(unsigned)blocks, 256, 0, s>>>(x, n, flag);
    return cudaGetLastError();
}

}  // namespace zj
