// ns_tc.cu -- the split-BF16 form of the Navier-Stokes stage kernel at P4
// and P5 (precision split_bf16): the same scheme as k_ns_stage<P, RIEM,
// float> (ns_kernels.cuh), with its largest operator product on the tensor
// cores.
//
// Per block of EB = 8 elements one matrix product gives, for every element
// and variable (N = 32 columns), the divergence D_xi F~ + D_eta G~ at the
// n_sp solution points and the traces of the transformed flux normal to each
// edge at the 4 (P+1) flux points:
//   [div; Fn] (M = 64 rows, n_sp + 4(P+1) used) =
//       A (the reference's dense operators diff_xi | diff_eta and the edge
//          rows of interp, basis.cpp:503-569, as one M x 2 n_sp matrix)
//     x B (F~ then G~ of the block, 2 n_sp x 32).
// Both factors are split into BF16 pairs x = hi + lo (hi = bf16(x),
// lo = bf16(x - hi)) and multiplied as three products Al Bh + Ah Bl + Ah Bh
// (the Al Bl term, 2^-16 relative, is dropped), accumulated in FP32 in
// tensor memory by tcgen05.mma (kind::f16, M = 64, N = 32, K = 16 per
// instruction).  A is built once on the host from the FP64 operators and
// reaches each CTA's shared memory through a TMA tensor copy
// (cp.async.bulk.tensor.2d); B is written by the solution-point threads.
// The element's Riemann and viscous face fluxes are evaluated while the
// tensor cores run; the FP64 state, the SSP-RK3 update and the norm partials
// are those of the precision form.
#include <cuda.h>
#include <cuda_bf16.h>

#include "ns_kernels.cuh"
#include "zj_tc.cuh"

namespace zj {
namespace {

using namespace dev;
using namespace phys;

template <int P>
struct TcShape {
    static constexpr int N1 = P + 1, NSP = N1 * N1, NFT = 4 * N1;
    static constexpr int EB = 8;                      // elements per CTA
    static constexpr int TPE = NSP;                   // >= NFT from P3 up
    static constexpr int THREADS = EB * TPE;          // 288 at P5, 200 at P4
    static constexpr int K = 2 * NSP;                 // F~ then G~
    static constexpr int KP = (K + 15) / 16 * 16;     // 80 at P5, 64 at P4
    static constexpr int KSTEPS = KP / 16;
    static constexpr int M = 64;
    static constexpr int N = EB * 4;                  // 32
    static constexpr int A_LBO = M * 16;              // operator image: chunk stride
    static constexpr int A_TERM = (KP / 8) * A_LBO;   // one BF16 term of A
    static constexpr int B_LBO = N * 16 + 16;         // padded: chunks on distinct banks
    static constexpr int B_TERM = (KP / 8) * B_LBO;
    static constexpr int RS_ = N + 4;                 // result tile row stride (floats)
    static constexpr int A_ROWS16 = 2 * A_TERM / 16;  // 16-byte rows of the TMA image
    static_assert(NSP + NFT <= M, "divergence and edge rows fit one M = 64 tile");
    static_assert(A_ROWS16 % 256 == 0, "whole TMA boxes");
};

constexpr int kWaitPolls = 1 << 20;   // bounded mbarrier waits

template <int P>
struct TcSmem {
    using C = TcShape<P>;
    using S = Shape<P>;
    static constexpr int FS = Tiles<P, float>::FS, DS = Tiles<P, float>::DS;
    static constexpr size_t A_OFF = 0;
    static constexpr size_t B_OFF = A_OFF + 2 * C::A_TERM;
    static constexpr size_t R_OFF = B_OFF + 2 * C::B_TERM;
    static constexpr size_t OPS_OFF = R_OFF + sizeof(float) * C::M * C::RS_;
    static constexpr size_t U_OFF = OPS_OFF + sizeof(float) * ((S::NOPS + 3) & ~3);
    static constexpr size_t D_OFF = U_OFF + sizeof(float) * C::EB * FS;
    static constexpr size_t RED_OFF = (D_OFF + sizeof(float) * C::EB * DS + 7) & ~size_t(7);
    static constexpr size_t BAR_OFF = RED_OFF + sizeof(double) * 32;
    static constexpr size_t SLOT_OFF = BAR_OFF + 2 * sizeof(uint64_t);
    static constexpr size_t BYTES = SLOT_OFF + 16;
};

// BF16 bits of finite x rounded to nearest even, by integer arithmetic on the
// ALU pipe (the float-to-BF16 conversion instruction runs on the XU pipe,
// which the kernel's reciprocals and square roots already load).
__device__ __forceinline__ uint32_t bf16_bits_rn(float x) {
    const uint32_t u = __float_as_uint(x);
    return (u + 0x7FFFu + ((u >> 16) & 1u)) >> 16;
}

// x = hi + lo + r, |r| <= 2^-18 |x|: hi the nearest BF16 to x, lo the nearest
// to the (exact) FP32 remainder x - hi.
__device__ __forceinline__ void split_bf16(float x, unsigned short& hi, unsigned short& lo) {
    const uint32_t h = bf16_bits_rn(x);
    hi = static_cast<unsigned short>(h);
    lo = static_cast<unsigned short>(bf16_bits_rn(x - __uint_as_float(h << 16)));
}

template <int P, int RIEM>
__global__ void __launch_bounds__(TcShape<P>::THREADS, 3)
k_ns_stage_tc(const StageArgsT<float> a, const __grid_constant__ CUtensorMap amap) {
    using S = Shape<P>;
    using C = TcShape<P>;
    using L = TcSmem<P>;
    constexpr int N1 = C::N1, NSP = C::NSP, NFT = C::NFT, TPE = C::TPE, EB = C::EB;
    constexpr int RS = S::RS, VS = S::VS, FS = L::FS, DS = L::DS;
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sA = smem + L::A_OFF;
    unsigned char* sB = smem + L::B_OFF;
    float* sR = reinterpret_cast<float*>(smem + L::R_OFF);
    float* sOps = reinterpret_cast<float*>(smem + L::OPS_OFF);
    float* sU = reinterpret_cast<float*>(smem + L::U_OFF);
    float* sD = reinterpret_cast<float*>(smem + L::D_OFF);
    double* sRed = reinterpret_cast<double*>(smem + L::RED_OFF);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + L::BAR_OFF);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + L::SLOT_OFF);
    const uint32_t bar_tma = tc::smem_u32(&bars[0]), bar_mma = tc::smem_u32(&bars[1]);

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (warp == 0) tc::tmem_alloc(tc::smem_u32(slot), 32);
    if (tid == 0) {
        tc::mbar_init(bar_tma, 1);
        tc::mbar_init(bar_mma, 1);
        tc::fence_mbar_init();
    }
    // the padded K rows of B must be zeros (A is zero there, and 0 * NaN of
    // stale shared memory would not be)
    for (int t = tid; t < 2 * C::B_TERM / 16; t += blockDim.x)
        reinterpret_cast<uint4*>(sB)[t] = make_uint4(0u, 0u, 0u, 0u);
    for (int t = tid; t < S::NOPS; t += blockDim.x) sOps[t] = a.ops[t];
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem_d = *slot;
    if (tid == 0) {
        // the operator image (both BF16 terms) by TMA, 256 rows of 16 bytes a box
        tc::mbar_expect_tx(bar_tma, 2 * C::A_TERM);
        for (int r = 0; r < C::A_ROWS16; r += 256) tc::tma_load_2d(tc::smem_u32(sA + r * 16), &amap, 0, r, bar_tma);
    }
    pdl_launch_dependents();
    pdl_wait();   // the state and traces come from the previous stage

    const int el = tid / TPE, k = tid - el * TPE;
    const long long e0 = (long long)blockIdx.x * EB;
    const long long e = e0 + el;
    const bool valid = e < a.n_elem;
    const bool is_sp = valid && k < NSP, is_fp = valid && k < NFT;
    const float g = float(a.gamma);
    const int edge = k / N1, fp = k - edge * N1;
    const int i = k % N1, j = k / N1;

    // ---- A1: loads, face jumps, stage state into shared memory
    FacePoint<float> f;
    f.r = EdgeRec{-1, 0, kEdgeOrphan, 0};
    float Qo[8], Qn[8];
    if (is_fp) {
        load_face_point<N1>(a, e, edge, fp, f);
        const float* qt = a.TQ + (e * NFT + k) * 8;
        gload8_nc(qt, Qo);
#pragma unroll
        for (int v = 0; v < 8; ++v) Qn[v] = Qo[v];
        if (has_neighbour_gradient(f.r)) {
            const float* qn = a.TQ + (neighbour_row(f.r, a.n_elem) * N1 + (N1 - 1 - fp)) * 8;
            gload8_nc(qn, Qn);
        }
        float d[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) d[v] = (f.r.flags & kEdgeOrphan) ? 0.f : 0.5f * (f.qn[v] - f.qo[v]);
        store4(sD + el * DS + k * 4, d);
    }
    float ue[4] = {0.f, 0.f, 0.f, 0.f};   // the element's reference state
    if (valid) load_state(a.U + e * NSP * 4, ue);
    float u[4], ji[4], Jd = 1.f;
    if (is_sp) {
        const long long idx = e * NSP + k;
        double ud[4];
        stage_state(a, idx, ud, u);
        load4_nc(a.Jinv + idx * 4, ji);
        Jd = ldg_any(a.J + idx);
        if ((k & 3) == 0 && a.stage >= 2) prefetch_l2(a.U0 + idx * 4);
        float w[4];
        state_minus_ref(ud, ue, w);
        float* su = sU + el * FS + j * RS + i;
#pragma unroll
        for (int v = 0; v < 4; ++v) su[v * VS] = w[v];
    }
    __syncthreads();

    // ---- A2: gradient, total transformed fluxes as the BF16 pairs of B
    if (is_sp) {
        float Qx[4], Qy[4], Fv[4], Gv[4];
        corrected_gradient<N1, RS, VS>(sU + el * FS, sD + el * DS, sOps, i, j, ji, Qx, Qy);
        const float ir = rcp_any(u[0]);
        viscous_flux_f(u, ir, Qx, Qy, g, inv_reynolds(a), float(a.kfac), Fv, Gv);
        float F[4], G[4], Fe[4], Ge[4];
        euler_flux_ir(u, ir, g, F, G);
        euler_flux(ue, g, Fe, Ge);
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float Fx = F[v] - Fe[v] - Fv[v], Gy = G[v] - Ge[v] - Gv[v];
            const float ft = Jd * (ji[0] * Fx + ji[1] * Gy);   // F~
            const float gt = Jd * (ji[2] * Fx + ji[3] * Gy);   // G~
            const int n = el * 4 + v;
            unsigned short h, l;
            // F~ at K = k, G~ at K = NSP + k; term 0 = hi, term 1 = lo
            const int kf = k, kg = NSP + k;
            unsigned char* pf = sB + (kf >> 3) * C::B_LBO + n * 16 + (kf & 7) * 2;
            unsigned char* pg = sB + (kg >> 3) * C::B_LBO + n * 16 + (kg & 7) * 2;
            split_bf16(ft, h, l);
            *reinterpret_cast<unsigned short*>(pf) = h;
            *reinterpret_cast<unsigned short*>(pf + C::B_TERM) = l;
            split_bf16(gt, h, l);
            *reinterpret_cast<unsigned short*>(pg) = h;
            *reinterpret_cast<unsigned short*>(pg + C::B_TERM) = l;
        }
    }
    tc::fence_proxy_async();
    __syncthreads();   // B complete; the face jumps in sD and the state tile are dead

    bool ok = true;
    if (tid == 0) {
        tc::fence_after_sync();
        ok = tc::mbar_wait(bar_tma, 0, kWaitPolls);   // the operator image has landed
        if (ok) {
            constexpr uint32_t idesc = tc::idesc_bf16_f32(C::M, C::N);
            const uint32_t a0 = tc::smem_u32(sA), b0 = tc::smem_u32(sB);
            // (A term, B term): lo x hi, hi x lo, then hi x hi
            const int ta[3] = {1, 0, 0}, tb[3] = {0, 1, 0};
            uint32_t acc = 0;
#pragma unroll
            for (int t = 0; t < 3; ++t)
#pragma unroll
                for (int s2 = 0; s2 < C::KSTEPS; ++s2) {
                    const uint64_t ad = tc::smem_desc(a0 + ta[t] * C::A_TERM + 2 * s2 * C::A_LBO, C::A_LBO, 128);
                    const uint64_t bd = tc::smem_desc(b0 + tb[t] * C::B_TERM + 2 * s2 * C::B_LBO, C::B_LBO, 128);
                    tc::mma_bf16(tmem_d, ad, bd, idesc, acc);
                    acc = 1;
                }
            tc::mma_commit(bar_mma);
        }
    }

    // ---- B1: the common flux of each flux point while the MMAs run
    float Fc[4] = {0.f, 0.f, 0.f, 0.f};
    const bool face = is_fp && !(f.r.flags & kEdgeOrphan);
    const bool right = (f.r.flags & kEdgeRight) != 0;
    if (face) {
        float UL[4], UR[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) { UL[v] = right ? f.qn[v] : f.qo[v]; UR[v] = right ? f.qo[v] : f.qn[v]; }
        riemann<RIEM>(UL, UR, f.nx, f.ny, g, Fc);
        float Fe[4];
        ref_flux_n(ue, g, f.nx, f.ny, Fe);
        float Ua[4], dxa[4], dya[4], Fv[4], Gv[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            Fc[v] -= Fe[v];
            Ua[v] = 0.5f * (UL[v] + UR[v]);
            dxa[v] = 0.5f * (Qo[v] + Qn[v]);
            dya[v] = 0.5f * (Qo[4 + v] + Qn[4 + v]);
        }
        viscous_flux_f(Ua, rcp_any(Ua[0]), dxa, dya, g, inv_reynolds(a), float(a.kfac), Fv, Gv);
        float Fvn[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) Fvn[v] = Fv[v] * f.nx + Gv[v] * f.ny;
        boundary_viscous_closure(f.r, a.bc, f.nx, f.ny, Fvn);
#pragma unroll
        for (int v = 0; v < 4; ++v) Fc[v] -= Fvn[v];
    }

    // ---- the product: tensor memory -> the result tile (rows 16q..16q+15 sit
    // in lanes 32q..32q+15 for M = 64)
    ok = __syncthreads_and(ok);
    bool done = ok && tc::mbar_wait(bar_mma, 0, kWaitPolls);
    done = __syncthreads_and(done);
    tc::fence_after_sync();
    if (done && warp < 4) {
        float r[32];
        tc::tmem_ld32(tmem_d + (static_cast<uint32_t>(32 * warp) << 16), r);
        if (lane < 16) {
            float4* row = reinterpret_cast<float4*>(sR + (16 * warp + lane) * C::RS_);
#pragma unroll
            for (int c = 0; c < 8; ++c) row[c] = make_float4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
        }
    }
    if (!done && tid == 0 && a.tc_err) atomicExch(a.tc_err, 1);
    tc::fence_before_sync();
    __syncthreads();

    // ---- B2: flux differences with the edge traces of the product
    if (is_fp) {
        float Fd[4] = {0.f, 0.f, 0.f, 0.f};
        if (face) {
            const float ss = right ? -0.5f * f.len : 0.5f * f.len;
            const float4 tn = *reinterpret_cast<const float4*>(sR + (NSP + k) * C::RS_ + el * 4);
            const float Fn[4] = {tn.x, tn.y, tn.z, tn.w};
            const float sgn = (edge == 0 || edge == 3) ? -1.f : 1.f;
#pragma unroll
            for (int v = 0; v < 4; ++v) Fd[v] = ss * Fc[v] - sgn * Fn[v];
        }
        store4(sD + el * DS + k * 4, Fd);
    }
    __syncthreads();

    // ---- C: divergence (the product), VCJH correction, 1/J, stage update
    double rsq = 0.0;
    if (is_sp) {
        const long long idx = e * NSP + k;
        double u0[4];
        if (a.stage >= 2) gload4(a.U0 + idx * 4, u0);
        const float* gL = sOps + N1 * N1 + 2 * N1;
        const float* gR = gL + N1;
        const float gRi = gR[i], gLi = gL[i], gRj = gR[j], gLj = gL[j];
        const float* d = sD + el * DS;
        float c1[4], c3[4], c2[4], c0[4];
        load4(d + (1 * N1 + j) * 4, c1);
        load4(d + (3 * N1 + (N1 - 1 - j)) * 4, c3);
        load4(d + (2 * N1 + (N1 - 1 - i)) * 4, c2);
        load4(d + (0 * N1 + i) * 4, c0);
        const float4 dv = *reinterpret_cast<const float4*>(sR + k * C::RS_ + el * 4);
        const float div[4] = {dv.x, dv.y, dv.z, dv.w};
        const float iJ = rcp_any(Jd);
        float res[4];
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const float corr = gRi * c1[v] - gLi * c3[v] + gRj * c2[v] - gLj * c0[v];
            res[v] = -(div[v] + corr) * iJ;
        }
        if (a.stage == 0) {
            store_residual(a, idx, res, rsq);
        } else {
            double us[4];
            gload4(a.U + idx * 4, us);
            double uo[4];
            rk_update(a.stage, *a.dt, us, u0, res, uo);
            gstore4(a.Uout + idx * 4, uo);
            float un[4];
            state_minus_ref(uo, ue, un);
            float* su = sU + el * FS + j * RS + i;
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
    __syncthreads();

    // ---- D: traces of the new state
    if (a.stage != 0 && is_fp) {
        float t[4];
        trace_point<N1, RS, VS>(sU + el * FS, sOps + N1 * N1, sOps + N1 * N1 + N1, edge, fp, t);
#pragma unroll
        for (int v = 0; v < 4; ++v) t[v] += ue[v];
        gstore4(a.Tout + (e * NFT + k) * 4, t);
        if (boundary_condition_edge(f.r)) store_ghost<N1>(a, f.r, f.nx, f.ny, fp, t);
    }

    // ---- teardown: every copy and product has completed (or the waits gave
    // up: then wait once more, bounded, before the memory goes back)
    if (!done && tid == 0) {
        tc::mbar_wait(bar_tma, 0, kWaitPolls);
        if (ok) tc::mbar_wait(bar_mma, 0, kWaitPolls);
    }
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem_d, 32);
    }
}

template <int P, int RIEM>
cudaError_t ns_stage_tc_t(const StageArgs32& a, const CUtensorMap& amap, cudaStream_t s) {
    using C = TcShape<P>;
    const long long grid = (a.n_elem + C::EB - 1) / C::EB;
    if (grid <= 0) return cudaSuccess;
    static bool set = false;
    if (!set) {
        cudaError_t e = cudaFuncSetAttribute(k_ns_stage_tc<P, RIEM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)TcSmem<P>::BYTES);
        if (e != cudaSuccess) return e;
        set = true;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3(C::THREADS);
    cfg.dynamicSmemBytes = TcSmem<P>::BYTES;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_ns_stage_tc<P, RIEM>, a, amap);
}

template <int P>
cudaError_t ns_stage_tc_p(int riemann, const StageArgs32& a, const CUtensorMap& amap, cudaStream_t s) {
    switch (riemann) {
        case ZJ_RIEMANN_RUSANOV: return ns_stage_tc_t<P, ZJ_RIEMANN_RUSANOV>(a, amap, s);
        case ZJ_RIEMANN_ROE: return ns_stage_tc_t<P, ZJ_RIEMANN_ROE>(a, amap, s);
        case ZJ_RIEMANN_HLLC: return ns_stage_tc_t<P, ZJ_RIEMANN_HLLC>(a, amap, s);
        default: return cudaErrorInvalidValue;
    }
}

// Host image of A for order P: [term hi, lo][chunk K/8][row M][8] BF16, rows
// 0..n_sp-1 the divergence of solution point k = j n1 + i (D1[i][m] at
// K = j n1 + m on F~, D1[j][m] at K = n_sp + m n1 + i on G~), rows
// n_sp + edge n1 + fp the edge traces in trace_point's order (edge 0: Lm on
// G~ column fp; 1: Lp on F~ row fp; 2: Lp on G~ column n1-1-fp; 3: Lm on F~
// row n1-1-fp).
template <int P>
void build_image(const Operators1D& o, std::vector<uint16_t>& img) {
    using C = TcShape<P>;
    constexpr int N1 = C::N1, NSP = C::NSP;
    std::vector<double> A((size_t)C::M * C::KP, 0.0);
    auto at = [&](int r, int kk) -> double& { return A[(size_t)r * C::KP + kk]; };
    for (int j = 0; j < N1; ++j)
        for (int i = 0; i < N1; ++i) {
            const int r = j * N1 + i;
            for (int m = 0; m < N1; ++m) {
                at(r, j * N1 + m) += o.D1[(size_t)i * N1 + m];
                at(r, NSP + m * N1 + i) += o.D1[(size_t)j * N1 + m];
            }
        }
    for (int fp = 0; fp < N1; ++fp)
        for (int m = 0; m < N1; ++m) {
            at(NSP + 0 * N1 + fp, NSP + m * N1 + fp) = o.Lm[(size_t)m];
            at(NSP + 1 * N1 + fp, fp * N1 + m) = o.Lp[(size_t)m];
            at(NSP + 2 * N1 + fp, NSP + m * N1 + (N1 - 1 - fp)) = o.Lp[(size_t)m];
            at(NSP + 3 * N1 + fp, (N1 - 1 - fp) * N1 + m) = o.Lm[(size_t)m];
        }
    img.assign((size_t)2 * C::A_TERM / 2, 0);
    for (int r = 0; r < C::M; ++r)
        for (int kk = 0; kk < C::KP; ++kk) {
            const double x = at(r, kk);
            const __nv_bfloat16 hi = __double2bfloat16(x);
            const __nv_bfloat16 lo = __double2bfloat16(x - (double)__bfloat162float(hi));
            const size_t off = (size_t)(kk >> 3) * (C::A_LBO / 2) + (size_t)r * 8 + (kk & 7);
            img[off] = __bfloat16_as_ushort(hi);
            img[(size_t)C::A_TERM / 2 + off] = __bfloat16_as_ushort(lo);
        }
}

}  // namespace

bool tc_order_supported(int P) { return P == 4 || P == 5; }

int tc_grid(int P, long long n) {
    return (int)((n + TcShape<4>::EB - 1) / TcShape<4>::EB);   // EB = 8 at P4 and P5
}

bool build_tc_image(int P, const Operators1D& o, std::vector<uint16_t>& img) {
    if (P == 4) { build_image<4>(o, img); return true; }
    if (P == 5) { build_image<5>(o, img); return true; }
    return false;
}

// Tensor map of the operator image: a 2-D BF16 tensor of 8 x rows (16-byte
// rows), boxes of 8 x 256; cuTensorMapEncodeTiled from the driver through
// the runtime's entry-point query.
cudaError_t make_tc_tensor_map(int P, const void* dev_img, void* map_out) {
    const int rows = (P == 4) ? TcShape<4>::A_ROWS16 : TcShape<5>::A_ROWS16;
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    void* fn = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    cudaError_t e = cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q);
    if (e != cudaSuccess) return e;
    if (!fn || q != cudaDriverEntryPointSuccess) return cudaErrorNotSupported;
    const cuuint64_t dims[2] = {8, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {16};
    const cuuint32_t box[2] = {8, 256};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = reinterpret_cast<Encode>(fn)(static_cast<CUtensorMap*>(map_out), CU_TENSOR_MAP_DATA_TYPE_BFLOAT16,
                                               2, const_cast<void*>(dev_img), dims, strides, box, estr,
                                               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                               CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_ns_stage_tc(int P, int riemann, const StageArgs32& a, const void* map, cudaStream_t s) {
    const CUtensorMap& m = *static_cast<const CUtensorMap*>(map);
    switch (P) {
        case 4: return ns_stage_tc_p<4>(riemann, a, m, s);
        case 5: return ns_stage_tc_p<5>(riemann, a, m, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace zj
