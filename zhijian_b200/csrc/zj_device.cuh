// zj_device.cuh -- device helpers shared by the residual kernels: CTA shape
// of an element block, vectorised global/shared accesses, the branch-free
// trace of a flux point, block reductions.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

#include "zj_math.h"

namespace zj {
namespace dev {

// Threads per CTA of the element-block kernels (rounded down to whole
// elements).  128-thread CTAs interleave the load, shared-memory and
// arithmetic phases of more blocks per SM than 256-thread ones (measured on
// the Navier-Stokes residual at P3: 4-6% faster); launch bounds scale their
// minimum resident blocks with it (kCtaScale), so the register limits per
// thread stay those of the 256-thread tuning.
#ifndef ZJ_CTA_THREADS
#define ZJ_CTA_THREADS 128
#endif
constexpr int kCtaThreads = ZJ_CTA_THREADS;
constexpr int kCtaScale = 256 / ZJ_CTA_THREADS;

// EBDIV > 1 packs fewer elements per CTA: the dual-number instantiation
// (16-byte values) uses EBDIV = 3 so its shared tiles stay within the 48 KB
// of static shared memory.
template <int P, int EBDIV = 1>
struct Shape {
    static constexpr int N1 = P + 1;
    static constexpr int NSP = N1 * N1;
    static constexpr int NFT = 4 * N1;                 // flux points per element
    static constexpr int TPE = NSP > NFT ? NSP : NFT;  // threads per element
    static constexpr int EB = (kCtaThreads / TPE / EBDIV) > 0 ? (kCtaThreads / TPE / EBDIV) : 1;
    static constexpr int THREADS = EB * TPE;
    static constexpr int NOPS = N1 * N1 + 4 * N1;
    // Shared-memory layout of per-element fields (doubles): [var][eta row][xi]
    // with rows padded to an even length so every row starts 16-byte aligned
    // (vector loads), and a per-element stride of 6 mod 16 so the elements
    // that share a warp start on different banks.  Flux differences use
    // [flux point][var] with a per-element stride of 2 mod 16.
    static constexpr int RS = (N1 + 1) & ~1;
    static constexpr int VS = N1 * RS;
    static constexpr int FS = 4 * VS + (6 - (4 * VS) % 16 + 16) % 16;
    static constexpr int DS = 4 * NFT + 2;
};

template <typename T>
struct EbDiv { static constexpr int value = sizeof(T) > 8 ? 3 : 1; };

__device__ __forceinline__ void load4(const double* p, double* v) {
    const double2 a = *reinterpret_cast<const double2*>(p);
    const double2 b = *reinterpret_cast<const double2*>(p + 2);
    v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}
// Global rows of four doubles: one 32-byte access per thread (sm_100
// ld/st .v4.f64), so a warp's request covers each 32-byte sector once; two
// 16-byte accesses fetch the same sectors twice.  The rows are 32-byte
// aligned: the library's buffers come from cudaMalloc with every row at a
// multiple of 32 bytes, and the entry points refuse caller arrays that are
// not 32-byte aligned.
__device__ __forceinline__ void load4_nc(const double* p, double* v) {
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3]) : "l"(p));
}
__device__ __forceinline__ void gload4(const double* p, double* v) {
    asm volatile("ld.global.v4.f64 {%0, %1, %2, %3}, [%4];"
                 : "=d"(v[0]), "=d"(v[1]), "=d"(v[2]), "=d"(v[3])
                 : "l"(p)
                 : "memory");
}
__device__ __forceinline__ void gstore4(double* p, const double* v) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};" ::"l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3])
                 : "memory");
}
// Eight values (a gradient-trace point): two 32-byte accesses.
__device__ __forceinline__ void gload8_nc(const double* p, double* v) {
    load4_nc(p, v);
    load4_nc(p + 4, v + 4);
}
__device__ __forceinline__ void gstore8(double* p, const double* v) {
    gstore4(p, v);
    gstore4(p + 4, v + 4);
}
__device__ __forceinline__ void store4(double* p, const double* v) {
    *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}

// FP32 twins (the mixed-precision kernels' traces, metrics and tiles).
__device__ __forceinline__ void load4(const float* p, float* v) {
    const float4 a = *reinterpret_cast<const float4*>(p);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void load4_nc(const float* p, float* v) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(p));
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
}
__device__ __forceinline__ void store4(float* p, const float* v) {
    *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
}
// Global float rows: four values are one 16-byte access; eight (a gradient
// trace point, 32-byte aligned like the double rows) one 32-byte access.
__device__ __forceinline__ void gstore4(float* p, const float* v) { store4(p, v); }
__device__ __forceinline__ void gload8_nc(const float* p, float* v) {
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7])
        : "l"(p));
}
__device__ __forceinline__ void gstore8(float* p, const float* v) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "f"(v[0]), "f"(v[1]),
                 "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
}

__device__ __forceinline__ double ldg_any(const double* p) { return __ldg(p); }
__device__ __forceinline__ float ldg_any(const float* p) { return __ldg(p); }

// (nx, ny, len) of an edge-normal record.
__device__ __forceinline__ void load_normal(const double4* p, double* n) {
    double pad;
    asm("ld.global.nc.v4.f64 {%0, %1, %2, %3}, [%4];" : "=d"(n[0]), "=d"(n[1]), "=d"(n[2]), "=d"(pad) : "l"(p));
}
__device__ __forceinline__ void load_normal(const float4* p, float* n) {
    const float4 a = __ldg(p);
    n[0] = a.x; n[1] = a.y; n[2] = a.z;
}

// 1/x: Newton-Raphson for positive normal x, IEEE division otherwise (zero,
// negative or non-finite densities, which the reference also divides by).
__device__ __forceinline__ double rcp_any(double x) {
    return (x > 1e-300 && x < 1e300) ? zj_rcp(x) : 1.0 / x;
}

// FP32 (the mixed-precision form): the hardware's approximate reciprocal and
// square root (rcp.approx / sqrt.approx, within 1-2 ulp of float), whose
// error sits at the FP32 rounding level the form already carries.
__device__ __forceinline__ float rcp_any(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ double sqrt_any(double a) { return zj_sqrt(a); }
__device__ __forceinline__ float sqrt_any(float a) {
    float y;
    asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    return y;
}
// Correctly rounded square root (the reference's sqrt where it is not on a
// hot path).
__device__ __forceinline__ double sqrt_ieee(double a) { return sqrt(a); }
__device__ __forceinline__ float sqrt_ieee(float a) { return sqrtf(a); }
// a / b: IEEE division in FP64, a * (1/b) in FP32.
__device__ __forceinline__ double div_any(double a, double b) { return a / b; }
__device__ __forceinline__ float div_any(float a, float b) { return a * rcp_any(b); }
__device__ __forceinline__ double pow_any(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float pow_any(float a, float b) { return __powf(a, b); }
// T^0.7 of the viscosity law: the series routine of zj_math.h in FP64 (within
// 2 ulp of pow(T, 0.7)), the hardware exp2/log2 form in FP32.
__device__ __forceinline__ double visc_pow(double t) { return zj_pow07(t); }
__device__ __forceinline__ float visc_pow(float t) { return __powf(t, 0.7f); }
__device__ __forceinline__ double fma_any(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float fma_any(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double max_any(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float max_any(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ double abs_any(double a) { return fabs(a); }
__device__ __forceinline__ float abs_any(float a) { return fabsf(a); }

__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// N values of a 16-byte aligned shared-memory row, with 16-byte loads.
template <int N>
__device__ __forceinline__ void load_row(const float* row, float* out) {
#pragma unroll
    for (int m = 0; m + 1 < N; m += 2) {
        const float2 t = *reinterpret_cast<const float2*>(row + m);
        out[m] = t.x;
        out[m + 1] = t.y;
    }
    if (N & 1) out[N - 1] = row[N - 1];
}
template <int N>
__device__ __forceinline__ void load_row(const double* row, double* out) {
#pragma unroll
    for (int m = 0; m + 1 < N; m += 2) {
        const double2 t = *reinterpret_cast<const double2*>(row + m);
        out[m] = t.x;
        out[m + 1] = t.y;
    }
    if (N & 1) out[N - 1] = row[N - 1];
}

// Row r of an N1 x N1 operator in a 16-byte aligned table: vector loads
// when every row starts on a 16-byte boundary, scalar ones otherwise.
template <int N1, typename T>
__device__ __forceinline__ void load_op_row(const T* op, int r, T* out) {
    if constexpr ((std::is_same<T, float>::value || std::is_same<T, double>::value) &&
                  (N1 * sizeof(T)) % 16 == 0) {
        load_row<N1>(op + r * N1, out);
    } else {
#pragma unroll
        for (int m = 0; m < N1; ++m) out[m] = op[r * N1 + m];
    }
}

// Trace of one flux point from a state held in shared memory as
// s[var*VS + j*RS + i] (i: xi index, j: eta index).  Edge parametrisations
// follow FROperators::initQuad (basis.cpp:540-552): edges 0,1 run with +s,
// edges 2,3 with -s, so fp on edges 2,3 meets xi/eta index N1-1-fp.  The sum
// runs over the index the reference's dense row has nonzero weights on,
// ascending:  edge 0: sum_j l_j(-1) s[j][fp]     edge 1: sum_i l_i(1) s[fp][i]
//             edge 2: sum_j l_j(1) s[j][N1-1-fp] edge 3: sum_i l_i(-1) s[N1-1-fp][i]
// Written without branches on the edge (the four edges share a warp).
template <int N1, int RS, int VS, typename T>
__device__ __forceinline__ void trace_point(const T* s, const T* Lm, const T* Lp,
                                            int edge, int fp, T* out) {
    const int line = (edge >= 2) ? (N1 - 1 - fp) : fp;
    const bool along_eta = (edge == 0 || edge == 2);
    const int base = along_eta ? line : line * RS;
    const int stride = along_eta ? RS : 1;
    const T* W = (edge == 0 || edge == 3) ? Lm : Lp;
    T w[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) w[m] = W[m];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const T* sv = s + v * VS + base;
        T t = T(0);
#pragma unroll
        for (int m = 0; m < N1; ++m) t = fma_any(w[m], sv[m * stride], t);
        out[v] = t;
    }
}

// Programmatic dependent launch (sm_90+): a kernel launched with
// cudaLaunchAttributeProgrammaticStreamSerialization may start while the
// previous kernel in its stream finishes.  pdl_launch_dependents lets the
// next such kernel's CTAs start once every CTA of this grid has run it;
// pdl_wait returns once the previous grid has completed and its memory
// operations are visible, so nothing a kernel reads before it may come from
// a kernel (only operators, geometry and kernel parameters).  Both are no-ops
// for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Launch with programmatic stream serialisation: the kernel (which calls
// pdl_wait before reading anything a kernel writes) may start while the
// previous kernel in the stream drains.
template <typename... KA, typename... AA>
cudaError_t launch_programmatic_smem(void (*kernel)(KA...), unsigned grid, unsigned threads, size_t smem,
                                     cudaStream_t s, AA&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<AA&&>(args)...);
}
template <typename... KA, typename... AA>
cudaError_t launch_programmatic(void (*kernel)(KA...), unsigned grid, unsigned threads, cudaStream_t s,
                                AA&&... args) {
    return launch_programmatic_smem(kernel, grid, threads, 0, s, static_cast<AA&&>(args)...);
}

// Trace of one flux point from row `line` of a [var][row][col] tile (weights W
// over the columns), with the row loads of load_row; the sum runs in the
// order of trace_point, so the two agree bit for bit on the same values.
template <int N1, int RS, int VS, typename T>
__device__ __forceinline__ void trace_row(const T* s, const T* W, int line, T* out) {
    T w[N1];
#pragma unroll
    for (int m = 0; m < N1; ++m) w[m] = W[m];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        T r[N1];
        load_row<N1>(s + v * VS + line * RS, r);
        T t = T(0);
#pragma unroll
        for (int m = 0; m < N1; ++m) t = fma_any(w[m], r[m], t);
        out[v] = t;
    }
}

// Block-wide deterministic sum; result valid in thread 0.
__device__ __forceinline__ double block_sum(double x, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) red[w] = x;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        for (int i = 0; i < nw; ++i) s += red[i];
    }
    return s;
}

}  // namespace dev
}  // namespace zj
