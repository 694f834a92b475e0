// jvp.cu -- Jacobian-vector products of the physics-mode residual: the
// stage-0 kernels of phys_kernels.cuh / ns_kernels.cuh instantiated on dual
// numbers (zj_dual.cuh).  One launch computes R(U) and dR/dU . V (+ dR/dRe
// dRe) exactly, with the FP64 operation order of the residual path.
#include "ns_kernels.cuh"

namespace zj {

int dual_grid(int P, long long n_elem) {
    int eb = 1;
    switch (P) {
        case 1: eb = Shape<1, EbDiv<Dual>::value>::EB; break;
        case 2: eb = Shape<2, EbDiv<Dual>::value>::EB; break;
        case 3: eb = Shape<3, EbDiv<Dual>::value>::EB; break;
        case 4: eb = Shape<4, EbDiv<Dual>::value>::EB; break;
        case 5: eb = Shape<5, EbDiv<Dual>::value>::EB; break;
        default: return 0;
    }
    return (int)((n_elem + eb - 1) / eb);
}

cudaError_t launch_phys_traces(int P, const StageArgsDual& a, cudaStream_t s) {
    return phys_traces_dispatch(P, a, s);
}

cudaError_t launch_phys_stage(int P, int riemann, const StageArgsDual& a, cudaStream_t s) {
    return phys_stage_dispatch(P, riemann, a, s);
}

cudaError_t launch_ns_grad(int P, const StageArgsDual& a, cudaStream_t s) {
    return ns_grad_dispatch(P, a, s);
}

cudaError_t launch_ns_stage(int P, int riemann, const StageArgsDual& a, cudaStream_t s) {
    return ns_stage_dispatch(P, riemann, a, s);
}

}  // namespace zj

// ------------------------------------------------ helpers of the adjoint --
namespace zj {
namespace {

__global__ void k_to_dual(const double* __restrict__ x, Dual* __restrict__ y, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        y[i] = Dual(x[i], 0.0);
}

// out = a x + b y + c z (y, z may be NULL when their weight is 0)
__global__ void k_lincomb(double* __restrict__ out, double a, const double* x, double b,
                          const double* y, double c, const double* z, long long n) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x) {
        double r = a * x[i];
        if (y) r += b * y[i];
        if (z) r += c * z[i];
        out[i] = r;
    }
}

// Per-CTA partial dot products with a fixed grid (deterministic order).
__global__ void k_dot_partial(const double* __restrict__ x, const double* __restrict__ y,
                              long long n, double* partials) {
    __shared__ double red[32];
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        s = fma(x[i], y[i], s);
    const double b = dev::block_sum(s, red);
    if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

constexpr int kFillGrid = 148 * 8;

}  // namespace

cudaError_t launch_to_dual(const double* x, Dual* y, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_to_dual<<<kFillGrid, 256, 0, s>>>(x, y, n);
    return cudaGetLastError();
}

cudaError_t launch_lincomb(double* out, double a, const double* x, double b, const double* y,
                           double c, const double* z, long long n, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    k_lincomb<<<kFillGrid, 256, 0, s>>>(out, a, x, b, y, c, z, n);
    return cudaGetLastError();
}

int dot_grid() { return kFillGrid; }

cudaError_t launch_dot(const double* x, const double* y, long long n, double* partials,
                       double* out, cudaStream_t s) {
    k_dot_partial<<<kFillGrid, 256, 0, s>>>(x, y, n, partials);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_reduce_sum(partials, kFillGrid, out, s);
}

}  // namespace zj
