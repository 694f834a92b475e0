// ns_fp32.cu -- mixed-precision instantiation of the Navier-Stokes gradient
// and stage kernels of ns_kernels.cuh: FP32 gradients, fluxes, faces,
// operator products, traces and metrics; FP64 state, SSP-RK3 accumulation and
// residual-norm partials.
#include "ns_kernels.cuh"

namespace zj {

cudaError_t launch_ns_grad(int P, const StageArgs32& a, cudaStream_t s) {
    return ns_grad_dispatch(P, a, s);
}

cudaError_t launch_ns_stage(int P, int riemann, const StageArgs32& a, cudaStream_t s) {
    return ns_stage_dispatch(P, riemann, a, s);
}

}  // namespace zj
