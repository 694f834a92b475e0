// phys_fp32.cu -- mixed-precision instantiation of the physics-mode
// (inviscid) stage and trace kernels of phys_kernels.cuh: FP32 fluxes, faces,
// operator products, traces and metrics; FP64 state, SSP-RK3 accumulation and
// residual-norm partials.
#include "phys_kernels.cuh"

namespace zj {

cudaError_t launch_phys_traces(int P, const StageArgs32& a, cudaStream_t s) {
    return phys_traces_dispatch(P, a, s);
}

cudaError_t launch_phys_stage(int P, int riemann, const StageArgs32& a, cudaStream_t s) {
    return phys_stage_dispatch(P, riemann, a, s);
}

}  // namespace zj
