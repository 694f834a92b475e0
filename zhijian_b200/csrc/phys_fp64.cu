// phys_fp64.cu -- FP64 instantiation of the physics-mode (inviscid) stage and
// trace kernels of phys_kernels.cuh: the path that matches the reference's
// residual to 1e-12.
#include "phys_kernels.cuh"

namespace zj {

cudaError_t launch_phys_traces(int P, const StageArgs& a, cudaStream_t s) {
    return phys_traces_dispatch(P, a, s);
}

cudaError_t launch_phys_stage(int P, int riemann, const StageArgs& a, cudaStream_t s) {
    return phys_stage_dispatch(P, riemann, a, s);
}

}  // namespace zj
