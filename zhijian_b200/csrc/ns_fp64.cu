// ns_fp64.cu -- FP64 instantiation of the Navier-Stokes gradient and stage
// kernels of ns_kernels.cuh: the path that matches the reference's residual
// to 1e-12.
#include "ns_kernels.cuh"

namespace zj {

cudaError_t launch_ns_grad(int P, const StageArgs& a, cudaStream_t s) {
    return ns_grad_dispatch(P, a, s);
}

cudaError_t launch_ns_stage(int P, int riemann, const StageArgs& a, cudaStream_t s) {
    return ns_stage_dispatch(P, riemann, a, s);
}

}  // namespace zj
