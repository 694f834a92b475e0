// tri_fp32.cu -- mixed-precision instantiation of the triangle kernels
// (tri_kernels.cuh).
#include "tri_kernels.cuh"

namespace zj {

cudaError_t launch_tri(int what, int P, int riemann, bool viscous, const StageArgs32& a,
                       const int32_t* elist, long long n, cudaStream_t s) {
    return tri_dispatch(what, P, riemann, viscous, a, elist, n, s);
}

}  // namespace zj
