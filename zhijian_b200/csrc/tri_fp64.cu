// tri_fp64.cu -- FP64 instantiation of the triangle kernels (tri_kernels.cuh).
#include "tri_kernels.cuh"

namespace zj {

cudaError_t launch_tri(int what, int P, int riemann, bool viscous, const StageArgs& a, const int32_t* elist,
                       long long n, cudaStream_t s) {
    return tri_dispatch(what, P, riemann, viscous, a, elist, n, s);
}

int tri_grid(int P, long long n) {
    switch (P) {
        case 1: return tri_grid_t<1>(n);
        case 2: return tri_grid_t<2>(n);
        case 3: return tri_grid_t<3>(n);
        case 4: return tri_grid_t<4>(n);
        case 5: return tri_grid_t<5>(n);
        default: return 0;
    }
}

int quad_grid(int P, long long n) {
    int eb = 1;
    switch (P) {
        case 1: eb = Shape<1>::EB; break;
        case 2: eb = Shape<2>::EB; break;
        case 3: eb = Shape<3>::EB; break;
        case 4: eb = Shape<4>::EB; break;
        case 5: eb = Shape<5>::EB; break;
        default: return 0;
    }
    return (int)((n + eb - 1) / eb);
}

}  // namespace zj
