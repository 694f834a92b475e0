// zj_kernels.h -- launch interface between the C-ABI and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>

#include "zj_dual.cuh"
#include "zj_internal.h"

namespace zj {

// Arguments of one fused residual / RK-stage launch.  Device pointers.  T is
// the arithmetic type of the kernels (double: FP64 path; float: the
// mixed-precision form); the conserved state, the residual output, dt and the
// norm partials are FP64 in both.
template <typename T> struct Vec4Of;
template <> struct Vec4Of<double> { using type = double4; };
template <> struct Vec4Of<float> { using type = float4; };
template <> struct Vec4Of<Dual> { using type = Dual4; };

template <typename T>
struct StageArgsT {
    const double* U;        // stage input state, AoS [E][n_sp][4]
    const double* U0;       // RK base state (stages 2, 3)
    double* Uout;           // stage output state
    const T* Tin;           // traces of U, [E][4 edges][n1][4], then the physics-mode
                            // boundary ghost rows [n_bnd][n1][4] (stored mirrored)
    T* Tout;                // traces of Uout
    double* R;              // residual output (stage 0 only)
    const T* Jinv;          // [E][n_sp][4] = (xi_x, xi_y, eta_x, eta_y)
    const T* J;             // [E][n_sp]
    const EdgeRec* edges;   // [E][4]
    const typename Vec4Of<T>::type* enrm;  // [E][4] = (face nx, face ny, edge length, 0), or
                                           // [E][4][n1] per flux point (nrm_pp) on curved meshes
                                           // with 2 |dx/dt| in the length slot
    const T* bc;            // [slots][8]
    const T* ops;           // packed 1D operators, see OpsLayout
    const double* dt;       // device scalar: step size
    double* partials;       // [grid] per-CTA sum of R^2 (stage 3 and stage 0)
    long long n_elem;
    double gamma;
    int stage;              // 0: residual only; 1..3: SSP-RK3 stage
    // Navier-Stokes
    const T* TQ;            // gradient traces of U, [E][4 edges][n1][8] = (dU/dx, dU/dy)
    T* TQout;               // gradient traces written by the gradient launch
    double Re, Pr;
    double iRe, kfac;       // 1/Re and gamma/((gamma-1) Pr) of the viscosity law
    int* tc_err;            // split-BF16 kernel: set to 1 if a bounded wait gave up
    int nrm_pp;             // 1: enrm holds one record per flux point (curved elements)
    // Element list of a mesh with several element kinds: the launch visits
    // elist[0..n_list) (NULL: every element 0..n_elem)
    const int32_t* elist;
    long long n_list;
    // Jacobian-vector product (T = Dual): tangent of the stage state and of
    // Re in, tangent of the residual out (stage 0)
    const double* dU;
    double* dR;
    double dRe;
};
using StageArgs = StageArgsT<double>;
using StageArgs32 = StageArgsT<float>;
using StageArgsDual = StageArgsT<Dual>;

// Packed operator block: D1[n1*n1], Lm[n1], Lp[n1], gL[n1], gR[n1].
inline int ops_size(int n1) { return n1 * n1 + 4 * n1; }
void pack_ops(const Operators1D& o, std::vector<double>& out);

// Compat-mode FP64 launches (reference residual semantics).
cudaError_t launch_compat_stage(int P, const StageArgs& a, cudaStream_t s, int* grid_out);
// Physics-mode launches (conservative FR, VCJH, selected Riemann solver),
// FP64 and mixed precision.
cudaError_t launch_phys_stage(int P, int riemann, const StageArgs& a, cudaStream_t s);
cudaError_t launch_phys_stage(int P, int riemann, const StageArgs32& a, cudaStream_t s);
// Physics-mode traces of a.U into a.Tout, boundary ghost rows included.
cudaError_t launch_phys_traces(int P, const StageArgs& a, cudaStream_t s);
cudaError_t launch_phys_traces(int P, const StageArgs32& a, cudaStream_t s);
// Navier-Stokes: gradient traces of a stage state, then the stage itself.
cudaError_t launch_ns_grad(int P, const StageArgs& a, cudaStream_t s);
cudaError_t launch_ns_grad(int P, const StageArgs32& a, cudaStream_t s);
cudaError_t launch_ns_stage(int P, int riemann, const StageArgs& a, cudaStream_t s);
cudaError_t launch_ns_stage(int P, int riemann, const StageArgs32& a, cudaStream_t s);
// Jacobian-vector products: the stage-0 kernels on dual numbers.  Grid:
// dual_grid(P, E) CTAs (partials sized for it).
cudaError_t launch_phys_traces(int P, const StageArgsDual& a, cudaStream_t s);
cudaError_t launch_phys_stage(int P, int riemann, const StageArgsDual& a, cudaStream_t s);
cudaError_t launch_ns_grad(int P, const StageArgsDual& a, cudaStream_t s);
cudaError_t launch_ns_stage(int P, int riemann, const StageArgsDual& a, cudaStream_t s);
int dual_grid(int P, long long n_elem);
// Triangles (tri_kernels.cuh): what = 0 traces (+ ghost rows) of a.U into
// a.Tout, 1 gradient traces (Navier-Stokes), 2 residual / stage; over the
// triangle list elist[0..n).  a.ops holds the packed triangle operators.
cudaError_t launch_tri(int what, int P, int riemann, bool viscous, const StageArgs& a, const int32_t* elist,
                       long long n, cudaStream_t s);
cudaError_t launch_tri(int what, int P, int riemann, bool viscous, const StageArgs32& a,
                       const int32_t* elist, long long n, cudaStream_t s);
int tri_grid(int P, long long n);
// Split-BF16 Navier-Stokes stage (ns_tc.cu), precision form at P4/P5 on
// quad meshes: the operator image (BF16 hi/lo terms, build_tc_image) is
// staged by TMA through the tensor map make_tc_tensor_map writes (128 bytes,
// a CUtensorMap); grid tc_grid(P, E) CTAs (partials sized for it).
bool tc_order_supported(int P);
int tc_grid(int P, long long n);
bool build_tc_image(int P, const Operators1D& o, std::vector<uint16_t>& img);
cudaError_t make_tc_tensor_map(int P, const void* dev_img, void* map_out);
cudaError_t launch_ns_stage_tc(int P, int riemann, const StageArgs32& a, const void* map, cudaStream_t s);
// Quad CTA count of a launch over n elements.
int quad_grid(int P, long long n);
// Elementwise helpers of the differentiation entry points (jvp.cu).
cudaError_t launch_to_dual(const double* x, Dual* y, long long n, cudaStream_t s);
cudaError_t launch_lincomb(double* out, double a, const double* x, double b, const double* y,
                           double c, const double* z, long long n, cudaStream_t s);
int dot_grid();
// out[0] = x . y, deterministic (fixed grid; partials has dot_grid() entries).
cudaError_t launch_dot(const double* x, const double* y, long long n, double* partials,
                       double* out, cudaStream_t s);
cudaError_t launch_traces(int P, const double* U, double* T, const double* ops,
                          long long n_elem, cudaStream_t s);
int stage_grid(int P, long long n_elem);

// Vector-Jacobian product of the physics-mode residual (adjoint.cu).  Device
// pointers; T / TQ are the forward traces (with ghost rows) and gradient
// traces of U; Db, Tb, DUb are [E][4][n1][4] scratch.
struct AdjArgs {
    const double* U;
    const double* L;        // residual adjoint (lambda)
    double* W;              // (dR/dU)^T L
    const double* T;
    const double* TQ;
    double* Db;             // dFbar per flux point
    double* Tb;             // trace adjoint before the neighbour gather (NS)
    double* DUb;            // adjoint of the gradient's face jumps (NS)
    const double* Jinv;
    const double* J;
    const EdgeRec* edges;
    const double4* enrm;
    const double* bc;
    const double* ops;
    long long n_elem;
    double gamma, Re, Pr;
    double* re_part;        // optional, Navier-Stokes: per-CTA L . dR/dRe, adj_ns_grid entries
    // optional fused output: out = c0 X0 + c1 X1 + c2 X2 + cw (dR/dU)^T L
    // (an SSP-RK3 stage's adjoint update; X* may be NULL when c* is 0, out may
    // alias any X*); out == NULL writes (dR/dU)^T L into W
    double* out;
    const double* X0;
    const double* X1;
    const double* X2;
    double c0, c1, c2, cw;
};
cudaError_t launch_rhs_vjp(int P, int riemann, bool viscous, const AdjArgs& a, cudaStream_t s);
int adj_ns_grid(int P, long long n_elem);

// Deterministic reduction of per-CTA partial sums into out[0].
cudaError_t launch_reduce_sum(const double* partials, int n, double* out, cudaStream_t s);
// out[0] = min over states of CFL*h/(ws*(2P+1)); h per element.
// Triangles (etype[e] == ZJ_ELEM_TRI) count their first nt slots only.
cudaError_t launch_compute_dt(const double* U, const double* h, long long n_elem, int n_sp,
                              double gamma, double cfl, int P, double* scratch, int scratch_n,
                              double* out, cudaStream_t s, const int8_t* etype = nullptr, int nt = 0);
// flag[0] = 1 if any value of x[0..n) is NaN/Inf.
cudaError_t launch_check_finite(const double* x, long long n, int* flag, cudaStream_t s);

}  // namespace zj
