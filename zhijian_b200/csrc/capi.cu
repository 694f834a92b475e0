// capi.cu -- the extern "C" boundary declared in include/zj_fr.h.
//
// A zj_solver owns every device buffer, allocated once in zj_solver_create:
//   state   3 x [E][n_sp][4] f64   rotating stage buffers (no stage writes a
//                                  buffer it reads, so no aliasing)
//   traces  3 x [E][4][n1][4]      ping-pong pair for the stepper + one for
//                                  zj_rhs (+ boundary ghost rows)
//   metrics [E][n_sp][4] Jinv, [E][n_sp] J, per-element edge records, bc
//   scratch state + residual for the host-buffer entry points, reductions
// Traces, gradient traces, metrics, normals, operators and bc data exist in
// the arithmetic type of the handle: FP64, or FP32 for the mixed-precision
// form (whose state and reductions stay FP64).
// An SSP-RK3 step is three fused stage launches; the first step after a state
// upload is preceded by one trace launch.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <mutex>
#include <vector>

#include "zj_internal.h"
#include "zj_kernels.h"

using namespace zj;

struct zj_gmsh_mesh {
    GmshMesh g;
    zj_mesh_desc desc{};
};

struct zj_solver {
    zj_params prm{};
    HostMesh mesh;
    Operators1D ops;
    int P = 0, n1 = 0, nsp = 0;
    long long E = 0;
    size_t state_n = 0, trace_n = 0;
    double* dU[3] = {nullptr, nullptr, nullptr};
    double* dT[3] = {nullptr, nullptr, nullptr};
    double* dTQ = nullptr;      // gradient traces (Navier-Stokes)
    double* dUs = nullptr;      // scratch state (host-buffer residual)
    double* dRs = nullptr;      // scratch residual
    double* dJinv = nullptr;
    double* dJ = nullptr;
    double* dOps = nullptr;
    double* dBC = nullptr;
    double* dH = nullptr;       // sqrt(element area) for the CFL step
    double* dScal = nullptr;    // [0] dt, [1] step norm^2, [2] dt out, [3] rhs norm^2
    double* dPart = nullptr;    // per-CTA partial sums, stepper
    double* dPartR = nullptr;   // per-CTA partial sums, zj_rhs
    double* dScratch = nullptr; // CFL reduction scratch
    int scratch_n = 0;
    int* dFlag = nullptr;
    EdgeRec* dEdges = nullptr;
    double4* dNrm = nullptr;
    // mixed-precision form: FP32 traces, gradient traces and geometry
    bool mixed = false;
    int nrm_pp = 0;             // curved elements in physics mode: normals per flux point
    float* fT[3] = {nullptr, nullptr, nullptr};
    float* fTQ = nullptr;
    float* fJinv = nullptr;
    float* fJ = nullptr;
    float* fOps = nullptr;
    float* fBC = nullptr;
    float4* fNrm = nullptr;
    // split-BF16 Navier-Stokes stage (P4/P5, quads): BF16 operator image,
    // its TMA tensor map and the kernel's wait-timeout flag
    bool tc = false;
    uint16_t* dTcImg = nullptr;
    int* dTcErr = nullptr;
    alignas(64) CUtensorMap tc_map;
    // meshes with triangles: element lists per kind, triangle operators
    int64_t n_tri = 0, n_quad = 0;
    int nt = 0;                     // triangle solution points
    int grid_q = 0, grid_t = 0;
    int32_t* dElistQ = nullptr;
    int32_t* dElistT = nullptr;
    double* dTriOps = nullptr;
    float* fTriOps = nullptr;
    int8_t* dEtype = nullptr;
    std::vector<int8_t> etype;
    // differentiation: dual-number geometry and traces (Jacobian-vector
    // products) and adjoint scratch, allocated on first use
    size_t n_jinv = 0, n_j = 0, n_ops = 0, n_bcd = 0, n_nrm = 0;
    bool diff_ready = false;
    Dual* xJinv = nullptr;
    Dual* xJ = nullptr;
    Dual* xOps = nullptr;
    Dual* xBC = nullptr;
    Dual4* xNrm = nullptr;
    Dual* xT = nullptr;
    Dual* xTQ = nullptr;
    double* xPart = nullptr;
    double* aDb = nullptr;      // dFbar per flux point
    double* aTb = nullptr;      // trace adjoint (NS)
    double* aDUb = nullptr;     // gradient-jump adjoint (NS)
    double* aW = nullptr;       // VJP output scratch
    double* aS1 = nullptr;      // stage states U(1), U(2)
    double* aS2 = nullptr;
    double* aB0 = nullptr;      // stage adjoints
    double* aB1 = nullptr;
    double* aB2 = nullptr;
    double* aR = nullptr;       // residual scratch of a JVP
    double* aJV = nullptr;      // dR/dRe
    double* aZero = nullptr;    // zero tangent
    double* aDot = nullptr;     // dot-product partials
    double* aScal = nullptr;    // [0] dJ/dRe accumulator, [1] dot result
    double* aRePart = nullptr;  // per-CTA L . dR/dRe of the NS VJP
    int grid = 0;
    int cur = 0, tpar = 0;
    bool traces_valid = false;
    // Step graphs: the stage buffers rotate with period 3 and the trace
    // buffers with period 2, so six steps return to the starting (cur, tpar);
    // one captured 6-step block per starting phase, replayed by zj_step.
    cudaGraphExec_t gexec[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool graphs_on = true;      // zj_set_step_graphs
    bool graphs_failed = false; // a capture failed: plain launches from then on
    bool stepped = false;       // a plain step ran (the kernels' one-time attributes are set)
    bool has_norm = false;
    cudaStream_t own = nullptr, stream = nullptr;
    int device = 0;             // the device current at zj_solver_create
    // one part of a partitioned mesh (zj_solver_create_part): the part's
    // view, its halo rows (sent: its side of each interface; received: the
    // interfaces' ghost rows) and exchange buffers of n_iface rows of n1*8
    // values in the handle's arithmetic type
    bool is_part = false;
    PartSlice part;
    int64_t n_ghost = 0;        // ghost rows after the element rows: boundary slots + interfaces
    int32_t* dSendRows = nullptr;
    int32_t* dRecvRows = nullptr;
    void* dSendBuf = nullptr;
    void* dRecvBuf = nullptr;
    cudaEvent_t ev_pack = nullptr, ev_done = nullptr;
    cudaEvent_t ev_join = nullptr;   // step graphs of a partition: fork/join of the parts' streams
    double time = 0.0;
    int iter = 0;
    double last_dt = -1.0;
    std::string err;
};

namespace {

thread_local std::string g_create_err;

zj_status fail(zj_solver* s, zj_status code, const std::string& msg) {
    if (s) s->err = msg; else g_create_err = msg;
    return code;
}

zj_status cuda_fail(zj_solver* s, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
    return fail(s, ZJ_ERR_CUDA, m);
}

#define ZJ_CK(s, call, what)                                   \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail((s), e_, what); \
    } while (0)

template <class T>
cudaError_t dalloc(T** p, size_t n) {
    return cudaMalloc(reinterpret_cast<void**>(p), (n ? n : 1) * sizeof(T));
}

void free_all(zj_solver* s) {
    for (auto& p : s->dU) { if (p) cudaFree(p); p = nullptr; }
    for (auto& p : s->dT) { if (p) cudaFree(p); p = nullptr; }
    if (s->dTQ) cudaFree(s->dTQ);
    s->dTQ = nullptr;
    double** ds[] = {&s->dUs, &s->dRs, &s->dJinv, &s->dJ, &s->dOps, &s->dBC, &s->dH,
                     &s->dScal, &s->dPart, &s->dPartR, &s->dScratch};
    for (auto pp : ds) { if (*pp) cudaFree(*pp); *pp = nullptr; }
    for (auto& p : s->fT) { if (p) cudaFree(p); p = nullptr; }
    float** fs[] = {&s->fTQ, &s->fJinv, &s->fJ, &s->fOps, &s->fBC};
    for (auto pp : fs) { if (*pp) cudaFree(*pp); *pp = nullptr; }
    if (s->fNrm) cudaFree(s->fNrm);
    s->fNrm = nullptr;
    void* tcs[] = {s->dTcImg, s->dTcErr};
    for (void* p : tcs) if (p) cudaFree(p);
    s->dTcImg = nullptr; s->dTcErr = nullptr;
    void* ts[] = {s->dElistQ, s->dElistT, s->dTriOps, s->fTriOps, s->dEtype};
    for (void* p : ts) if (p) cudaFree(p);
    s->dElistQ = s->dElistT = nullptr; s->dTriOps = nullptr; s->fTriOps = nullptr; s->dEtype = nullptr;
    void* xs[] = {s->xJinv, s->xJ, s->xOps, s->xBC, s->xNrm, s->xT, s->xTQ, s->xPart, s->aDb, s->aTb,
                  s->aDUb, s->aW, s->aS1, s->aS2, s->aB0, s->aB1, s->aB2, s->aR, s->aJV, s->aZero,
                  s->aDot, s->aScal, s->aRePart};
    for (void* p : xs) if (p) cudaFree(p);
    s->diff_ready = false;
    if (s->dFlag) cudaFree(s->dFlag);
    if (s->dEdges) cudaFree(s->dEdges);
    if (s->dNrm) cudaFree(s->dNrm);
    s->dFlag = nullptr; s->dEdges = nullptr; s->dNrm = nullptr;
    for (auto& g : s->gexec) { if (g) cudaGraphExecDestroy(g); g = nullptr; }
    void* hs[] = {s->dSendRows, s->dRecvRows, s->dSendBuf, s->dRecvBuf};
    for (void* p : hs) if (p) cudaFree(p);
    s->dSendRows = s->dRecvRows = nullptr; s->dSendBuf = s->dRecvBuf = nullptr;
    if (s->ev_pack) cudaEventDestroy(s->ev_pack);
    if (s->ev_done) cudaEventDestroy(s->ev_done);
    if (s->ev_join) cudaEventDestroy(s->ev_join);
    s->ev_pack = s->ev_done = s->ev_join = nullptr;
    if (s->own) cudaStreamDestroy(s->own);
    s->own = nullptr;
}

zj_status validate_params(const zj_params* p, std::string& msg) {
    if (p->poly_order < 1 || p->poly_order > kMaxP) { msg = "poly_order must be 1..5"; return ZJ_ERR_ARG; }
    if (!(p->gamma > 1.0)) { msg = "gamma must be > 1"; return ZJ_ERR_ARG; }
    if (!(p->rho_inf > 0.0) || !(p->p_inf > 0.0)) { msg = "rho_inf and p_inf must be > 0"; return ZJ_ERR_ARG; }
    if (p->flux_type < 0 || p->flux_type > 3) { msg = "flux_type must be DG, SD, HU or GA"; return ZJ_ERR_ARG; }
    if (p->riemann < 0 || p->riemann > 2) { msg = "riemann must be Rusanov, Roe or HLLC"; return ZJ_ERR_ARG; }
    if (p->n_bc < 0 || p->n_bc > ZJ_MAX_BC) { msg = "n_bc out of range"; return ZJ_ERR_ARG; }
    if (!p->compat && p->viscous && !(p->Re > 0.0 && p->Pr > 0.0)) { msg = "Re and Pr must be > 0"; return ZJ_ERR_ARG; }
    if (p->precision != ZJ_FP64 && p->precision != ZJ_MIXED && p->precision != ZJ_SPLIT_BF16) {
        msg = "precision must be fp64, mixed or split_bf16";
        return ZJ_ERR_ARG;
    }
    if (p->precision != ZJ_FP64 && p->compat) {
        msg = "the mixed-precision form needs physics mode (compat off): compat mode is the reference's FP64 residual";
        return ZJ_ERR_UNSUPPORTED;
    }
    return ZJ_OK;
}

bool is_ns(const zj_solver* s) { return !s->prm.compat && s->prm.viscous; }

// Buffers of the handle's arithmetic type.
template <typename T> T* tbuf(const zj_solver* s, int i);
template <> double* tbuf<double>(const zj_solver* s, int i) { return s->dT[i]; }
template <> float* tbuf<float>(const zj_solver* s, int i) { return s->fT[i]; }

template <typename T> const T* tri_ops(const zj_solver* s);
template <> const double* tri_ops<double>(const zj_solver* s) { return s->dTriOps; }
template <> const float* tri_ops<float>(const zj_solver* s) { return s->fTriOps; }

template <typename T> StageArgsT<T> base_args(const zj_solver* s);
template <> StageArgsT<double> base_args<double>(const zj_solver* s) {
    StageArgsT<double> a{};
    a.Jinv = s->dJinv; a.J = s->dJ; a.enrm = s->dNrm; a.bc = s->dBC; a.ops = s->dOps;
    a.TQ = s->dTQ; a.TQout = s->dTQ; a.nrm_pp = s->nrm_pp;
    return a;
}
template <> StageArgsT<float> base_args<float>(const zj_solver* s) {
    StageArgsT<float> a{};
    a.Jinv = s->fJinv; a.J = s->fJ; a.enrm = s->fNrm; a.bc = s->fBC; a.ops = s->fOps;
    a.TQ = s->fTQ; a.TQout = s->fTQ; a.nrm_pp = s->nrm_pp;
    return a;
}

// 1/Re and gamma/((gamma-1) Pr), the viscosity law's constants, once per
// launch instead of two divisions per viscous flux.
template <typename T>
void set_viscous_constants(StageArgsT<T>& a) {
    a.iRe = 1.0 / a.Re;
    a.kfac = a.gamma / ((a.gamma - 1.0) * a.Pr);
}

template <typename T>
StageArgsT<T> stage_args(const zj_solver* s) {
    StageArgsT<T> a = base_args<T>(s);
    a.edges = s->dEdges;
    a.dt = s->dScal;
    a.n_elem = s->E;
    a.gamma = s->prm.gamma;
    a.Re = s->prm.Re;
    a.Pr = s->prm.Pr;
    set_viscous_constants(a);
    return a;
}

// One residual or RK-stage evaluation in the handle's mode: one launch, or
// the gradient launch then the stage launch for Navier-Stokes.
template <typename T>
cudaError_t launch_stage(const zj_solver* s, const StageArgsT<T>& a) {
    if constexpr (sizeof(T) == 8) {
        if (s->prm.compat) return launch_compat_stage(s->P, a, s->stream, nullptr);
    }
    if (s->n_tri == 0) {
        if (!is_ns(s)) return launch_phys_stage(s->P, s->prm.riemann, a, s->stream);
        cudaError_t e = launch_ns_grad(s->P, a, s->stream);
        if (e != cudaSuccess) return e;
        if constexpr (sizeof(T) == 4) {
            if (s->tc) {
                StageArgsT<T> t = a;
                t.tc_err = s->dTcErr;
                return launch_ns_stage_tc(s->P, s->prm.riemann, t, &s->tc_map, s->stream);
            }
        }
        return launch_ns_stage(s->P, s->prm.riemann, a, s->stream);
    }
    // quads and triangles: every gradient trace before any stage (a face's
    // neighbour may be of the other kind); the triangles' CTAs write their
    // partial sums after the quads'
    StageArgsT<T> q = a, t = a;
    q.elist = s->dElistQ; q.n_list = s->n_quad;
    t.ops = tri_ops<T>(s);
    t.partials = a.partials ? a.partials + s->grid_q : nullptr;
    cudaError_t e = cudaSuccess;
    if (is_ns(s)) {
        if (s->n_quad > 0) e = launch_ns_grad(s->P, q, s->stream);
        if (e == cudaSuccess) e = launch_tri(1, s->P, s->prm.riemann, true, t, s->dElistT, s->n_tri, s->stream);
        if (e == cudaSuccess && s->n_quad > 0) e = launch_ns_stage(s->P, s->prm.riemann, q, s->stream);
    } else if (s->n_quad > 0) {
        e = launch_phys_stage(s->P, s->prm.riemann, q, s->stream);
    }
    if (e == cudaSuccess) e = launch_tri(2, s->P, s->prm.riemann, is_ns(s), t, s->dElistT, s->n_tri, s->stream);
    return e;
}

// Traces of U into Tb in the handle's mode (physics mode adds the ghost rows).
template <typename T>
cudaError_t launch_trace_any(const zj_solver* s, const double* U, T* Tb) {
    if constexpr (sizeof(T) == 8) {
        if (s->prm.compat) return launch_traces(s->P, U, Tb, s->dOps, s->E, s->stream);
    }
    StageArgsT<T> a = stage_args<T>(s);
    a.U = U;
    a.Tout = Tb;
    if (s->n_tri == 0) return launch_phys_traces(s->P, a, s->stream);
    cudaError_t e = cudaSuccess;
    if (s->n_quad > 0) {
        StageArgsT<T> q = a;
        q.elist = s->dElistQ; q.n_list = s->n_quad;
        e = launch_phys_traces(s->P, q, s->stream);
    }
    if (e != cudaSuccess) return e;
    a.ops = tri_ops<T>(s);
    return launch_tri(0, s->P, s->prm.riemann, is_ns(s), a, s->dElistT, s->n_tri, s->stream);
}

template <typename T>
zj_status enqueue_step(zj_solver* s) {
    const int c = s->cur, a1 = (c + 1) % 3, b1 = (c + 2) % 3, p = s->tpar;
    StageArgsT<T> a = stage_args<T>(s);
    a.partials = s->dPart;
    // stage 1: U(1) = U0 + dt R(U0)
    a.U = s->dU[c]; a.U0 = s->dU[c]; a.Uout = s->dU[a1]; a.Tin = tbuf<T>(s, p); a.Tout = tbuf<T>(s, 1 - p);
    a.stage = 1;
    ZJ_CK(s, launch_stage(s, a), "stage 1 launch");
    // stage 2: U(2) = 3/4 U0 + 1/4 U(1) + 1/4 dt R(U(1))
    a.U = s->dU[a1]; a.Uout = s->dU[b1]; a.Tin = tbuf<T>(s, 1 - p); a.Tout = tbuf<T>(s, p);
    a.stage = 2;
    ZJ_CK(s, launch_stage(s, a), "stage 2 launch");
    // stage 3: U = 1/3 U0 + 2/3 U(2) + 2/3 dt R(U(2))
    a.U = s->dU[b1]; a.Uout = s->dU[a1]; a.Tin = tbuf<T>(s, p); a.Tout = tbuf<T>(s, 1 - p);
    a.stage = 3;
    ZJ_CK(s, launch_stage(s, a), "stage 3 launch");
    s->cur = a1;
    s->tpar = 1 - p;
    return ZJ_OK;
}

constexpr int kGraphSteps = 6;

// dt[0] = v: the step size reaches the device as a kernel argument, so a
// zj_step inside a graph the caller captures records the value itself (a copy
// from a host variable would record a pointer to it).
__global__ void k_set_dt(double* dt, double v) { *dt = v; }

// The 6-step block starting at the handle's (cur, tpar), captured on first
// use; nullptr where graphs cannot be used: the legacy default stream (not
// capturable), a stream the caller is capturing (the plain launches join the
// caller's graph), or a failed capture (plain launches from then on).
template <typename T>
cudaGraphExec_t step_graph(zj_solver* s) {
    if (!s->graphs_on || s->graphs_failed || !s->stepped || s->stream == nullptr) return nullptr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    const int idx = s->cur * 2 + s->tpar;
    if (s->gexec[idx]) return s->gexec[idx];
    const int cur0 = s->cur, tpar0 = s->tpar;
    const std::string err0 = s->err;
    if (cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        (void)cudaGetLastError();
        s->graphs_failed = true;
        return nullptr;
    }
    zj_status st = ZJ_OK;
    for (int k = 0; k < kGraphSteps && st == ZJ_OK; ++k) st = enqueue_step<T>(s);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    s->cur = cur0;       // six steps come back to the starting phase; nothing ran yet
    s->tpar = tpar0;
    cudaGraphExec_t exec = nullptr;
    if (st == ZJ_OK && e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (st != ZJ_OK || e != cudaSuccess || !exec) {
        (void)cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        s->err = err0;
        s->graphs_failed = true;
        return nullptr;
    }
    s->gexec[idx] = exec;
    return exec;
}

// After the handle's first plain step: capture the 6-step graphs of all six
// buffer phases and upload them, so no later zj_step captures or uploads (a
// caller timing a later call sees only graph launches).
template <typename T>
void capture_all_phases(zj_solver* s) {
    if (!s->graphs_on || s->graphs_failed || !s->stepped || s->stream == nullptr) return;
    const int cur0 = s->cur, tpar0 = s->tpar;
    for (int c = 0; c < 3 && !s->graphs_failed; ++c)
        for (int p = 0; p < 2 && !s->graphs_failed; ++p) {
            s->cur = c;
            s->tpar = p;
            cudaGraphExec_t g = step_graph<T>(s);
            if (g && cudaGraphUpload(g, s->stream) != cudaSuccess) {
                (void)cudaGetLastError();
                s->graphs_failed = true;
            }
        }
    s->cur = cur0;
    s->tpar = tpar0;
}

template <typename T>
zj_status step_impl(zj_solver* s, int nsteps, double dt) {
    if (!s->traces_valid) {
        ZJ_CK(s, launch_trace_any(s, s->dU[s->cur], tbuf<T>(s, s->tpar)), "trace launch");
        s->traces_valid = true;
    }
    const bool first = !s->stepped;
    // blocks of six steps replay a captured graph (one launch instead of six
    // to twelve); the rest, and the handle's first step, launch directly
    for (int k = 0; k < nsteps;) {
        cudaGraphExec_t g = (nsteps - k >= kGraphSteps) ? step_graph<T>(s) : nullptr;
        if (g) {
            ZJ_CK(s, cudaGraphLaunch(g, s->stream), "step graph launch");
            for (int i = 0; i < kGraphSteps; ++i) { s->time += dt; s->iter += 1; }
            k += kGraphSteps;
        } else {
            zj_status st = enqueue_step<T>(s);
            if (st != ZJ_OK) return st;
            s->time += dt;
            s->iter += 1;
            s->stepped = true;
            ++k;
        }
    }
    if (first) capture_all_phases<T>(s);
    return ZJ_OK;
}

// Residual of U_dev into R_dev with the given trace / gradient-trace /
// partial-sum scratch.
template <typename T>
zj_status rhs_impl(zj_solver* s, const double* U_dev, double* R_dev, T* traces, T* grad_traces,
                   double* partials) {
    ZJ_CK(s, launch_trace_any(s, U_dev, traces), "trace launch");
    StageArgsT<T> a = stage_args<T>(s);
    a.U = U_dev; a.U0 = U_dev; a.Uout = nullptr; a.Tin = traces; a.Tout = nullptr;
    a.R = R_dev; a.partials = partials; a.stage = 0;
    if (grad_traces) { a.TQ = grad_traces; a.TQout = grad_traces; }
    ZJ_CK(s, launch_stage(s, a), "residual launch");
    return ZJ_OK;
}

template <typename T>
std::vector<T> narrow(const std::vector<double>& v) {
    return std::vector<T>(v.begin(), v.end());
}

}  // namespace

extern "C" {

int zj_abi_version(void) { return ZJ_ABI_VERSION; }

const char* zj_last_error(const zj_solver* s) {
    return s ? s->err.c_str() : g_create_err.c_str();
}

}  // extern "C"

namespace {

// The one creation path: the whole mesh (part == NULL), or part `rank` of a
// partition (the global per-element arrays are built, then restricted to the
// part's elements, with the cut faces as interface ghost rows).
zj_status create_impl(const zj_mesh_desc* mesh, const zj_params* params, const int32_t* part, int nparts,
                      int rank, zj_solver** out) {
    if (!out) return fail(nullptr, ZJ_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!mesh || !params) return fail(nullptr, ZJ_ERR_ARG, "mesh or params is NULL");
    std::string msg;
    zj_status st = validate_params(params, msg);
    if (st != ZJ_OK) return fail(nullptr, st, msg);

    zj_solver* s = new zj_solver();
    s->prm = *params;
    s->P = params->poly_order;
    s->n1 = s->P + 1;
    s->nsp = s->n1 * s->n1;
    if (!build_mesh(mesh, params, s->mesh, msg)) { delete s; return fail(nullptr, ZJ_ERR_ARG, msg); }
    s->E = s->mesh.n_elem;
    if (part) {
        if (params->compat) {
            delete s;
            return fail(nullptr, ZJ_ERR_UNSUPPORTED, "partitioned meshes run in physics mode (compat off)");
        }
        if (s->mesh.n_tri > 0) {
            delete s;
            return fail(nullptr, ZJ_ERR_UNSUPPORTED, "partitioned meshes are quadrilateral meshes");
        }
        if (!make_part_slice(s->mesh, part, nparts, rank, s->part, msg)) { delete s; return fail(nullptr, ZJ_ERR_ARG, msg); }
        s->is_part = true;
    }
    if (s->E > (1LL << 31) / (4LL * s->nsp)) { delete s; return fail(nullptr, ZJ_ERR_ARG, "mesh too large"); }
    if (params->compat) build_operators_compat(s->P, s->ops);
    else build_operators_vcjh(s->P, params->flux_type, s->ops);
    s->n_tri = s->mesh.n_tri;
    s->n_quad = s->E - s->n_tri;
    TriOperators tri;
    std::vector<double> tri_packed;
    if (s->n_tri > 0) {
        if (params->compat) {
            delete s;
            return fail(nullptr, ZJ_ERR_UNSUPPORTED, "triangles need physics mode (compat off): the reference's residual is quad-only");
        }
        if (!build_operators_tri(s->P, params->flux_type, tri, msg)) { delete s; return fail(nullptr, ZJ_ERR_ARG, msg); }
        s->nt = tri.nt;
        tri_packed = tri.Dr;
        tri_packed.insert(tri_packed.end(), tri.Ds.begin(), tri.Ds.end());
        tri_packed.insert(tri_packed.end(), tri.L.begin(), tri.L.end());
        tri_packed.insert(tri_packed.end(), tri.Phi.begin(), tri.Phi.end());
    }
    s->etype = s->mesh.etype;
    std::vector<double> J, Jinv, bc, nrm, area, packed;
    std::vector<EdgeRec> rec;
    if (!build_metrics(s->mesh, s->ops, J, Jinv, msg, s->n_tri ? &tri : nullptr)) {
        delete s;
        return fail(nullptr, ZJ_ERR_ARG, msg);
    }
    build_bc_data(s->mesh, params, bc);
    build_edge_records(s->mesh, rec, nrm);
    if (!params->compat && s->mesh.order > 1) {
        // curved elements: the conservative face term takes the normal and
        // the edge Jacobian of every flux point (compat mode keeps the
        // reference's one normal per face)
        build_point_normals(s->mesh, s->ops, nrm);
        s->nrm_pp = 1;
    }
    element_areas(s->mesh, area);
    for (auto& a : area) a = std::sqrt(a);
    pack_ops(s->ops, packed);
    s->n_ghost = s->mesh.n_bnd_faces;
    if (s->is_part) {
        // this part's rows of every per-element array
        const PartSlice& ps = s->part;
        J = slice_rows(ps, J, (size_t)s->nsp);
        Jinv = slice_rows(ps, Jinv, (size_t)s->nsp * 4);
        nrm = slice_rows(ps, nrm, (size_t)(s->nrm_pp ? 4 * s->n1 * 4 : 4 * 4));
        area = slice_rows(ps, area, 1);
        std::vector<EdgeRec> lrec;
        slice_edge_records(ps, rec, lrec);
        rec.swap(lrec);
        bc = slice_bc_data(ps, bc);
        std::vector<int8_t> et;
        for (int64_t g : ps.elems) et.push_back(s->etype[(size_t)g]);
        s->etype.swap(et);
        s->E = (int64_t)ps.elems.size();
        s->n_quad = s->E;
        s->n_ghost = (int64_t)(ps.bnd_slots.size() + ps.mine.size());
    }

    s->n_jinv = Jinv.size(); s->n_j = J.size(); s->n_ops = packed.size();
    s->n_bcd = bc.size(); s->n_nrm = nrm.size() / 4;
    s->state_n = (size_t)s->E * s->nsp * 4;
    // element traces, then one ghost row per boundary slot and, for a part,
    // per interface (physics mode)
    s->trace_n = ((size_t)s->E * 4 + (size_t)s->n_ghost) * s->n1 * 4;
    s->grid = stage_grid(s->P, s->E);
    std::vector<int32_t> listq, listt;
    if (s->n_tri > 0) {
        for (int64_t e2 = 0; e2 < s->E; ++e2)
            (s->etype[(size_t)e2] == ZJ_ELEM_TRI ? listt : listq).push_back((int32_t)e2);
        s->grid_q = quad_grid(s->P, s->n_quad);
        s->grid_t = tri_grid(s->P, s->n_tri);
        s->grid = s->grid_q + s->grid_t;
    }
    s->scratch_n = 148 * 8;
    cudaError_t e = cudaGetDevice(&s->device);
#define ZJ_ALLOC(ptr, n)                                                     \
    if (e == cudaSuccess) e = dalloc(&(ptr), (n));
    for (int i = 0; i < 3; ++i) { ZJ_ALLOC(s->dU[i], s->state_n); }
    s->mixed = params->precision != ZJ_FP64;
    s->tc = params->precision == ZJ_SPLIT_BF16 && tc_order_supported(s->P) && is_ns(s) && s->n_tri == 0;
    std::vector<uint16_t> tc_img;
    if (s->tc) {
        build_tc_image(s->P, s->ops, tc_img);
        s->grid = tc_grid(s->P, s->E);
        ZJ_ALLOC(s->dTcImg, tc_img.size());
        ZJ_ALLOC(s->dTcErr, 1);
    }
    if (!s->mixed) {
        for (int i = 0; i < 3; ++i) { ZJ_ALLOC(s->dT[i], s->trace_n); }
        if (is_ns(s)) { ZJ_ALLOC(s->dTQ, 2 * s->trace_n); }
    } else {
        for (int i = 0; i < 3; ++i) { ZJ_ALLOC(s->fT[i], s->trace_n); }
        if (is_ns(s)) { ZJ_ALLOC(s->fTQ, 2 * s->trace_n); }
        ZJ_ALLOC(s->fJinv, Jinv.size());
        ZJ_ALLOC(s->fJ, J.size());
        ZJ_ALLOC(s->fOps, packed.size());
        ZJ_ALLOC(s->fBC, bc.size());
        ZJ_ALLOC(s->fNrm, nrm.size() / 4);
    }
    ZJ_ALLOC(s->dUs, s->state_n);
    ZJ_ALLOC(s->dRs, s->state_n);
    ZJ_ALLOC(s->dJinv, Jinv.size());
    ZJ_ALLOC(s->dJ, J.size());
    ZJ_ALLOC(s->dOps, packed.size());
    ZJ_ALLOC(s->dBC, bc.size());
    ZJ_ALLOC(s->dH, area.size());
    ZJ_ALLOC(s->dScal, 8);
    ZJ_ALLOC(s->dPart, (size_t)s->grid);
    ZJ_ALLOC(s->dPartR, (size_t)s->grid);
    ZJ_ALLOC(s->dScratch, (size_t)s->scratch_n);
    ZJ_ALLOC(s->dFlag, 1);
    ZJ_ALLOC(s->dEdges, rec.size());
    ZJ_ALLOC(s->dNrm, nrm.size() / 4);
    if (s->n_tri > 0) {
        ZJ_ALLOC(s->dElistQ, listq.size());
        ZJ_ALLOC(s->dElistT, listt.size());
        ZJ_ALLOC(s->dTriOps, tri_packed.size());
        ZJ_ALLOC(s->dEtype, (size_t)s->E);
        if (s->mixed) { ZJ_ALLOC(s->fTriOps, tri_packed.size()); }
    }
#undef ZJ_ALLOC
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemcpy(s->dJinv, Jinv.data(), Jinv.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->dJ, J.data(), J.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->dOps, packed.data(), packed.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->dBC, bc.data(), bc.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->dH, area.data(), area.size() * 8, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->dEdges, rec.data(), rec.size() * sizeof(EdgeRec), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(s->dNrm, nrm.data(), nrm.size() * 8, cudaMemcpyHostToDevice);
    if (s->tc) {
        if (e == cudaSuccess) e = cudaMemcpy(s->dTcImg, tc_img.data(), tc_img.size() * 2, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(s->dTcErr, 0, sizeof(int));
        if (e == cudaSuccess) e = make_tc_tensor_map(s->P, s->dTcImg, &s->tc_map);
    }
    if (s->mixed) {
        // The geometry is computed once in FP64 on the host and rounded to
        // FP32 for the mixed-precision kernels.
        const std::vector<float> fJinv = narrow<float>(Jinv), fJ = narrow<float>(J),
                                 fOps = narrow<float>(packed), fBC = narrow<float>(bc),
                                 fNrm = narrow<float>(nrm);
        if (e == cudaSuccess) e = cudaMemcpy(s->fJinv, fJinv.data(), fJinv.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->fJ, fJ.data(), fJ.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->fOps, fOps.data(), fOps.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->fBC, fBC.data(), fBC.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->fNrm, fNrm.data(), fNrm.size() * 4, cudaMemcpyHostToDevice);
    }
    if (s->n_tri > 0) {
        if (e == cudaSuccess && !listq.empty())
            e = cudaMemcpy(s->dElistQ, listq.data(), listq.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->dElistT, listt.data(), listt.size() * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess)
            e = cudaMemcpy(s->dTriOps, tri_packed.data(), tri_packed.size() * 8, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(s->dEtype, s->etype.data(), (size_t)s->E, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && s->mixed) {
            const std::vector<float> f = narrow<float>(tri_packed);
            e = cudaMemcpy(s->fTriOps, f.data(), f.size() * 4, cudaMemcpyHostToDevice);
        }
    }
    if (s->is_part && e == cudaSuccess) {
        // halo rows: this part's side of every interface (sent), and the
        // interfaces' ghost rows E*4 + n_bnd + k (received), in the plan's
        // order (neighbours ascending, global face order within each)
        const PartSlice& ps = s->part;
        const size_t ni = ps.mine.size();
        std::vector<int32_t> send(ni), recv(ni);
        const int64_t nb = (int64_t)ps.bnd_slots.size();
        for (size_t k = 0; k < ni; ++k) {
            send[k] = (int32_t)(ps.g2l[(size_t)(ps.mine[k] / 4)] * 4 + ps.mine[k] % 4);
            recv[k] = (int32_t)(s->E * 4 + nb + (int64_t)k);
        }
        const size_t tsz = s->mixed ? sizeof(float) : sizeof(double);
        e = dalloc(&s->dSendRows, ni);
        if (e == cudaSuccess) e = dalloc(&s->dRecvRows, ni);
        if (e == cudaSuccess) e = cudaMalloc(&s->dSendBuf, std::max<size_t>(ni, 1) * s->n1 * 8 * tsz);
        if (e == cudaSuccess) e = cudaMalloc(&s->dRecvBuf, std::max<size_t>(ni, 1) * s->n1 * 8 * tsz);
        if (e == cudaSuccess && ni)
            e = cudaMemcpy(s->dSendRows, send.data(), ni * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess && ni)
            e = cudaMemcpy(s->dRecvRows, recv.data(), ni * 4, cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_pack, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->ev_join, cudaEventDisableTiming);
    }
    // every state buffer starts at zero: slots no kernel writes (a
    // triangle's unused ones) stay finite through the buffer rotation
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaMemset(s->dU[i], 0, s->state_n * 8);
    if (e == cudaSuccess) e = cudaMemset(s->dScal, 0, 8 * 8);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        std::string m = std::string("device setup: ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")";
        free_all(s);
        delete s;
        return fail(nullptr, ZJ_ERR_CUDA, m);
    }
    s->stream = s->own;
    *out = s;
    return ZJ_OK;
}

}  // namespace

extern "C" {

zj_status zj_solver_create(const zj_mesh_desc* mesh, const zj_params* params, zj_solver** out) {
    return create_impl(mesh, params, nullptr, 1, 0, out);
}

void zj_solver_destroy(zj_solver* s) {
    if (!s) return;
    if (s->stream) cudaStreamSynchronize(s->stream);
    free_all(s);
    delete s;
}

int64_t zj_num_elements(const zj_solver* s) { return s ? s->E : 0; }
int zj_num_solution_points(const zj_solver* s) { return s ? s->nsp : 0; }
int64_t zj_num_faces(const zj_solver* s) { return s ? s->mesh.n_faces : 0; }
int64_t zj_state_size(const zj_solver* s) { return s ? (int64_t)s->state_n : 0; }
double zj_time(const zj_solver* s) { return s ? s->time : 0.0; }
int zj_iteration(const zj_solver* s) { return s ? s->iter : 0; }

zj_status zj_solution_point_coords(const zj_solver* s, double* xy) {
    if (!s || !xy) return ZJ_ERR_ARG;
    std::vector<double> c;
    TriOperators tri;
    std::string msg;
    if (s->n_tri > 0 && !build_operators_tri(s->P, s->prm.flux_type, tri, msg)) return fail(const_cast<zj_solver*>(s), ZJ_ERR_ARG, msg);
    sp_coords(s->mesh, s->ops, c, s->n_tri ? &tri : nullptr);
    if (s->is_part) c = slice_rows(s->part, c, (size_t)s->nsp * 2);
    std::memcpy(xy, c.data(), c.size() * sizeof(double));
    return ZJ_OK;
}

zj_status zj_element_kinds(const zj_solver* s, int32_t* kinds) {
    if (!s || !kinds) return ZJ_ERR_ARG;
    for (int64_t e = 0; e < s->E; ++e) kinds[e] = s->etype[(size_t)e];
    return ZJ_OK;
}

int zj_num_triangle_points(const zj_solver* s) { return s ? ((s->P + 1) * (s->P + 2) / 2) : 0; }

zj_status zj_set_stream(zj_solver* s, void* stream) {
    if (!s) return ZJ_ERR_ARG;
    s->stream = static_cast<cudaStream_t>(stream);
    return ZJ_OK;
}

void* zj_get_stream(const zj_solver* s) { return s ? static_cast<void*>(s->stream) : nullptr; }

zj_status zj_set_step_graphs(zj_solver* s, int enable) {
    if (!s) return ZJ_ERR_ARG;
    s->graphs_on = enable != 0;
    return ZJ_OK;
}

zj_status zj_set_state(zj_solver* s, const double* U) {
    if (!s || !U) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(s->dU[s->cur], U, s->state_n * 8, cudaMemcpyHostToDevice, s->stream), "set_state copy");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "set_state sync");
    s->traces_valid = false;
    s->has_norm = false;
    s->time = 0.0;
    s->iter = 0;
    return ZJ_OK;
}

zj_status zj_get_state(zj_solver* s, double* U) {
    if (!s || !U) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(U, s->dU[s->cur], s->state_n * 8, cudaMemcpyDeviceToHost, s->stream), "get_state copy");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "get_state sync");
    return ZJ_OK;
}

zj_status zj_set_state_async(zj_solver* s, const double* U) {
    if (!s || !U) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(s->dU[s->cur], U, s->state_n * 8, cudaMemcpyHostToDevice, s->stream), "set_state_async copy");
    s->traces_valid = false;
    s->has_norm = false;
    s->time = 0.0;
    s->iter = 0;
    return ZJ_OK;
}

zj_status zj_get_state_async(zj_solver* s, double* U) {
    if (!s || !U) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(U, s->dU[s->cur], s->state_n * 8, cudaMemcpyDeviceToHost, s->stream), "get_state_async copy");
    return ZJ_OK;
}

zj_status zj_set_state_device(zj_solver* s, const double* U) {
    if (!s || !U) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(s->dU[s->cur], U, s->state_n * 8, cudaMemcpyDeviceToDevice, s->stream), "set_state_device copy");
    s->traces_valid = false;
    s->has_norm = false;
    s->time = 0.0;
    s->iter = 0;
    return ZJ_OK;
}

zj_status zj_get_state_device(zj_solver* s, double* U) {
    if (!s || !U) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(U, s->dU[s->cur], s->state_n * 8, cudaMemcpyDeviceToDevice, s->stream), "get_state_device copy");
    return ZJ_OK;
}

// A part's interfaces are filled by the multi-part driver (zj_parts_*).
static zj_status refuse_part(zj_solver* s) {
    return fail(s, ZJ_ERR_UNSUPPORTED, "a part of a partitioned mesh steps and evaluates through zj_parts_step / zj_parts_rhs");
}

zj_status zj_step(zj_solver* s, double dt, int nsteps) {
    if (!s) return ZJ_ERR_ARG;
    if (s->is_part) return refuse_part(s);
    if (nsteps < 0 || !std::isfinite(dt)) return fail(s, ZJ_ERR_ARG, "bad dt or nsteps");
    if (nsteps == 0) return ZJ_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    ZJ_CK(s, cudaStreamIsCapturing(s->stream, &cs), "capture query");
    if (cs != cudaStreamCaptureStatusNone) {
        // a caller's capture: the graph sets dt on every replay, and the next
        // direct call sets it again (replays may have changed it)
        k_set_dt<<<1, 1, 0, s->stream>>>(s->dScal, dt);
        ZJ_CK(s, cudaGetLastError(), "dt launch");
        s->last_dt = std::nan("");
    } else if (dt != s->last_dt) {
        k_set_dt<<<1, 1, 0, s->stream>>>(s->dScal, dt);
        ZJ_CK(s, cudaGetLastError(), "dt launch");
        s->last_dt = dt;
    }
    zj_status st = s->mixed ? step_impl<float>(s, nsteps, dt) : step_impl<double>(s, nsteps, dt);
    if (st != ZJ_OK) return st;
    s->has_norm = true;
    return ZJ_OK;
}

zj_status zj_synchronize(zj_solver* s) {
    if (!s) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "synchronize");
    return ZJ_OK;
}

}  // extern "C"

namespace {
// The kernels read and write state rows as single 32-byte accesses, so a
// caller's device arrays must start on a 32-byte boundary (cudaMalloc and
// torch allocations do).
bool misaligned(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 31u) != 0; }
constexpr const char* kAlignMsg = "device arrays must be 32-byte aligned";
}  // namespace

extern "C" {

zj_status zj_rhs(zj_solver* s, const double* U_dev, double* R_dev) {
    if (!s || !U_dev || !R_dev) return ZJ_ERR_ARG;
    if (s->is_part) return refuse_part(s);
    if (misaligned(U_dev) || misaligned(R_dev)) return fail(s, ZJ_ERR_ARG, kAlignMsg);
    if (s->mixed) return rhs_impl<float>(s, U_dev, R_dev, s->fT[2], nullptr, s->dPartR);
    return rhs_impl<double>(s, U_dev, R_dev, s->dT[2], nullptr, s->dPartR);
}

zj_status zj_rhs_host(zj_solver* s, const double* U, double* R) {
    if (!s || !U || !R) return ZJ_ERR_ARG;
    ZJ_CK(s, cudaMemcpyAsync(s->dUs, U, s->state_n * 8, cudaMemcpyHostToDevice, s->stream), "rhs upload");
    zj_status st = zj_rhs(s, s->dUs, s->dRs);
    if (st != ZJ_OK) return st;
    ZJ_CK(s, cudaMemcpyAsync(R, s->dRs, s->state_n * 8, cudaMemcpyDeviceToHost, s->stream), "rhs download");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "rhs sync");
    return ZJ_OK;
}

zj_status zj_residual_norm(zj_solver* s, double* out) {
    if (!s || !out) return ZJ_ERR_ARG;
    if (!s->has_norm) { *out = 0.0; return ZJ_OK; }
    ZJ_CK(s, launch_reduce_sum(s->dPart, s->grid, s->dScal + 1, s->stream), "norm reduce");
    double v = 0.0;
    ZJ_CK(s, cudaMemcpyAsync(&v, s->dScal + 1, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "norm copy");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "norm sync");
    *out = std::sqrt(v);
    return ZJ_OK;
}

zj_status zj_compute_dt(zj_solver* s, double* dt_out) {
    if (!s || !dt_out) return ZJ_ERR_ARG;
    ZJ_CK(s, launch_compute_dt(s->dU[s->cur], s->dH, s->E, s->nsp, s->prm.gamma, s->prm.CFL, s->P,
                               s->dScratch, s->scratch_n, s->dScal + 2, s->stream, s->dEtype, s->nt),
          "dt launch");
    double v = 0.0;
    ZJ_CK(s, cudaMemcpyAsync(&v, s->dScal + 2, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "dt copy");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "dt sync");
    *dt_out = v;
    return ZJ_OK;
}

zj_status zj_check_state(zj_solver* s) {
    if (!s) return ZJ_ERR_ARG;
    ZJ_CK(s, launch_check_finite(s->dU[s->cur], (long long)s->state_n, s->dFlag, s->stream), "check launch");
    int flag = 0;
    ZJ_CK(s, cudaMemcpyAsync(&flag, s->dFlag, sizeof(int), cudaMemcpyDeviceToHost, s->stream), "check copy");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "check sync");
    if (flag) return fail(s, ZJ_ERR_NAN, "state holds NaN or Inf");
    if (s->tc) {
        int tflag = 0;
        ZJ_CK(s, cudaMemcpy(&tflag, s->dTcErr, sizeof(int), cudaMemcpyDeviceToHost), "tensor-core flag copy");
        if (tflag)
            return fail(s, ZJ_ERR_TIMEOUT, "a split-BF16 stage gave up waiting for its operator copy or its tensor-core product");
    }
    return ZJ_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free residual.  Some callers may not allocate device memory at
// the point where they need a residual: a host application whose device
// memory is reserved up front by its own pool allocator, or a time-critical
// loop where the implicit synchronisation of cudaMalloc/cudaFree is not
// allowed.  zj_rhs_noalloc serves them: its per-call scratch (the trace buffer
// of the residual and the per-CTA partial sums) lives in this file-scope
// array instead of the handle's buffers, so the call allocates and frees
// nothing.  The array is a fixed ZJ_NOALLOC_SCRATCH_BYTES that every GPU which
// loads this library holds until the process exits.
static __device__ __align__(256) double g_noalloc_scratch[ZJ_NOALLOC_SCRATCH_BYTES / sizeof(double)];

namespace {

// Device address of g_noalloc_scratch per device.  In host code the array's
// name only stands in for the symbol; a kernel must be given the address
// cudaGetSymbolAddress returns with that device current.  The address is
// looked up once per device and kept for the life of the process, so the
// library must not be used across a cudaDeviceReset of that device (which
// reloads the module).
constexpr int kMaxDevices = 64;
double* g_noalloc_ptr[kMaxDevices] = {};
std::mutex g_noalloc_mutex;

cudaError_t noalloc_scratch(double** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return cudaSuccess;
}

}  // namespace

extern "C" {

zj_status zj_rhs_noalloc(zj_solver* s, const double* U_dev, double* R_dev) {
    if (!s || !U_dev || !R_dev) return ZJ_ERR_ARG;
    if (s->is_part) return refuse_part(s);
    if (misaligned(U_dev) || misaligned(R_dev)) return fail(s, ZJ_ERR_ARG, kAlignMsg);
    int dev = -1;
    ZJ_CK(s, cudaGetDevice(&dev), "current device");
    if (dev != s->device)
        return fail(s, ZJ_ERR_ARG,
                    "zj_rhs_noalloc: device " + std::to_string(dev) + " is current, the handle was created on device " +
                        std::to_string(s->device) + " (the static scratch is per device)");
    const size_t tsz = s->mixed ? sizeof(float) : sizeof(double);
    const size_t trace_bytes = (is_ns(s) ? 3 : 1) * s->trace_n * tsz;
    const size_t part_bytes = (size_t)s->grid * sizeof(double);
    const size_t need = trace_bytes + part_bytes;
    if (need > ZJ_NOALLOC_SCRATCH_BYTES)
        return fail(s, ZJ_ERR_ARG,
                    "mesh too large for zj_rhs_noalloc: needs " + std::to_string(need) +
                        " bytes of scratch, the static limit is " +
                        std::to_string((size_t)ZJ_NOALLOC_SCRATCH_BYTES) + " bytes");
    double* scratch = nullptr;
    ZJ_CK(s, noalloc_scratch(&scratch), "static scratch address");
    // Every scratch value is written before it is read (all traces by the
    // trace launch, the gradient traces by the gradient launch, one partial
    // per CTA), so nothing needs clearing.  The gradient traces (read and
    // written as 32-byte rows) come first, at the array's 256-byte aligned
    // start; the traces follow at 2 trace_n values (a multiple of 32 bytes,
    // trace_n being a multiple of 4), the partials after them at a multiple of
    // 16 bytes.
    char* base = reinterpret_cast<char*>(scratch);
    double* partials = reinterpret_cast<double*>(base + trace_bytes);
    const size_t tq_n = is_ns(s) ? 2 * s->trace_n : 0;
    if (s->mixed) {
        float* tq = reinterpret_cast<float*>(base);
        return rhs_impl<float>(s, U_dev, R_dev, tq + tq_n, is_ns(s) ? tq : nullptr, partials);
    }
    return rhs_impl<double>(s, U_dev, R_dev, scratch + tq_n, is_ns(s) ? scratch : nullptr, partials);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Differentiation (physics mode, FP64): Jacobian-vector products on dual
// numbers (jvp.cu), vector-Jacobian products by the transposed kernels
// (adjoint.cu), the adjoint of an SSP-RK3 step and the checkpointed discrete
// adjoint of a run.
namespace {

zj_status diff_supported(zj_solver* s) {
    if (s->prm.compat) return fail(s, ZJ_ERR_UNSUPPORTED, "differentiation needs physics mode (compat off)");
    if (s->mixed) return fail(s, ZJ_ERR_UNSUPPORTED, "differentiation runs on the FP64 path (precision fp64)");
    if (s->n_tri > 0) return fail(s, ZJ_ERR_UNSUPPORTED, "differentiation runs on quadrilateral meshes");
    if (s->nrm_pp) return fail(s, ZJ_ERR_UNSUPPORTED, "differentiation runs on straight-edged (Q1) meshes");
    if (s->is_part) return fail(s, ZJ_ERR_UNSUPPORTED, "differentiation runs on a whole mesh, not a part");
    return ZJ_OK;
}


zj_status ensure_diff(zj_solver* s) {
    if (s->diff_ready) return ZJ_OK;
    cudaError_t e = cudaSuccess;
#define ZJ_ALLOC(ptr, n) \
    if (e == cudaSuccess) e = dalloc(&(ptr), (n));
    ZJ_ALLOC(s->xJinv, s->n_jinv);
    ZJ_ALLOC(s->xJ, s->n_j);
    ZJ_ALLOC(s->xOps, s->n_ops);
    ZJ_ALLOC(s->xBC, s->n_bcd);
    ZJ_ALLOC(s->xNrm, s->n_nrm);
    ZJ_ALLOC(s->xT, s->trace_n);
    ZJ_ALLOC(s->xTQ, 2 * s->trace_n);
    ZJ_ALLOC(s->xPart, (size_t)dual_grid(s->P, s->E));
    const size_t fpn = (size_t)s->E * 4 * s->n1 * 4;
    ZJ_ALLOC(s->aDb, fpn);
    ZJ_ALLOC(s->aTb, fpn);
    ZJ_ALLOC(s->aDUb, fpn);
    double** st[] = {&s->aW, &s->aS1, &s->aS2, &s->aB0, &s->aB1, &s->aB2, &s->aR, &s->aJV, &s->aZero};
    for (auto pp : st) { ZJ_ALLOC(*pp, s->state_n); }
    ZJ_ALLOC(s->aDot, (size_t)dot_grid());
    ZJ_ALLOC(s->aScal, 8);
    ZJ_ALLOC(s->aRePart, (size_t)adj_ns_grid(s->P, s->E));
#undef ZJ_ALLOC
    if (e == cudaSuccess) e = launch_to_dual(s->dJinv, s->xJinv, (long long)s->n_jinv, s->stream);
    if (e == cudaSuccess) e = launch_to_dual(s->dJ, s->xJ, (long long)s->n_j, s->stream);
    if (e == cudaSuccess) e = launch_to_dual(s->dOps, s->xOps, (long long)s->n_ops, s->stream);
    if (e == cudaSuccess) e = launch_to_dual(s->dBC, s->xBC, (long long)s->n_bcd, s->stream);
    if (e == cudaSuccess)
        e = launch_to_dual(reinterpret_cast<const double*>(s->dNrm), reinterpret_cast<Dual*>(s->xNrm),
                           (long long)s->n_nrm * 4, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->aZero, 0, s->state_n * 8, s->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->aScal, 0, 8 * 8, s->stream);
    if (e != cudaSuccess) return cuda_fail(s, e, "differentiation buffers");
    s->diff_ready = true;
    return ZJ_OK;
}

// R (if R != NULL) and JV = dR/dU . V + dR/dRe dRe.
zj_status jvp_core(zj_solver* s, const double* U, const double* V, double dRe, double* R, double* JV) {
    StageArgsT<Dual> a{};
    a.Jinv = s->xJinv; a.J = s->xJ; a.enrm = s->xNrm; a.bc = s->xBC; a.ops = s->xOps;
    a.edges = s->dEdges; a.dt = s->dScal; a.n_elem = s->E; a.gamma = s->prm.gamma;
    a.Re = s->prm.Re; a.Pr = s->prm.Pr; a.dRe = dRe;
    set_viscous_constants(a);
    a.U = U; a.U0 = U; a.dU = V; a.Tout = s->xT;
    ZJ_CK(s, launch_phys_traces(s->P, a, s->stream), "jvp trace launch");
    a.Tin = s->xT; a.TQ = s->xTQ; a.TQout = s->xTQ;
    a.R = R ? R : s->aR; a.dR = JV; a.partials = s->xPart; a.stage = 0;
    if (is_ns(s)) {
        ZJ_CK(s, launch_ns_grad(s->P, a, s->stream), "jvp gradient launch");
        ZJ_CK(s, launch_ns_stage(s->P, s->prm.riemann, a, s->stream), "jvp residual launch");
    } else {
        ZJ_CK(s, launch_phys_stage(s->P, s->prm.riemann, a, s->stream), "jvp residual launch");
    }
    return ZJ_OK;
}

// Fused output of a VJP: out = c0 X0 + c1 X1 + c2 X2 + cw (dR/dU)^T L.
struct VjpOut {
    double* out = nullptr;
    const double* X0 = nullptr;
    const double* X1 = nullptr;
    const double* X2 = nullptr;
    double c0 = 0.0, c1 = 0.0, c2 = 0.0, cw = 1.0;
};

// W = (dR/dU)^T L (or the fused update o); for Navier-Stokes with
// re_weight != 0 also aScal[0] += re_weight * L . dR/dRe (reduced from the
// VJP's per-CTA sums).
zj_status vjp_core(zj_solver* s, const double* U, const double* L, double* W, double re_weight = 0.0,
                   const VjpOut& o = VjpOut(), const double* T = nullptr, const double* TQ = nullptr) {
    if (!T) {
        // traces and gradient traces of U, unless the caller kept them from
        // the forward recomputation
        ZJ_CK(s, launch_trace_any(s, U, s->dT[2]), "vjp trace launch");
        T = s->dT[2];
        if (is_ns(s)) {
            StageArgs a = stage_args<double>(s);
            a.U = U; a.Tin = T; a.TQout = s->dTQ;
            ZJ_CK(s, launch_ns_grad(s->P, a, s->stream), "vjp gradient launch");
            TQ = s->dTQ;
        }
    }
    AdjArgs g{};
    g.U = U; g.L = L; g.W = W; g.T = T; g.TQ = TQ;
    g.Db = s->aDb; g.Tb = s->aTb; g.DUb = s->aDUb;
    g.Jinv = s->dJinv; g.J = s->dJ; g.edges = s->dEdges; g.enrm = s->dNrm; g.bc = s->dBC; g.ops = s->dOps;
    g.n_elem = s->E; g.gamma = s->prm.gamma; g.Re = s->prm.Re; g.Pr = s->prm.Pr;
    const bool re = is_ns(s) && re_weight != 0.0;
    g.re_part = re ? s->aRePart : nullptr;
    g.out = o.out; g.X0 = o.X0; g.X1 = o.X1; g.X2 = o.X2;
    g.c0 = o.c0; g.c1 = o.c1; g.c2 = o.c2; g.cw = o.cw;
    ZJ_CK(s, launch_rhs_vjp(s->P, s->prm.riemann, is_ns(s), g, s->stream), "vjp launch");
    if (re) {
        ZJ_CK(s, launch_reduce_sum(s->aRePart, adj_ns_grid(s->P, s->E), s->aScal + 1, s->stream), "re reduce");
        ZJ_CK(s, launch_lincomb(s->aScal, 1.0, s->aScal, re_weight, s->aScal + 1, 0.0, nullptr, 1, s->stream),
              "re accumulate");
    }
    return ZJ_OK;
}

zj_status set_dt(zj_solver* s, double dt) {
    if (dt != s->last_dt) {
        ZJ_CK(s, cudaMemcpyAsync(s->dScal, &dt, sizeof(double), cudaMemcpyHostToDevice, s->stream), "dt upload");
        ZJ_CK(s, cudaStreamSynchronize(s->stream), "dt upload sync");
        s->last_dt = dt;
    }
    return ZJ_OK;
}

// Per-stage traces and gradient traces kept from a forward recomputation
// (T[k], TQ[k] of stage input state k = X, U(1), U(2)); NULL entries mean
// the handle's scratch buffers.
struct StageTraces {
    double* T[3] = {nullptr, nullptr, nullptr};
    double* TQ[3] = {nullptr, nullptr, nullptr};
};

// Stage launches of one SSP-RK3 step from X (handle's stage machinery on
// caller buffers): U(1) into S1, U(2) into S2 and, if Xout != NULL, the new
// state into Xout (may be X).  Without keep, uses the stepper's trace
// buffers; with keep, writes every stage input's traces and gradient traces
// into keep's buffers (the third stage's gradient traces even when Xout is
// NULL).
zj_status rk3_stages(zj_solver* s, const double* X, double* S1, double* S2, double* Xout,
                     const StageTraces* keep = nullptr) {
    double* T[3] = {s->dT[0], s->dT[1], s->dT[0]};
    double* TQ[3] = {s->dTQ, s->dTQ, s->dTQ};
    if (keep)
        for (int k = 0; k < 3; ++k) { T[k] = keep->T[k]; TQ[k] = keep->TQ[k]; }
    ZJ_CK(s, launch_trace_any(s, X, T[0]), "trace launch");
    StageArgs a = stage_args<double>(s);
    a.partials = s->dPartR;
    a.U = X; a.U0 = X; a.Uout = S1; a.Tin = T[0]; a.Tout = T[1]; a.TQ = a.TQout = TQ[0]; a.stage = 1;
    ZJ_CK(s, launch_stage(s, a), "stage 1 launch");
    a.U = S1; a.Uout = S2; a.Tin = T[1]; a.Tout = T[2]; a.TQ = a.TQout = TQ[1]; a.stage = 2;
    ZJ_CK(s, launch_stage(s, a), "stage 2 launch");
    a.U = S2; a.Tin = T[2]; a.TQ = a.TQout = TQ[2];
    if (Xout) {
        a.Uout = Xout; a.Tout = s->dT[1]; a.stage = 3;
        ZJ_CK(s, launch_stage(s, a), "stage 3 launch");
    } else if (keep && is_ns(s)) {
        ZJ_CK(s, launch_ns_grad(s->P, a, s->stream), "gradient launch");
    }
    s->traces_valid = false;   // the stepper's traces now hold this step's
    return ZJ_OK;
}

// Adjoint of one SSP-RK3 step from U0 (dt already on the device):
//   U1 = U0 + dt R(U0), U2 = 3/4 U0 + 1/4 U1 + 1/4 dt R(U1),
//   U3 = 1/3 U0 + 2/3 U2 + 2/3 dt R(U2);
// B = dJ/dU3 in, A = dJ/dU0 out (A may alias B).  S1, S2: the stage states
// if the caller kept them, else NULL (recomputed here).  With re, w dt times
// each stage's L . dR/dRe is added to aScal[0].
zj_status step_vjp_core(zj_solver* s, const double* U0, const double* S1, const double* S2, double dt,
                        const double* B, double* A, bool re, const StageTraces* kept = nullptr) {
    zj_status st = ZJ_OK;
    if (!S1) {
        if ((st = rk3_stages(s, U0, s->aS1, s->aS2, nullptr)) != ZJ_OK) return st;
        S1 = s->aS1;
        S2 = s->aS2;
    }
    const double* T[3] = {nullptr, nullptr, nullptr};
    const double* TQ[3] = {nullptr, nullptr, nullptr};
    if (kept)
        for (int k = 0; k < 3; ++k) { T[k] = kept->T[k]; TQ[k] = kept->TQ[k]; }
    // stage 3: B2 = 2/3 B + 2/3 dt (dR/dU(U2))^T B
    VjpOut o3;
    o3.out = s->aB2; o3.X0 = B; o3.c0 = 2.0 / 3.0; o3.cw = 2.0 / 3.0 * dt;
    if ((st = vjp_core(s, S2, B, s->aW, re ? 2.0 / 3.0 * dt : 0.0, o3, T[2], TQ[2])) != ZJ_OK) return st;
    // stage 2: B1 = 1/4 B2 + 1/4 dt (dR/dU(U1))^T B2
    VjpOut o2;
    o2.out = s->aB1; o2.X0 = s->aB2; o2.c0 = 0.25; o2.cw = 0.25 * dt;
    if ((st = vjp_core(s, S1, s->aB2, s->aW, re ? 0.25 * dt : 0.0, o2, T[1], TQ[1])) != ZJ_OK) return st;
    // stage 1: A = 1/3 B + 3/4 B2 + B1 + dt (dR/dU(U0))^T B1
    VjpOut o1;
    o1.out = A; o1.X0 = B; o1.c0 = 1.0 / 3.0; o1.X1 = s->aB2; o1.c1 = 0.75; o1.X2 = s->aB1; o1.c2 = 1.0;
    o1.cw = dt;
    if ((st = vjp_core(s, U0, s->aB1, s->aW, re ? dt : 0.0, o1, T[0], TQ[0])) != ZJ_OK) return st;
    return ZJ_OK;
}

}  // namespace

extern "C" {

zj_status zj_rhs_jvp(zj_solver* s, const double* U_dev, const double* V_dev, double dRe,
                     double* R_dev, double* JV_dev) {
    if (!s || !U_dev || !V_dev || !JV_dev) return ZJ_ERR_ARG;
    if (misaligned(U_dev) || misaligned(V_dev) || misaligned(JV_dev) || (R_dev && misaligned(R_dev)))
        return fail(s, ZJ_ERR_ARG, kAlignMsg);
    zj_status st = diff_supported(s);
    if (st == ZJ_OK) st = ensure_diff(s);
    if (st == ZJ_OK) st = jvp_core(s, U_dev, V_dev, dRe, R_dev, JV_dev);
    return st;
}

zj_status zj_rhs_vjp(zj_solver* s, const double* U_dev, const double* L_dev, double* W_dev,
                     double* dRe_out) {
    if (!s || !U_dev || !L_dev || !W_dev) return ZJ_ERR_ARG;
    if (misaligned(U_dev) || misaligned(L_dev) || misaligned(W_dev))
        return fail(s, ZJ_ERR_ARG, kAlignMsg);
    zj_status st = diff_supported(s);
    if (st == ZJ_OK) st = ensure_diff(s);
    if (st != ZJ_OK) return st;
    if (dRe_out) ZJ_CK(s, cudaMemsetAsync(s->aScal, 0, sizeof(double), s->stream), "clear");
    if ((st = vjp_core(s, U_dev, L_dev, W_dev, dRe_out ? 1.0 : 0.0)) != ZJ_OK || !dRe_out) return st;
    ZJ_CK(s, cudaMemcpyAsync(dRe_out, s->aScal, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "dRe copy");
    ZJ_CK(s, cudaStreamSynchronize(s->stream), "vjp sync");
    return ZJ_OK;
}

zj_status zj_step_vjp(zj_solver* s, const double* U_dev, double dt, const double* B_dev,
                      double* A_dev, double* dRe_acc) {
    if (!s || !U_dev || !B_dev || !A_dev) return ZJ_ERR_ARG;
    if (misaligned(U_dev) || misaligned(B_dev) || misaligned(A_dev)) return fail(s, ZJ_ERR_ARG, kAlignMsg);
    if (!std::isfinite(dt)) return fail(s, ZJ_ERR_ARG, "bad dt");
    zj_status st = diff_supported(s);
    if (st == ZJ_OK) st = ensure_diff(s);
    if (st == ZJ_OK) st = set_dt(s, dt);
    if (st != ZJ_OK) return st;
    if (dRe_acc) ZJ_CK(s, cudaMemsetAsync(s->aScal, 0, sizeof(double), s->stream), "clear");
    if ((st = step_vjp_core(s, U_dev, nullptr, nullptr, dt, B_dev, A_dev, dRe_acc != nullptr)) != ZJ_OK)
        return st;
    if (dRe_acc) {
        double v = 0.0;
        ZJ_CK(s, cudaMemcpyAsync(&v, s->aScal, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "dRe copy");
        ZJ_CK(s, cudaStreamSynchronize(s->stream), "step vjp sync");
        *dRe_acc += v;
    }
    return ZJ_OK;
}

zj_status zj_adjoint_run(zj_solver* s, double dt, int nsteps, int k_ckpt, double* G_dev, double* dRe,
                         int64_t* bytes, double* ms_forward, double* ms_adjoint) {
    if (!s || !G_dev) return ZJ_ERR_ARG;
    if (misaligned(G_dev)) return fail(s, ZJ_ERR_ARG, kAlignMsg);
    if (nsteps < 1 || k_ckpt < 1 || !std::isfinite(dt)) return fail(s, ZJ_ERR_ARG, "bad dt, nsteps or k_ckpt");
    zj_status st = diff_supported(s);
    if (st == ZJ_OK) st = ensure_diff(s);
    if (st == ZJ_OK) st = set_dt(s, dt);
    if (st != ZJ_OK) return st;
    const int n_ck = (nsteps + k_ckpt - 1) / k_ckpt;
    const int seg_n = std::min(k_ckpt, nsteps);
    const size_t sb = s->state_n * sizeof(double);
    double* ck = nullptr;    // checkpoints [n_ck][state]
    double* seg = nullptr;   // step-start states of one segment [seg_n][state]
    double* X = nullptr;     // forward work state
    // per step of a segment: 3 states, and 3 trace sets (traces + gradient
    // traces) of the stage inputs
    const size_t tset = s->trace_n * (is_ns(s) ? 3 : 1);
    double* trs = nullptr;
    cudaError_t e = dalloc(&ck, (size_t)n_ck * s->state_n);
    if (e == cudaSuccess) e = dalloc(&seg, (size_t)3 * seg_n * s->state_n);
    if (e == cudaSuccess) e = dalloc(&trs, (size_t)3 * seg_n * tset);
    if (e == cudaSuccess) e = dalloc(&X, s->state_n);
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int i = 0; i < 4 && e == cudaSuccess; ++i) e = cudaEventCreate(&ev[i]);
    auto cleanup = [&]() {
        for (auto x : ev) if (x) cudaEventDestroy(x);
        if (ck) cudaFree(ck);
        if (seg) cudaFree(seg);
        if (trs) cudaFree(trs);
        if (X) cudaFree(X);
    };
    if (e != cudaSuccess) { cleanup(); return cuda_fail(s, e, "adjoint checkpoint buffers"); }
    const long long n = (long long)s->state_n;
    auto run = [&]() -> zj_status {
        zj_status r = ZJ_OK;
        ZJ_CK(s, cudaMemsetAsync(s->aScal, 0, sizeof(double), s->stream), "clear");
        ZJ_CK(s, cudaMemcpyAsync(X, s->dU[s->cur], sb, cudaMemcpyDeviceToDevice, s->stream), "state copy");
        // segment layout: step m's start state, U(1), U(2) at seg + 3 m states
        auto st_at = [&](int m, int which) { return seg + (size_t)(3 * m + which) * s->state_n; };
        auto traces_at = [&](int m) {
            StageTraces t;
            for (int k = 0; k < 3; ++k) {
                double* base = trs + (size_t)(3 * m + k) * tset;
                t.T[k] = base;
                t.TQ[k] = is_ns(s) ? base + s->trace_n : nullptr;
            }
            return t;
        };
        // forward sweep with checkpoints every k_ckpt steps; the last
        // segment's steps write their stage states and traces straight into
        // the segment buffers (the same kernels with other outputs), so the
        // backward sweep starts without recomputing it
        const int last_first = (n_ck - 1) * k_ckpt, last_len = nsteps - last_first;
        ZJ_CK(s, cudaEventRecord(ev[0], s->stream), "event");
        for (int i = 0; i < nsteps; ++i) {
            if (i < last_first) {
                if (i % k_ckpt == 0)
                    ZJ_CK(s, cudaMemcpyAsync(ck + (size_t)(i / k_ckpt) * s->state_n, X, sb,
                                             cudaMemcpyDeviceToDevice, s->stream), "checkpoint");
                if ((r = rk3_stages(s, X, s->aS1, s->aS2, X)) != ZJ_OK) return r;
                continue;
            }
            const int m = i - last_first;
            if (m == 0)
                ZJ_CK(s, cudaMemcpyAsync(st_at(0, 0), X, sb, cudaMemcpyDeviceToDevice, s->stream), "segment start");
            const StageTraces t = traces_at(m);
            if ((r = rk3_stages(s, st_at(m, 0), st_at(m, 1), st_at(m, 2),
                                (m + 1 < last_len) ? st_at(m + 1, 0) : X, &t)) != ZJ_OK)
                return r;
        }
        ZJ_CK(s, cudaEventRecord(ev[1], s->stream), "event");
        // backward sweep: recompute each earlier segment from its checkpoint,
        // then the step adjoints in reverse
        for (int c = n_ck - 1; c >= 0; --c) {
            const int first = c * k_ckpt, len = std::min(k_ckpt, nsteps - first);
            if (c < n_ck - 1) {
                ZJ_CK(s, cudaMemcpyAsync(st_at(0, 0), ck + (size_t)c * s->state_n, sb,
                                         cudaMemcpyDeviceToDevice, s->stream), "segment start");
                for (int m = 0; m < len; ++m) {
                    const StageTraces t = traces_at(m);
                    if ((r = rk3_stages(s, st_at(m, 0), st_at(m, 1), st_at(m, 2),
                                        (m + 1 < len) ? st_at(m + 1, 0) : nullptr, &t)) != ZJ_OK)
                        return r;
                }
            }
            for (int m = len - 1; m >= 0; --m) {
                const StageTraces t = traces_at(m);
                if ((r = step_vjp_core(s, st_at(m, 0), st_at(m, 1), st_at(m, 2), dt, G_dev, G_dev,
                                       dRe != nullptr, &t)) != ZJ_OK)
                    return r;
            }
        }
        ZJ_CK(s, cudaEventRecord(ev[2], s->stream), "event");
        (void)n;
        return ZJ_OK;
    };
    st = run();
    if (st == ZJ_OK) {
        double v = 0.0;
        e = cudaMemcpyAsync(&v, s->aScal, sizeof(double), cudaMemcpyDeviceToHost, s->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) st = cuda_fail(s, e, "adjoint sync");
        float f = 0.0f, b = 0.0f;
        if (st == ZJ_OK) {
            cudaEventElapsedTime(&f, ev[0], ev[1]);
            cudaEventElapsedTime(&b, ev[1], ev[2]);
            if (dRe) *dRe = v;
            if (ms_forward) *ms_forward = f;
            if (ms_adjoint) *ms_adjoint = b;
            if (bytes)
                *bytes = (int64_t)((size_t)(n_ck + 3 * seg_n + 1 + 9) * sb + (size_t)3 * seg_n * tset * 8);
        }
    }
    cleanup();
    return st;
}

}  // extern "C"

// ------------------------------------------------------------- restart --
namespace {

constexpr char kRestartMagic[8] = {'Z', 'J', 'R', 'E', 'S', 'T', 'R', 'T'};
constexpr uint32_t kRestartVersion = 1;

uint64_t fnv1a(const unsigned char* p, size_t n, uint64_t h = 1469598103934665603ULL) {
    for (size_t i = 0; i < n; ++i) { h ^= p[i]; h *= 1099511628211ULL; }
    return h;
}

struct Bytes {
    std::vector<unsigned char> b;
    template <class T> void put(const T& v) {
        const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
        b.insert(b.end(), p, p + sizeof(T));
    }
    void put_raw(const void* p, size_t n) {
        const unsigned char* c = static_cast<const unsigned char*>(p);
        b.insert(b.end(), c, c + n);
    }
};

}  // namespace

extern "C" {

zj_status zj_restart_write(zj_solver* s, const char* path) {
    if (!s || !path) return ZJ_ERR_ARG;
    std::vector<double> U(s->state_n);
    zj_status st = zj_get_state(s, U.data());
    if (st != ZJ_OK) return st;
    Bytes f;
    f.put_raw(kRestartMagic, 8);
    f.put(kRestartVersion);
    f.put(uint32_t(0));
    f.put(s->time);
    f.put(int32_t(s->iter));
    f.put(int32_t(s->P));
    f.put(s->prm.gamma);
    f.put(int64_t(s->E));
    std::vector<int32_t> nsp((size_t)s->E, s->nsp);
    f.put_raw(nsp.data(), nsp.size() * sizeof(int32_t));
    f.put_raw(U.data(), U.size() * sizeof(double));
    f.put(fnv1a(f.b.data(), f.b.size()));
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(s, ZJ_ERR_IO, std::string("cannot create restart file ") + path);
    const size_t w = std::fwrite(f.b.data(), 1, f.b.size(), fp);
    const int c = std::fclose(fp);
    if (w != f.b.size() || c != 0) return fail(s, ZJ_ERR_IO, std::string("short write to ") + path);
    return ZJ_OK;
}

zj_status zj_restart_read(zj_solver* s, const char* path) {
    if (!s || !path) return ZJ_ERR_ARG;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(s, ZJ_ERR_IO, std::string("cannot open restart file ") + path);
    std::vector<unsigned char> b;
    unsigned char buf[1 << 16];
    size_t n;
    while ((n = std::fread(buf, 1, sizeof(buf), fp)) > 0) b.insert(b.end(), buf, buf + n);
    std::fclose(fp);
    const size_t head = 8 + 4 + 4 + 8 + 4 + 4 + 8 + 8;
    if (b.size() < head + 8) return fail(s, ZJ_ERR_IO, "restart file too short");
    if (std::memcmp(b.data(), kRestartMagic, 8) != 0) return fail(s, ZJ_ERR_ARG, "not a restart file");
    size_t o = 8;
    auto get = [&](auto& v) { std::memcpy(&v, b.data() + o, sizeof(v)); o += sizeof(v); };
    uint32_t version = 0, reserved = 0;
    double time = 0.0, gamma = 0.0;
    int32_t iter = 0, order = 0;
    int64_t ne = 0;
    get(version); get(reserved); get(time); get(iter); get(order); get(gamma); get(ne);
    if (version != kRestartVersion) return fail(s, ZJ_ERR_ARG, "unsupported restart version " + std::to_string(version));
    if (ne != s->E)
        return fail(s, ZJ_ERR_ARG, "restart file has " + std::to_string(ne) + " elements, the mesh " + std::to_string(s->E));
    const size_t need = head + (size_t)ne * 4 + s->state_n * 8 + 8;
    if (b.size() != need) return fail(s, ZJ_ERR_ARG, "restart file size does not match its element count");
    uint64_t sum = 0;
    std::memcpy(&sum, b.data() + b.size() - 8, 8);
    if (sum != fnv1a(b.data(), b.size() - 8)) return fail(s, ZJ_ERR_ARG, "restart file checksum mismatch");
    if (order != s->P)
        return fail(s, ZJ_ERR_ARG, "restart file is poly_order " + std::to_string(order) + ", the solver " + std::to_string(s->P));
    if (gamma != s->prm.gamma) return fail(s, ZJ_ERR_ARG, "restart file gamma differs from the solver's");
    for (int64_t e = 0; e < ne; ++e) {
        int32_t k = 0;
        std::memcpy(&k, b.data() + head + (size_t)e * 4, 4);
        if (k != s->nsp) return fail(s, ZJ_ERR_ARG, "restart file element " + std::to_string(e) + " has a different n_sp");
    }
    const double* U = reinterpret_cast<const double*>(b.data() + head + (size_t)ne * 4);
    std::vector<double> Ua(U, U + s->state_n);     // aligned copy
    zj_status st = zj_set_state(s, Ua.data());
    if (st != ZJ_OK) return st;
    s->time = time;      // resume
    s->iter = iter;
    return ZJ_OK;
}

zj_status zj_gmsh_read(const char* msh_path, zj_gmsh_mesh** out) {
    if (!out) return fail(nullptr, ZJ_ERR_ARG, "out is NULL");
    *out = nullptr;
    if (!msh_path) return fail(nullptr, ZJ_ERR_ARG, "path is NULL");
    zj_gmsh_mesh* m = new zj_gmsh_mesh();
    std::string err;
    if (!read_gmsh(msh_path, m->g, err)) {
        delete m;
        const bool io = err.rfind("Failed to open", 0) == 0;
        return fail(nullptr, io ? ZJ_ERR_IO : ZJ_ERR_ARG, err);
    }
    m->desc.n_nodes = (int64_t)(m->g.xy.size() / 2);
    m->desc.xy = m->g.xy.data();
    m->desc.n_elem = (int64_t)m->g.etype.size();
    m->desc.elem_type = m->g.etype.data();
    m->desc.elem_order = m->g.eorder.data();
    m->desc.conn_offsets = m->g.offs.data();
    m->desc.conn = m->g.conn.data();
    m->desc.n_bnd_edges = (int64_t)(m->g.bnd.size() / 3);
    m->desc.bnd_edges = m->g.bnd.data();
    *out = m;
    return ZJ_OK;
}

void zj_gmsh_free(zj_gmsh_mesh* m) { delete m; }

const zj_mesh_desc* zj_gmsh_desc(const zj_gmsh_mesh* m) { return m ? &m->desc : nullptr; }

int zj_gmsh_num_groups(const zj_gmsh_mesh* m) { return m ? (int)m->g.groups.size() : 0; }

zj_status zj_gmsh_group(const zj_gmsh_mesh* m, int i, int* tag, int* bc_type, const char** name) {
    if (!m || i < 0 || i >= (int)m->g.groups.size()) return ZJ_ERR_ARG;
    const GmshGroup& g = m->g.groups[(size_t)i];
    if (tag) *tag = g.tag;
    if (bc_type) *bc_type = g.type;
    if (name) *name = g.name.c_str();
    return ZJ_OK;
}

zj_status zj_solver_create_from_gmsh(const char* msh_path, const zj_params* params, zj_solver** out) {
    if (out) *out = nullptr;
    if (!out || !params) return fail(nullptr, ZJ_ERR_ARG, "params or out is NULL");
    zj_gmsh_mesh* m = nullptr;
    zj_status st = zj_gmsh_read(msh_path, &m);
    if (st != ZJ_OK) return st;
    zj_params p = *params;
    for (const GmshGroup& g : m->g.groups) {
        bool named = false;
        for (int k = 0; k < p.n_bc; ++k) named = named || p.bc[k].tag == g.tag;
        if (named) continue;
        if (p.n_bc >= ZJ_MAX_BC) { zj_gmsh_free(m); return fail(nullptr, ZJ_ERR_ARG, "too many boundary groups"); }
        zj_bc_spec& b = p.bc[p.n_bc++];
        b = zj_bc_spec{};
        b.tag = g.tag;
        b.type = g.type;
        b.dir_x = 1.0;
        b.dir_y = 0.0;
    }
    st = zj_solver_create(&m->desc, &p, out);
    zj_gmsh_free(m);
    return st;
}

}  // extern "C"

// ------------------------------------------------------- mesh partitions --
// A partitioned mesh runs as one handle per part (zj_solver_create_part);
// the parts couple only through the traces and gradient traces at the faces
// their partition cuts.  Each part's interface faces read the other side's
// trace rows from ghost rows, which an exchange fills after every launch that
// writes traces: the sender gathers its side's rows into a send buffer in the
// plan's order (neighbours ascending, global face order within each), the
// receiver copies the matching slice of it into its own memory (a peer copy
// across devices, an ordinary copy on one device) and scatters it into its
// ghost rows.  zj_parts_* drive all parts of a partition from one process,
// the parts' streams ordered by events.
namespace {

template <typename T>
__global__ void k_rows_gather(const T* __restrict__ src, const int32_t* __restrict__ rows, long long n, int w,
                              T* __restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * w) return;
    const long long k = i / w, j = i - k * w;
    dst[i] = src[(long long)rows[k] * w + j];
}

template <typename T>
__global__ void k_rows_scatter(const T* __restrict__ src, const int32_t* __restrict__ rows, long long n, int w,
                               T* __restrict__ dst) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n * w) return;
    const long long k = i / w, j = i - k * w;
    dst[(long long)rows[k] * w + j] = src[i];
}

struct DeviceGuard {
    int prev = -1;
    DeviceGuard() { cudaGetDevice(&prev); }
    ~DeviceGuard() { if (prev >= 0) cudaSetDevice(prev); }
};

// The parts of one partition, indexed by rank, checked for consistency.
zj_status parts_check(zj_solver* const* parts, int n, std::vector<zj_solver*>& by_rank) {
    if (!parts || n < 1) return fail(nullptr, ZJ_ERR_ARG, "parts is NULL or empty");
    by_rank.assign((size_t)n, nullptr);
    for (int i = 0; i < n; ++i) {
        zj_solver* s = parts[i];
        if (!s) return fail(nullptr, ZJ_ERR_ARG, "a part handle is NULL");
        if (!s->is_part || s->part.nparts != n)
            return fail(s, ZJ_ERR_ARG, "every handle must be a part of the same n-part partition");
        if (by_rank[(size_t)s->part.rank]) return fail(s, ZJ_ERR_ARG, "two handles hold the same part");
        if (s->mixed != parts[0]->mixed || s->P != parts[0]->P || s->tc != parts[0]->tc)
            return fail(s, ZJ_ERR_ARG, "the parts differ in order or precision");
        by_rank[(size_t)s->part.rank] = s;
    }
    return ZJ_OK;
}

// Rows of width w of every part's buffer bufs[rank] (trace rows: n1*4 values,
// gradient trace rows: n1*8) across the cuts.
template <typename T>
zj_status parts_exchange(const std::vector<zj_solver*>& P, const std::vector<T*>& bufs, int w) {
    const int threads = 256;
    for (zj_solver* s : P) {
        const long long ni = (long long)s->part.mine.size();
        ZJ_CK(s, cudaSetDevice(s->device), "set device");
        if (ni > 0) {
            k_rows_gather<T><<<(unsigned)((ni * w + threads - 1) / threads), threads, 0, s->stream>>>(
                bufs[(size_t)s->part.rank], s->dSendRows, ni, w, static_cast<T*>(s->dSendBuf));
            ZJ_CK(s, cudaGetLastError(), "halo gather");
        }
        ZJ_CK(s, cudaEventRecord(s->ev_pack, s->stream), "halo event");
    }
    for (zj_solver* q : P) {
        const PartSlice& pq = q->part;
        ZJ_CK(q, cudaSetDevice(q->device), "set device");
        for (size_t i = 0; i < pq.nbr.size(); ++i) {
            zj_solver* p = P[(size_t)pq.nbr[i]];
            const PartSlice& pp = p->part;
            size_t j = 0;
            while (j < pp.nbr.size() && pp.nbr[j] != pq.rank) ++j;
            const int64_t cnt = pq.nbr_off[i + 1] - pq.nbr_off[i];
            if (j == pp.nbr.size() || pp.nbr_off[j + 1] - pp.nbr_off[j] != cnt)
                return fail(q, ZJ_ERR_ARG, "the parts' halo plans do not match");
            ZJ_CK(q, cudaStreamWaitEvent(q->stream, p->ev_pack, 0), "halo wait");
            const size_t bytes = (size_t)cnt * w * sizeof(T);
            const T* src = static_cast<const T*>(p->dSendBuf) + (size_t)pp.nbr_off[j] * w;
            T* dst = static_cast<T*>(q->dRecvBuf) + (size_t)pq.nbr_off[i] * w;
            if (p->device == q->device) {
                ZJ_CK(q, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, q->stream), "halo copy");
            } else {
                ZJ_CK(q, cudaMemcpyPeerAsync(dst, q->device, src, p->device, bytes, q->stream), "halo peer copy");
            }
        }
        const long long ni = (long long)pq.mine.size();
        if (ni > 0) {
            k_rows_scatter<T><<<(unsigned)((ni * w + threads - 1) / threads), threads, 0, q->stream>>>(
                static_cast<const T*>(q->dRecvBuf), q->dRecvRows, ni, w, bufs[(size_t)pq.rank]);
            ZJ_CK(q, cudaGetLastError(), "halo scatter");
        }
        ZJ_CK(q, cudaEventRecord(q->ev_done, q->stream), "halo event");
    }
    // a part's send buffer is reused by its next exchange once its
    // neighbours have copied it
    for (zj_solver* p : P) {
        ZJ_CK(p, cudaSetDevice(p->device), "set device");
        for (int32_t r : p->part.nbr) ZJ_CK(p, cudaStreamWaitEvent(p->stream, P[(size_t)r]->ev_done, 0), "halo wait");
    }
    return ZJ_OK;
}

template <typename T>
T* grad_buf(const zj_solver* s);
template <> double* grad_buf<double>(const zj_solver* s) { return s->dTQ; }
template <> float* grad_buf<float>(const zj_solver* s) { return s->fTQ; }

// The stage launch of a part (physics mode, quadrilaterals): the
// Navier-Stokes stage after its gradient traces crossed, else the inviscid
// stage.
template <typename T>
cudaError_t launch_part_stage(zj_solver* s, const StageArgsT<T>& a) {
    if (!is_ns(s)) return launch_phys_stage(s->P, s->prm.riemann, a, s->stream);
    if constexpr (sizeof(T) == 4) {
        if (s->tc) {
            StageArgsT<T> t = a;
            t.tc_err = s->dTcErr;
            return launch_ns_stage_tc(s->P, s->prm.riemann, t, &s->tc_map, s->stream);
        }
    }
    return launch_ns_stage(s->P, s->prm.riemann, a, s->stream);
}

// One residual (stage 0) or SSP-RK3 stage of every part: for Navier-Stokes
// the gradient launches, their gradient traces across the cuts, then the
// stage launches; a stage's new traces cross after it.
template <typename T>
zj_status parts_stage(const std::vector<zj_solver*>& P, const std::vector<StageArgsT<T>>& A) {
    const bool ns = is_ns(P[0]);
    if (ns) {
        std::vector<T*> tq;
        for (size_t i = 0; i < P.size(); ++i) {
            ZJ_CK(P[i], cudaSetDevice(P[i]->device), "set device");
            ZJ_CK(P[i], launch_ns_grad(P[i]->P, A[i], P[i]->stream), "gradient launch");
            tq.push_back(grad_buf<T>(P[i]));
        }
        zj_status st = parts_exchange<T>(P, tq, P[0]->n1 * 8);
        if (st != ZJ_OK) return st;
    }
    std::vector<T*> out;
    for (size_t i = 0; i < P.size(); ++i) {
        zj_solver* s = P[i];
        ZJ_CK(s, cudaSetDevice(s->device), "set device");
        ZJ_CK(s, launch_part_stage<T>(s, A[i]), "stage launch");
        out.push_back(const_cast<T*>(A[i].Tout));
    }
    if (A[0].stage == 0) return ZJ_OK;
    return parts_exchange<T>(P, out, P[0]->n1 * 4);
}

template <typename T>
zj_status parts_traces(const std::vector<zj_solver*>& P, const std::vector<const double*>& U, const std::vector<T*>& Tb) {
    for (size_t i = 0; i < P.size(); ++i) {
        ZJ_CK(P[i], cudaSetDevice(P[i]->device), "set device");
        ZJ_CK(P[i], launch_trace_any(P[i], U[i], Tb[i]), "trace launch");
    }
    return parts_exchange<T>(P, Tb, P[0]->n1 * 4);
}

// One SSP-RK3 step of every part at their common buffer phase (cur, tpar):
// three stages with the exchanges between them; the phase advances.
// Launch arguments of SSP-RK3 stage `stage` of a part at its buffer phase.
template <typename T>
StageArgsT<T> part_stage_args(zj_solver* s, int stage) {
    const int c = s->cur, a1 = (c + 1) % 3, b1 = (c + 2) % 3, p = s->tpar;
    StageArgsT<T> a = stage_args<T>(s);
    a.partials = s->dPart;
    a.U0 = s->dU[c];
    a.stage = stage;
    if (stage == 1) { a.U = s->dU[c]; a.Uout = s->dU[a1]; a.Tin = tbuf<T>(s, p); a.Tout = tbuf<T>(s, 1 - p); }
    if (stage == 2) { a.U = s->dU[a1]; a.Uout = s->dU[b1]; a.Tin = tbuf<T>(s, 1 - p); a.Tout = tbuf<T>(s, p); }
    if (stage == 3) { a.U = s->dU[b1]; a.Uout = s->dU[a1]; a.Tin = tbuf<T>(s, p); a.Tout = tbuf<T>(s, 1 - p); }
    return a;
}

template <typename T>
zj_status parts_enqueue_step(const std::vector<zj_solver*>& P) {
    const size_t n = P.size();
    std::vector<StageArgsT<T>> A(n);
    for (int stage = 1; stage <= 3; ++stage) {
        for (size_t i = 0; i < n; ++i) A[i] = part_stage_args<T>(P[i], stage);
        zj_status st = parts_stage<T>(P, A);
        if (st != ZJ_OK) return st;
    }
    for (zj_solver* s : P) {
        s->cur = (s->cur + 1) % 3;
        s->tpar = 1 - s->tpar;
    }
    return ZJ_OK;
}

// One step of a partition whose parts share a device, as a graph: captured
// on the rank-0 part's stream with the other parts' streams forked from it
// and joined back (their kernels, copies and events keep their order inside
// the graph), one graph per buffer phase, kept on the rank-0 handle.  Parts on
// several devices, a disabled or failed capture, or a stream the caller is
// capturing step with plain launches.
template <typename T>
cudaGraphExec_t parts_step_graph(const std::vector<zj_solver*>& P) {
    zj_solver* s0 = P[0];
    if (!s0->graphs_on || s0->graphs_failed || !s0->stepped) return nullptr;
    for (zj_solver* s : P)
        if (s->device != s0->device || s->stream == nullptr) return nullptr;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    for (zj_solver* s : P)
        if (cudaStreamIsCapturing(s->stream, &cs) != cudaSuccess || cs != cudaStreamCaptureStatusNone) return nullptr;
    const int idx = s0->cur * 2 + s0->tpar;
    if (s0->gexec[idx]) return s0->gexec[idx];
    std::vector<std::pair<int, int>> phase0;
    for (zj_solver* s : P) phase0.push_back({s->cur, s->tpar});
    const std::string err0 = s0->err;
    if (cudaStreamBeginCapture(s0->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        (void)cudaGetLastError();
        s0->graphs_failed = true;
        return nullptr;
    }
    cudaError_t e = cudaEventRecord(s0->ev_join, s0->stream);
    for (size_t i = 1; i < P.size() && e == cudaSuccess; ++i) e = cudaStreamWaitEvent(P[i]->stream, s0->ev_join, 0);
    zj_status st = e == cudaSuccess ? parts_enqueue_step<T>(P) : ZJ_ERR_CUDA;
    // join every forked stream, also after a failure, so the capture closes
    for (size_t i = 1; i < P.size(); ++i) {
        if (cudaEventRecord(P[i]->ev_join, P[i]->stream) == cudaSuccess)
            (void)cudaStreamWaitEvent(s0->stream, P[i]->ev_join, 0);
    }
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(s0->stream, &graph);
    for (size_t i = 0; i < P.size(); ++i) {   // nothing ran: back to the starting phase
        P[i]->cur = phase0[i].first;
        P[i]->tpar = phase0[i].second;
    }
    cudaGraphExec_t exec = nullptr;
    if (st == ZJ_OK && e == cudaSuccess && graph) e = cudaGraphInstantiate(&exec, graph, 0);
    if (graph) cudaGraphDestroy(graph);
    if (st == ZJ_OK && e == cudaSuccess && exec) e = cudaGraphUpload(exec, s0->stream);
    if (st != ZJ_OK || e != cudaSuccess || !exec) {
        (void)cudaGetLastError();
        if (exec) cudaGraphExecDestroy(exec);
        s0->err = err0;
        s0->graphs_failed = true;
        return nullptr;
    }
    s0->gexec[idx] = exec;
    return exec;
}

template <typename T>
zj_status parts_step_t(const std::vector<zj_solver*>& P, double dt, int nsteps) {
    const size_t n = P.size();
    zj_solver* s0 = P[0];
    if (!s0->traces_valid) {
        std::vector<const double*> U(n);
        std::vector<T*> Tb(n);
        for (size_t i = 0; i < n; ++i) { U[i] = P[i]->dU[P[i]->cur]; Tb[i] = tbuf<T>(P[i], P[i]->tpar); }
        zj_status st = parts_traces<T>(P, U, Tb);
        if (st != ZJ_OK) return st;
        for (zj_solver* s : P) s->traces_valid = true;
    }
    const bool first = !s0->stepped;
    for (int step = 0; step < nsteps; ++step) {
        cudaGraphExec_t g = parts_step_graph<T>(P);
        if (g) {
            // the graph runs on the rank-0 stream after every part's queued
            // work; the parts' streams continue after it
            ZJ_CK(s0, cudaSetDevice(s0->device), "set device");
            for (size_t i = 1; i < n; ++i) {
                ZJ_CK(P[i], cudaEventRecord(P[i]->ev_join, P[i]->stream), "join event");
                ZJ_CK(s0, cudaStreamWaitEvent(s0->stream, P[i]->ev_join, 0), "join wait");
            }
            ZJ_CK(s0, cudaGraphLaunch(g, s0->stream), "partition step graph launch");
            ZJ_CK(s0, cudaEventRecord(s0->ev_join, s0->stream), "fork event");
            for (size_t i = 1; i < n; ++i) ZJ_CK(P[i], cudaStreamWaitEvent(P[i]->stream, s0->ev_join, 0), "fork wait");
            for (zj_solver* s : P) {
                s->cur = (s->cur + 1) % 3;
                s->tpar = 1 - s->tpar;
            }
        } else {
            zj_status st = parts_enqueue_step<T>(P);
            if (st != ZJ_OK) return st;
            s0->stepped = true;
        }
        for (zj_solver* s : P) {
            s->time += dt;
            s->iter += 1;
        }
    }
    if (first) {
        // capture (without running) the graphs of all six phases now, so
        // later calls only launch them
        std::vector<std::pair<int, int>> phase0;
        for (zj_solver* s : P) phase0.push_back({s->cur, s->tpar});
        for (int c = 0; c < 3 && !s0->graphs_failed; ++c)
            for (int p = 0; p < 2 && !s0->graphs_failed; ++p) {
                for (zj_solver* s : P) { s->cur = c; s->tpar = p; }
                (void)parts_step_graph<T>(P);
            }
        for (size_t i = 0; i < n; ++i) {
            P[i]->cur = phase0[i].first;
            P[i]->tpar = phase0[i].second;
        }
    }
    for (zj_solver* s : P) s->has_norm = true;
    return ZJ_OK;
}

// ---- one process per GPU: a part stepped alone; at each exchange its
// cut-face rows go to the caller's transport and come back as ghost rows

template <typename T>
zj_status part_exchange_cb(zj_solver* s, T* buf, int w, int kind, zj_exchange_fn fn, void* user) {
    const int threads = 256;
    const long long ni = (long long)s->part.mine.size();
    if (ni > 0) {
        k_rows_gather<T><<<(unsigned)((ni * w + threads - 1) / threads), threads, 0, s->stream>>>(
            buf, s->dSendRows, ni, w, static_cast<T*>(s->dSendBuf));
        ZJ_CK(s, cudaGetLastError(), "halo gather");
    }
    const int rc = fn(user, kind, (int)(w * sizeof(T)), s->dSendBuf, s->dRecvBuf, static_cast<void*>(s->stream));
    if (rc != 0) return fail(s, ZJ_ERR_IO, "the exchange callback returned " + std::to_string(rc));
    if (ni > 0) {
        k_rows_scatter<T><<<(unsigned)((ni * w + threads - 1) / threads), threads, 0, s->stream>>>(
            static_cast<const T*>(s->dRecvBuf), s->dRecvRows, ni, w, buf);
        ZJ_CK(s, cudaGetLastError(), "halo scatter");
    }
    return ZJ_OK;
}

template <typename T>
zj_status part_step_t(zj_solver* s, int nsteps, zj_exchange_fn fn, void* user, double dt) {
    zj_status st = ZJ_OK;
    if (!s->traces_valid) {
        T* tb = tbuf<T>(s, s->tpar);
        ZJ_CK(s, launch_trace_any(s, s->dU[s->cur], tb), "trace launch");
        if ((st = part_exchange_cb<T>(s, tb, s->n1 * 4, ZJ_XCHG_TRACES, fn, user)) != ZJ_OK) return st;
        s->traces_valid = true;
    }
    for (int step = 0; step < nsteps; ++step) {
        for (int stage = 1; stage <= 3; ++stage) {
            const StageArgsT<T> a = part_stage_args<T>(s, stage);
            if (is_ns(s)) {
                ZJ_CK(s, launch_ns_grad(s->P, a, s->stream), "gradient launch");
                if ((st = part_exchange_cb<T>(s, grad_buf<T>(s), s->n1 * 8, ZJ_XCHG_GRADIENTS, fn, user)) != ZJ_OK)
                    return st;
            }
            ZJ_CK(s, launch_part_stage<T>(s, a), "stage launch");
            if ((st = part_exchange_cb<T>(s, const_cast<T*>(a.Tout), s->n1 * 4, ZJ_XCHG_TRACES, fn, user)) != ZJ_OK)
                return st;
        }
        s->cur = (s->cur + 1) % 3;
        s->tpar = 1 - s->tpar;
        s->time += dt;
        s->iter += 1;
    }
    s->has_norm = true;
    return ZJ_OK;
}

template <typename T>
zj_status parts_rhs_t(const std::vector<zj_solver*>& P, const double* const* Ud, double* const* Rd) {
    const size_t n = P.size();
    std::vector<const double*> U(n);
    std::vector<T*> Tb(n);
    for (size_t i = 0; i < n; ++i) {
        const size_t r = (size_t)P[i]->part.rank;
        U[i] = Ud[r];
        Tb[i] = tbuf<T>(P[i], 2);
    }
    zj_status st = parts_traces<T>(P, U, Tb);
    if (st != ZJ_OK) return st;
    std::vector<StageArgsT<T>> A(n);
    for (size_t i = 0; i < n; ++i) {
        StageArgsT<T> a = stage_args<T>(P[i]);
        a.U = U[i]; a.U0 = U[i]; a.Uout = nullptr; a.Tin = Tb[i]; a.Tout = nullptr;
        a.R = Rd[(size_t)P[i]->part.rank]; a.partials = P[i]->dPartR; a.stage = 0;
        A[i] = a;
    }
    return parts_stage<T>(P, A);
}

}  // namespace

extern "C" {

zj_status zj_partition(const zj_mesh_desc* mesh, int nparts, int32_t* part) {
    if (!mesh || !part || nparts < 1) return fail(nullptr, ZJ_ERR_ARG, "mesh or part is NULL, or nparts < 1");
    HostMesh m;
    std::string msg;
    if (!build_mesh(mesh, nullptr, m, msg)) return fail(nullptr, ZJ_ERR_ARG, msg);
    if (m.n_elem < nparts) return fail(nullptr, ZJ_ERR_ARG, "fewer elements than parts");
    std::vector<int32_t> p;
    partition_rcb(m, nparts, p);
    std::memcpy(part, p.data(), p.size() * sizeof(int32_t));
    return ZJ_OK;
}

zj_status zj_halo_plan_size(const zj_mesh_desc* mesh, const int32_t* part, int nparts, int rank, int* n_nbr,
                            int64_t* n_iface, int64_t* n_elem) {
    if (!mesh || !part || !n_nbr || !n_iface) return fail(nullptr, ZJ_ERR_ARG, "NULL argument");
    HostMesh m;
    PartSlice ps;
    std::string msg;
    if (!build_mesh(mesh, nullptr, m, msg) || !make_part_slice(m, part, nparts, rank, ps, msg))
        return fail(nullptr, ZJ_ERR_ARG, msg);
    *n_nbr = (int)ps.nbr.size();
    *n_iface = (int64_t)ps.mine.size();
    if (n_elem) *n_elem = (int64_t)ps.elems.size();
    return ZJ_OK;
}

zj_status zj_halo_plan(const zj_mesh_desc* mesh, const int32_t* part, int nparts, int rank, int32_t* nbr,
                       int64_t* nbr_off, int64_t* face, int64_t* mine, int64_t* remote, int64_t* elems) {
    if (!mesh || !part || !nbr || !nbr_off || !face || !mine || !remote) return fail(nullptr, ZJ_ERR_ARG, "NULL argument");
    HostMesh m;
    PartSlice ps;
    std::string msg;
    if (!build_mesh(mesh, nullptr, m, msg) || !make_part_slice(m, part, nparts, rank, ps, msg))
        return fail(nullptr, ZJ_ERR_ARG, msg);
    std::copy(ps.nbr.begin(), ps.nbr.end(), nbr);
    std::copy(ps.nbr_off.begin(), ps.nbr_off.end(), nbr_off);
    std::copy(ps.face.begin(), ps.face.end(), face);
    std::copy(ps.mine.begin(), ps.mine.end(), mine);
    std::copy(ps.remote.begin(), ps.remote.end(), remote);
    if (elems) std::copy(ps.elems.begin(), ps.elems.end(), elems);
    return ZJ_OK;
}

zj_status zj_solver_create_part(const zj_mesh_desc* mesh, const zj_params* params, const int32_t* part,
                                int nparts, int rank, zj_solver** out) {
    if (!part) return fail(nullptr, ZJ_ERR_ARG, "part is NULL");
    return create_impl(mesh, params, part, nparts, rank, out);
}

zj_status zj_part_elements(const zj_solver* s, int64_t* global_ids) {
    if (!s || !global_ids) return ZJ_ERR_ARG;
    if (!s->is_part) {
        for (int64_t e = 0; e < s->E; ++e) global_ids[e] = e;
        return ZJ_OK;
    }
    std::copy(s->part.elems.begin(), s->part.elems.end(), global_ids);
    return ZJ_OK;
}

zj_status zj_parts_step(zj_solver* const* parts, int n, double dt, int nsteps) {
    std::vector<zj_solver*> P;
    zj_status st = parts_check(parts, n, P);
    if (st != ZJ_OK) return st;
    if (nsteps < 0 || !std::isfinite(dt)) return fail(P[0], ZJ_ERR_ARG, "bad dt or nsteps");
    if (nsteps == 0) return ZJ_OK;
    DeviceGuard guard;
    for (zj_solver* s : P) {
        ZJ_CK(s, cudaSetDevice(s->device), "set device");
        if (dt != s->last_dt) {
            k_set_dt<<<1, 1, 0, s->stream>>>(s->dScal, dt);
            ZJ_CK(s, cudaGetLastError(), "dt launch");
            s->last_dt = dt;
        }
    }
    return P[0]->mixed ? parts_step_t<float>(P, dt, nsteps) : parts_step_t<double>(P, dt, nsteps);
}

zj_status zj_part_step(zj_solver* s, double dt, int nsteps, zj_exchange_fn exchange, void* user) {
    if (!s) return ZJ_ERR_ARG;
    if (!s->is_part) return fail(s, ZJ_ERR_ARG, "zj_part_step steps a part of a partitioned mesh");
    if (!exchange) return fail(s, ZJ_ERR_ARG, "exchange is NULL");
    if (nsteps < 0 || !std::isfinite(dt)) return fail(s, ZJ_ERR_ARG, "bad dt or nsteps");
    if (nsteps == 0) return ZJ_OK;
    DeviceGuard guard;
    ZJ_CK(s, cudaSetDevice(s->device), "set device");
    if (dt != s->last_dt) {
        k_set_dt<<<1, 1, 0, s->stream>>>(s->dScal, dt);
        ZJ_CK(s, cudaGetLastError(), "dt launch");
        s->last_dt = dt;
    }
    return s->mixed ? part_step_t<float>(s, nsteps, exchange, user, dt) : part_step_t<double>(s, nsteps, exchange, user, dt);
}

zj_status zj_parts_rhs(zj_solver* const* parts, int n, const double* const* U_dev, double* const* R_dev) {
    std::vector<zj_solver*> P;
    zj_status st = parts_check(parts, n, P);
    if (st != ZJ_OK) return st;
    if (!U_dev || !R_dev) return fail(P[0], ZJ_ERR_ARG, "U_dev or R_dev is NULL");
    for (int i = 0; i < n; ++i)
        if (!U_dev[i] || !R_dev[i] || misaligned(U_dev[i]) || misaligned(R_dev[i]))
            return fail(P[0], ZJ_ERR_ARG, "U_dev and R_dev must be non-NULL, 32-byte aligned device arrays");
    DeviceGuard guard;
    return P[0]->mixed ? parts_rhs_t<float>(P, U_dev, R_dev) : parts_rhs_t<double>(P, U_dev, R_dev);
}

zj_status zj_parts_synchronize(zj_solver* const* parts, int n) {
    std::vector<zj_solver*> P;
    zj_status st = parts_check(parts, n, P);
    if (st != ZJ_OK) return st;
    DeviceGuard guard;
    for (zj_solver* s : P) {
        ZJ_CK(s, cudaSetDevice(s->device), "set device");
        ZJ_CK(s, cudaStreamSynchronize(s->stream), "synchronize");
    }
    return ZJ_OK;
}

zj_status zj_parts_residual_norm(zj_solver* const* parts, int n, double* out) {
    std::vector<zj_solver*> P;
    zj_status st = parts_check(parts, n, P);
    if (st != ZJ_OK) return st;
    if (!out) return fail(P[0], ZJ_ERR_ARG, "out is NULL");
    DeviceGuard guard;
    double sum = 0.0;
    for (zj_solver* s : P) {
        ZJ_CK(s, cudaSetDevice(s->device), "set device");
        if (!s->has_norm) continue;
        ZJ_CK(s, launch_reduce_sum(s->dPart, s->grid, s->dScal + 1, s->stream), "norm reduce");
        double v = 0.0;
        ZJ_CK(s, cudaMemcpyAsync(&v, s->dScal + 1, sizeof(double), cudaMemcpyDeviceToHost, s->stream), "norm copy");
        ZJ_CK(s, cudaStreamSynchronize(s->stream), "norm sync");
        sum += v;
    }
    *out = std::sqrt(sum);
    return ZJ_OK;
}

}  // extern "C"
