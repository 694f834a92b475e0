/*
 * zj_fr.h -- C-ABI of the B200-native Flux-Reconstruction hot path.
 *
 * One handle (zj_solver) replaces one reference zhijian::FRSolver
 * (include/solver/fr_solver.hpp:77-180 in the Zhijian project).  Plain
 * pointers and sizes only; no C++ or torch types cross this boundary.
 * Every call returns a zj_status and never exits the process; the text of the
 * last error is available from zj_last_error().
 *
 * State layout on both sides of the boundary is the reference's AoS layout
 * [element][solution point][variable], variables (rho, rho*u, rho*v, rho*E),
 * solution point sp = j*(P+1) + i with i the xi index and j the eta index
 * (src/basis/basis.cpp:479-487).
 */
#ifndef ZJ_FR_H
#define ZJ_FR_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ZJ_ABI_VERSION 1

/* Error codes.  The reference aborts through CUDA_CHECK -> std::exit
 * (include/common/cuda_utils.hpp:13-21); here every failure is returned. */
typedef enum zj_status {
    ZJ_OK = 0,
    ZJ_ERR_ARG = 1,          /* bad argument, size or mesh */
    ZJ_ERR_CUDA = 2,         /* CUDA runtime error */
    ZJ_ERR_NAN = 3,          /* non-finite value detected in the state */
    ZJ_ERR_TIMEOUT = 4,      /* a bounded device wait gave up */
    ZJ_ERR_UNSUPPORTED = 5,  /* valid request this build does not implement */
    ZJ_ERR_IO = 6            /* file could not be read or parsed */
} zj_status;

/* Boundary types, numbered as the reference BCType (include/common/types.hpp:47-56). */
typedef enum zj_bc_type {
    ZJ_BC_INTERIOR = 0, ZJ_BC_WALL = 1, ZJ_BC_SLIPWALL = 2, ZJ_BC_SYMMETRY = 3,
    ZJ_BC_FARFIELD = 4, ZJ_BC_INFLOW = 5, ZJ_BC_OUTFLOW = 6, ZJ_BC_PERIODIC = 7
} zj_bc_type;

/* FR correction family (types.hpp:59-64) and Riemann solver (types.hpp:67-71). */
typedef enum zj_flux_type { ZJ_FLUX_DG = 0, ZJ_FLUX_SD = 1, ZJ_FLUX_HU = 2, ZJ_FLUX_GA = 3 } zj_flux_type;
typedef enum zj_riemann { ZJ_RIEMANN_RUSANOV = 0, ZJ_RIEMANN_ROE = 1, ZJ_RIEMANN_HLLC = 2 } zj_riemann;

/* Arithmetic of the residual.  ZJ_FP64: FP64 end to end.  ZJ_MIXED: FP32
 * volume and face work, FP64 stage accumulation, reductions and metrics.
 * ZJ_SPLIT_BF16: the mixed form whose Navier-Stokes stage at P4/P5 on quad
 * meshes takes its dense operator product (divergence and edge flux traces)
 * on the tensor cores as three BF16 products accumulated in FP32; elsewhere
 * (P1-P3, Euler, meshes with triangles) it is the mixed form. */
typedef enum zj_precision { ZJ_FP64 = 0, ZJ_MIXED = 1, ZJ_SPLIT_BF16 = 2 } zj_precision;

/* Element kinds of the mesh descriptor (types.hpp:41-44). */
typedef enum zj_elem_type { ZJ_ELEM_TRI = 0, ZJ_ELEM_QUAD = 1 } zj_elem_type;

#define ZJ_MAX_BC 32

/* One "bc <tag> <type> [key value ...]" config line (src/main.cpp:132-166). */
typedef struct zj_bc_spec {
    int tag;
    int type;          /* zj_bc_type */
    double p_static;   /* outflow; 0 = p_inf */
    double p_total;    /* inflow; 0 = 1.2 p_inf */
    double T_total;    /* inflow; 0 = T_inf */
    double T_wall;     /* isothermal wall; 0 = adiabatic */
    double dir_x, dir_y;
} zj_bc_spec;

/* Solver parameters: the fields of the reference SimParams
 * (include/common/types.hpp:130-172) plus the two selectors of this build.
 * zj_params_default() gives the reference defaults. */
typedef struct zj_params {
    double gamma, Pr, Re, Mach, T_inf, p_inf, rho_inf, AoA;
    int poly_order;
    int flux_type;     /* zj_flux_type */
    int riemann;       /* zj_riemann */
    double CFL, dt, t_final;
    int max_iter;
    int viscous;
    int output_freq, restart_freq;
    char case_name[64];
    /* compat = 1: reproduce the reference residual exactly, quirks included
     * (hard-coded Rusanov, inviscid, Radau correction, no metric scaling of
     * the correction, dimensional clamps).  compat = 0: the conservative FR
     * scheme the parameters ask for (physics mode). */
    int compat;
    int precision;     /* zj_precision */
    int n_bc;
    zj_bc_spec bc[ZJ_MAX_BC];
} zj_params;

/* Mesh descriptor: borrowed for the duration of zj_solver_create only.
 * Element e has nodes conn[conn_offsets[e] .. conn_offsets[e+1]), vertices
 * first and counter-clockwise (Q1: 4 nodes, Q2: 9, Q4: 25; gmsh ordering as
 * src/basis/basis.cpp:706-770).  bnd_edges[3*k .. 3*k+2] = (v0, v1, tag);
 * the bc table of zj_params maps tags to boundary types.  Untagged boundary
 * edges are far-field (src/mesh/mesh.cpp:48-57). */
typedef struct zj_mesh_desc {
    int64_t n_nodes;
    const double* xy;            /* [n_nodes][2] */
    int64_t n_elem;
    const int32_t* elem_type;    /* [n_elem] zj_elem_type */
    const int32_t* elem_order;   /* [n_elem] 1, 2 or 4 */
    const int64_t* conn_offsets; /* [n_elem + 1] */
    const int64_t* conn;
    int64_t n_bnd_edges;
    const int64_t* bnd_edges;    /* [n_bnd_edges][3] */
} zj_mesh_desc;

typedef struct zj_solver zj_solver;

/* ---- parameters and configuration (src/main.cpp:78-170) ----------------- */
void zj_params_default(zj_params* p);
/* Parse a config file with the reference grammar: "key value" lines, '#'
 * comments, unknown keys ignored; adds keys "compat on|off" and
 * "precision fp64|mixed|split_bf16". */
zj_status zj_params_parse_file(const char* path, zj_params* p);
zj_status zj_params_parse_string(const char* text, zj_params* p);

/* ---- lifetime (FRSolver::initialize, fr_solver.cpp:30-73) -------------- */
/* Builds faces, normals, metrics and operators on the host, allocates every
 * device buffer once and uploads; later calls allocate nothing. */
zj_status zj_solver_create(const zj_mesh_desc* mesh, const zj_params* params,
                           zj_solver** out);
void zj_solver_destroy(zj_solver* s);
/* Last error text of this handle, or of the last failed create when s is NULL. */
const char* zj_last_error(const zj_solver* s);
int zj_abi_version(void);

/* ---- sizes ---------------------------------------------------------------- */
int64_t zj_num_elements(const zj_solver* s);
int zj_num_solution_points(const zj_solver* s);      /* per element */
int64_t zj_num_faces(const zj_solver* s);
int64_t zj_state_size(const zj_solver* s);            /* E * n_sp * 4 */

/* ---- initial condition (FRSolver::setInitialCondition, fr_solver.cpp:268-299)
 * A C ABI cannot carry std::function: fetch the physical coordinates of the
 * solution points, evaluate the initial state on the host, then set it. */
/* Meshes with triangles (physics mode): every element has (P+1)^2 state slots;
 * a triangle uses the first (P+1)(P+2)/2 of them (the reference's collapsed
 * Gauss-Legendre points, SolutionPoints::getTriangle, basis.cpp:391-416) and
 * its other slots are neither read nor written.  kinds[e] = zj_elem_type. */
zj_status zj_element_kinds(const zj_solver* s, int32_t* kinds);
int zj_num_triangle_points(const zj_solver* s);
zj_status zj_solution_point_coords(const zj_solver* s, double* xy /* [E][n_sp][2] */);
/* copyToDevice / copyToHost (fr_solver.cpp:835-871), host buffers.  Setting
 * the state resets time and iteration like setInitialCondition. */
zj_status zj_set_state(zj_solver* s, const double* U_host);
zj_status zj_get_state(zj_solver* s, double* U_host);
/* Same with device buffers (no host copy). */
zj_status zj_set_state_device(zj_solver* s, const double* U_dev);
zj_status zj_get_state_device(zj_solver* s, double* U_dev);
/* Host copies queued on the handle's stream without waiting (no reference
 * counterpart: copyToDevice/copyToHost block).  The host buffer must stay
 * valid, and unchanged for a set, until zj_synchronize; page-locked buffers
 * (cudaHostAlloc / cudaHostRegister) let the copy run on a copy engine while
 * other streams compute, so a caller streaming independent states through two
 * handles on two streams overlaps one handle's copies with the other's steps.
 * Setting the state resets time and iteration like zj_set_state. */
zj_status zj_set_state_async(zj_solver* s, const double* U_host);
zj_status zj_get_state_async(zj_solver* s, double* U_host);

/* ---- the hot path ---------------------------------------------------------- */
/* nsteps SSP-RK3 steps of size dt (FRSolver::advance, fr_solver.cpp:305-333),
 * queued on the handle's stream; returns once the steps are enqueued and
 * checked for launch errors.  zj_synchronize waits for them.  dt reaches the
 * device as a kernel argument, so zj_step may be captured into a caller's
 * graph with any dt (each replay sets it). */
zj_status zj_step(zj_solver* s, double dt, int nsteps);
/* Step graphs (no reference counterpart): zj_step replays blocks of six steps
 * from CUDA graphs (one graph per phase of the rotating stage and trace
 * buffers, six per handle), so a long zj_step costs one launch per six steps
 * instead of six to twelve.  The handle's first zj_step runs its steps with
 * plain launches and then captures and uploads all six graphs, so later calls
 * only launch them; remainders, the legacy default stream and a stream the
 * caller is capturing launch kernels directly, with identical results.
 * enable = 0 turns the graphs off for this handle. */
zj_status zj_set_step_graphs(zj_solver* s, int enable);
zj_status zj_synchronize(zj_solver* s);
/* One residual R = dU/dt on device buffers of E*n_sp*4 doubles, 32-byte
 * aligned (ZJ_ERR_ARG otherwise), on the handle's stream
 * (computeResidual_GPU, fr_solver.cpp:335-608).  Borrowed. */
zj_status zj_rhs(zj_solver* s, const double* U_dev, double* R_dev);
/* Same through host buffers: H2D, residual, D2H, synchronised. */
zj_status zj_rhs_host(zj_solver* s, const double* U_host, double* R_host);
/* L2 norm of the residual of the last stage of the last step
 * (FRSolver::computeResidual, fr_solver.cpp:818-833), reduced on the device. */
zj_status zj_residual_norm(zj_solver* s, double* out);
/* CFL time step over the current device state (FRSolver::computeTimeStep,
 * fr_solver.cpp:784-816; the reference evaluates it on a stale host copy). */
zj_status zj_compute_dt(zj_solver* s, double* dt_out);
/* Non-finite check of the current state: ZJ_ERR_NAN if any value is NaN/Inf
 * (replaces the reference's host-side checkNaN, fr_solver.cpp:11-22). */
zj_status zj_check_state(zj_solver* s);
double zj_time(const zj_solver* s);
int zj_iteration(const zj_solver* s);

/* Stream: the handle creates its own non-blocking stream and uses it until a
 * caller stream is set; NULL selects the CUDA legacy default stream.  To go
 * back to the handle's own stream pass the value zj_get_stream returned before
 * the first zj_set_stream.  cudaStream_t passed as void*. */
zj_status zj_set_stream(zj_solver* s, void* stream);
void* zj_get_stream(const zj_solver* s);

/* ---- allocation-free residual ------------------------------------------------
 * No counterpart in the reference.  The same residual as zj_rhs for callers
 * that may not allocate device memory when they need it (a host application
 * whose device memory is reserved up front by its own allocator, a
 * time-critical loop that must not hit cudaMalloc's implicit synchronisation).
 * Its per-call scratch lives in one file-scope device array of
 * ZJ_NOALLOC_SCRATCH_BYTES inside the library, which every GPU that loads the
 * library holds until the process exits; the call makes no cudaMalloc,
 * cudaFree or other allocating call.  Scratch bytes of a handle, with
 * n_t = (4 E + B) (P+1) 4 trace values (E elements, B boundary edges in
 * physics mode, 0 in compat mode), w = 8 (FP64) or 4 (precision mixed) and
 * G = the residual's CTA count (E/16 at P3, quads):
 *     k n_t w + 8 G,   k = 3 for Navier-Stokes (traces and the two gradient
 *                      trace components), 1 otherwise.
 * At P3 that admits about 65 000 elements in FP64 Euler or compat, 21 000 in
 * FP64 Navier-Stokes and 43 000 in the mixed form's Navier-Stokes; a larger
 * mesh is rejected with ZJ_ERR_ARG and a message giving the bytes it needs.
 * Call it with the device current on which the handle was created
 * (ZJ_ERR_ARG otherwise).  The first call on a device looks up the array's
 * device address (once per device, with that device current) and keeps it for
 * the life of the process: make that first call before any stream capture, and
 * do not use the library across a cudaDeviceReset of the device.  All calls
 * share the one array: calls that overlap on the GPU (other streams, other
 * handles, other host threads) race on it.  Inputs and outputs are the
 * caller's device buffers, 32-byte aligned, on the handle's stream. */
#define ZJ_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)
zj_status zj_rhs_noalloc(zj_solver* s, const double* U_dev, double* R_dev);

/* ---- mesh partitions (several GPUs) ----------------------------------------
 * Replace MeshPartitioner::partition (src/mesh/partitioner.cpp:10-93, METIS
 * k-way on the element dual graph) and MPICommunicator::exchangeHalo
 * (src/parallel/mpi_comm.cpp:68-171).  A partitioned mesh runs as one handle
 * per part; the parts couple only through the traces and gradient traces at
 * the faces the partition cuts, which cross after every launch that writes
 * them: the sender gathers its side's trace rows, the receiver copies them
 * into its own memory (a peer copy between devices) and scatters them into
 * the ghost rows its interface faces read.  Physics mode, quadrilateral
 * meshes (straight or curved), FP64, mixed or split_bf16; the result equals
 * the whole mesh's residual.
 *
 * zj_partition: recursive coordinate bisection of the element centroids into
 * nparts parts whose sizes differ by at most one element (deterministic);
 * part[E].  Host only. */
zj_status zj_partition(const zj_mesh_desc* mesh, int nparts, int32_t* part);
/* The halo plan of part `rank` (host only): n_nbr neighbouring parts nbr[]
 * (ascending) with their interfaces [nbr_off[i], nbr_off[i+1]) in the global
 * face order (the order both sides of a cut agree on); per interface the
 * global face id, this part's side and the other side as global
 * element*4 + local edge; elems (may be NULL) the part's global element ids,
 * ascending.  Sizes from zj_halo_plan_size (n_elem may be NULL). */
zj_status zj_halo_plan_size(const zj_mesh_desc* mesh, const int32_t* part, int nparts, int rank, int* n_nbr,
                            int64_t* n_iface, int64_t* n_elem);
zj_status zj_halo_plan(const zj_mesh_desc* mesh, const int32_t* part, int nparts, int rank, int32_t* nbr,
                       int64_t* nbr_off, int64_t* face, int64_t* mine, int64_t* remote, int64_t* elems);
/* The handle of part `rank`, on the device current at the call: its state is
 * [E_part][n_sp][4] over its elements in ascending global order
 * (zj_part_elements), set and read with zj_set_state / zj_get_state as
 * usual.  zj_step and zj_rhs refuse a part (ZJ_ERR_UNSUPPORTED): the parts
 * of a partition step together. */
zj_status zj_solver_create_part(const zj_mesh_desc* mesh, const zj_params* params, const int32_t* part,
                                int nparts, int rank, zj_solver** out);
zj_status zj_part_elements(const zj_solver* s, int64_t* global_ids);
/* All n parts of one partition from one process (any order; each on its own
 * device and stream, ordered by events): nsteps SSP-RK3 steps, one residual
 * of the device states U_dev[rank] into R_dev[rank] (32-byte aligned),
 * synchronisation, and the L2 norm of the last stage's residual over all
 * parts.  When every part is on one device, zj_parts_step replays one CUDA
 * graph per step after its first call (captured on the rank-0 part's stream
 * with the others forked from it); zj_set_step_graphs(rank-0 part, 0) turns
 * that off. */
zj_status zj_parts_step(zj_solver* const* parts, int n, double dt, int nsteps);
zj_status zj_parts_rhs(zj_solver* const* parts, int n, const double* const* U_dev, double* const* R_dev);
zj_status zj_parts_synchronize(zj_solver* const* parts, int n);
zj_status zj_parts_residual_norm(zj_solver* const* parts, int n, double* out);
/* One process per GPU (the caller's MPI or NCCL moves the rows; the
 * reference's MPICommunicator::exchangeHalo, mpi_comm.cpp:68-171): nsteps
 * SSP-RK3 steps of the part s alone, on its stream.  At each exchange (the
 * state traces before the first step, then per stage the gradient traces
 * after the gradient launch (Navier-Stokes) and the new traces after the
 * stage launch) the part's cut-face rows are gathered into send_dev, in the
 * halo plan's order (zj_halo_plan: rows [nbr_off[i], nbr_off[i+1]) for
 * neighbour nbr[i]; row_bytes bytes each), and exchange(user, kind,
 * row_bytes, send_dev, recv_dev, stream) is called on this host thread.  It
 * must fill recv_dev, in the same layout, with the rows every neighbour sent
 * for this part: complete when it returns, or ordered before work enqueued on
 * `stream` after it (NCCL sends and receives on that stream).  send_dev is
 * written by work queued on `stream` before the call.  Nonzero from exchange
 * stops the step with ZJ_ERR_IO.  The parts' residual norms combine as
 * sqrt(sum of zj_residual_norm(part)^2), their time steps as the minimum of
 * zj_compute_dt over the parts; every part must call zj_part_step with the same
 * dt and nsteps. */
enum { ZJ_XCHG_TRACES = 1, ZJ_XCHG_GRADIENTS = 2 };
typedef int (*zj_exchange_fn)(void* user, int kind, int row_bytes, const void* send_dev, void* recv_dev,
                              void* stream);
zj_status zj_part_step(zj_solver* s, double dt, int nsteps, zj_exchange_fn exchange, void* user);

/* ---- differentiation (physics mode, FP64) ----------------------------------
 * No reference counterpart: the reference has no adjoint.  All pointers are
 * device pointers to [E][n_sp][4] FP64 arrays, 32-byte aligned; the calls are
 * asynchronous on the handle's stream.  Compat mode and the mixed-precision
 * form return ZJ_ERR_UNSUPPORTED. */

/* Jacobian-vector product: R_dev = R(U), JV_dev = dR/dU . V + dR/dRe * dRe
 * (forward mode on dual numbers; exact to FP64 rounding).  R_dev may be NULL. */
zj_status zj_rhs_jvp(zj_solver* s, const double* U_dev, const double* V_dev, double dRe,
                     double* R_dev, double* JV_dev);

/* Vector-Jacobian product: W_dev = (dR/dU)^T L_dev (hand-written transposed
 * kernels).  If dRe_out is not NULL it receives L . dR/dRe (one extra dual
 * launch). */
zj_status zj_rhs_vjp(zj_solver* s, const double* U_dev, const double* L_dev, double* W_dev,
                     double* dRe_out);

/* Adjoint of one SSP-RK3 step of size dt taken from U_dev: given B_dev =
 * dJ/dU(n+1), writes dJ/dU(n) into A_dev (may alias B_dev) and adds
 * dJ/dRe contributions into *dRe_acc if it is not NULL.  The stage states
 * are recomputed from U_dev. */
zj_status zj_step_vjp(zj_solver* s, const double* U_dev, double dt, const double* B_dev,
                      double* A_dev, double* dRe_acc);

/* Discrete adjoint of nsteps SSP-RK3 steps of size dt from the handle's
 * current state (which is left unchanged): checkpoints every k_ckpt steps
 * on the device, segment recomputation, step adjoints backwards.
 * G_dev holds dJ/dU(final) on entry and dJ/dU(initial) on return.  Optional
 * outputs: *dRe = dJ/dRe, *bytes = device bytes the checkpoints and segment
 * states took, *ms_forward / *ms_adjoint = device times of the checkpointed
 * forward sweep and of the backward sweep (CUDA events). */
zj_status zj_adjoint_run(zj_solver* s, double dt, int nsteps, int k_ckpt, double* G_dev,
                         double* dRe, int64_t* bytes, double* ms_forward, double* ms_adjoint);

/* ---- restart files ------------------------------------------------------------
 * The fields of RestartIO (src/io/restart.cpp:8-144) -- attributes time,
 * iteration, poly_order, gamma; datasets elem_n_sp [E] and solution
 * [E][n_sp][4] f64 -- in a dependency-free little-endian binary file:
 *   "ZJRESTRT" u32 version=1 u32 reserved=0 f64 time i32 iteration
 *   i32 poly_order f64 gamma i64 n_elem i32 elem_n_sp[n_elem]
 *   f64 solution[sum n_sp * 4] u64 FNV-1a-64 of every preceding byte.
 * zj_restart_write stores the handle's current state, time and iteration
 * (synchronises); zj_restart_read checks the file against the handle (magic,
 * version, checksum, n_elem, n_sp, poly_order, gamma), loads the state and
 * resumes time and iteration, which the reference's reader leaves unused
 * (src/main.cpp:349-360).  ZJ_ERR_IO: cannot open/short file; ZJ_ERR_ARG:
 * mismatch or corrupt file. */
zj_status zj_restart_write(zj_solver* s, const char* path);
zj_status zj_restart_read(zj_solver* s, const char* path);

/* ---- Gmsh meshes -------------------------------------------------------------
 * Read an ASCII Gmsh MSH v2.2 / v4.1 mesh (GmshReader::read,
 * src/mesh/gmsh_reader.cpp:161-396) into library-owned arrays; no device is
 * touched.  Failures return ZJ_ERR_IO (cannot open) or ZJ_ERR_ARG (format,
 * unknown node tag, no 2D elements) with the reader's message in
 * zj_last_error(NULL). */
typedef struct zj_gmsh_mesh zj_gmsh_mesh;
zj_status zj_gmsh_read(const char* msh_path, zj_gmsh_mesh** out);
void zj_gmsh_free(zj_gmsh_mesh* m);
/* The mesh as a solver descriptor (valid until zj_gmsh_free). */
const zj_mesh_desc* zj_gmsh_desc(const zj_gmsh_mesh* m);
/* Boundary groups (GmshReader::mapBoundaryConditions, gmsh_reader.cpp:651-709):
 * physical tag, type inferred from the physical name (GmshReader::inferBCType,
 * gmsh_reader.cpp:117-155) and the name ("BC_<tag>" when unnamed). */
int zj_gmsh_num_groups(const zj_gmsh_mesh* m);
zj_status zj_gmsh_group(const zj_gmsh_mesh* m, int i, int* tag, int* bc_type, const char** name);

/* Read a Gmsh mesh and create a solver.  Boundary groups the params' bc table
 * does not name get their inferred type (as the reference's reader stamps
 * them on the faces, gmsh_reader.cpp:715-758). */
zj_status zj_solver_create_from_gmsh(const char* msh_path, const zj_params* params,
                                     zj_solver** out);

#ifdef __cplusplus
}
#endif
#endif /* ZJ_FR_H */
