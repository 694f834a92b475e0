/*
 * fr_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the reference Flux-Reconstruction residual and SSP-RK3
 * stepper ("compat" semantics: the reference's exact arithmetic, quirks and
 * clamps included).  Only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it, and only as the checker or the
 * timed CPU baseline.  The product library never links or calls it.
 *
 * Parity pins: operators, faces, normals and metrics are checked bit for bit
 * against the reference's own basis.cpp / mesh.cpp / fr_solver.cpp compiled
 * from the reference sources (oracle/ref/), and the residual against the
 * reference's own CUDA build run on a B200 (tests/golden/).
 */
#ifndef ZJ_FR_ORACLE_H
#define ZJ_FR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* Build the oracle for a quad mesh.  conn is [n_elem][nn] (nn = 4, 9 or 25 for
 * element order 1, 2 or 4; vertices CCW first).  bnd is [n_bnd][3] =
 * (v0, v1, tag).  tag_* give the BC type (reference BCType numbering) and the
 * outflow static pressure for each tag (0 = use p_inf).  Returns NULL on a bad
 * argument. */
orc_ctx* orc_create(int P, double gamma, double rho_inf, double p_inf,
                    double Mach, double AoA_deg,
                    int64_t n_nodes, const double* xy,
                    int64_t n_elem, int nn, int elem_order, const int64_t* conn,
                    int64_t n_bnd, const int64_t* bnd,
                    int n_tags, const int* tag_ids, const int* tag_types,
                    const double* tag_pstatic);
void orc_destroy(orc_ctx* c);
void orc_set_threads(orc_ctx* c, int n);

int64_t orc_num_faces(const orc_ctx* c);
int orc_num_sp(const orc_ctx* c);
/* Face table in the reference's face order (sorted vertex pair). */
void orc_faces(const orc_ctx* c, int* left_elem, int* left_local,
               int* right_elem, int* right_local, int* bc_type, int* bc_tag,
               double* normals);
/* J [E][n_sp], Jinv [E][n_sp][4] = (xi_x, xi_y, eta_x, eta_y). */
void orc_geometry(const orc_ctx* c, double* J, double* Jinv);
/* pts1d [n1], D1 [n1][n1], diff_xi/diff_eta [n_sp][n_sp],
 * interp [4][n1][n_sp], corr [4][n_sp]. */
void orc_operators(const orc_ctx* c, double* pts1d, double* D1,
                   double* diff_xi, double* diff_eta, double* interp,
                   double* corr);
/* Physical coordinates of every solution point, [E][n_sp][2]. */
void orc_sp_coords(const orc_ctx* c, double* xy);

/* One residual R = dU/dt on AoS [E][n_sp][4] data. */
void orc_rhs(orc_ctx* c, const double* U, double* R);
/* nsteps SSP-RK3 steps of size dt in place, positivity clamp after every
 * stage; R_last (may be NULL) receives the last stage's residual. */
void orc_step(orc_ctx* c, double* U, double dt, int nsteps, double* R_last);
/* CFL time step over state U (reference computeTimeStep formula). */
double orc_compute_dt(const orc_ctx* c, const double* U, double CFL);
/* L2 norm over n values, summed in index order. */
double orc_l2(const double* R, int64_t n);

/* ---- physics mode (compat off): conservative FR, VCJH, reference formula
 * sources for the Riemann solvers and ghost states. ---------------------- */
void orc_set_physics(orc_ctx* c, int flux_type, int riemann, int viscous, double Re, double Pr,
                     double T_inf);
/* per-tag inflow total pressure/temperature/direction and wall temperature */
void orc_set_bc_extra(orc_ctx* c, int n, const int* tag_ids, const double* p_total,
                      const double* T_total, const double* dir_x, const double* dir_y,
                      const double* T_wall);
void orc_get_vcjh(const orc_ctx* c, double* gL, double* gR);
void orc_vcjh(int P, int flux_type, const double* x, double* gL, double* gR);
void orc_rhs_phys(orc_ctx* c, const double* U, double* R);
/* viscous flux at one state with gradients dx = dU/dx, dy = dU/dy (the
 * kernel's viscosity law, kernels.cu:742-786) */
void orc_viscous_flux(const double* U, const double* dx, const double* dy, double g, double Re,
                      double Pr, double* Fv, double* Gv);
/* the same with law 0 (kernel law) or 1 (the header's Sutherland law,
 * navierstokes.hpp:17-96) */
void orc_viscous_flux_law(int law, const double* U, const double* dx, const double* dy, double g,
                          double Re, double Pr, double* Fv, double* Gv);
/* common normal viscous flux of a face point (BR2Scheme::commonFlux,
 * navierstokes.hpp:166-201) under law 0 or 1 */
void orc_common_viscous_law(int law, const double* UL, const double* UR, const double* dxL,
                            const double* dyL, const double* dxR, const double* dyR, double nx,
                            double ny, double g, double Re, double Pr, double* Fvn);
void orc_step_phys(orc_ctx* c, double* U, double dt, int nsteps, double* R_last);
/* pointwise pins: which = 0 Rusanov, 1 Roe, 2 HLLC */
void orc_riemann_point(int which, const double* UL, const double* UR, double nx, double ny,
                       double g, double* F);
void orc_ghost_point(const orc_ctx* c, int bc_type, int tag, const double* Ui, double nx,
                     double ny, double* Ug);
/* the walls' Neumann data on a boundary face's common normal viscous flux */
void orc_wall_viscous_closure(const orc_ctx* c, int bc_type, int tag, double nx, double ny,
                              double* Fvn);

#ifdef __cplusplus
}
#endif
#endif
