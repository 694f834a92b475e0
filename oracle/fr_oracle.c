/*
 * fr_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE (see fr_oracle.h).
 *
 * Plain-C restatement of the reference FR hot path in its own loop and
 * summation order.  Compile with -ffp-contract=off: every product and sum is
 * rounded as written, like the reference host code and unlike an FMA-fused
 * GPU build (which differs from it by a few ulp per operation).
 *
 * Reference map (paths inside the Zhijian project):
 *   Gauss-Legendre points      src/basis/basis.cpp:12-104
 *   Lagrange eval / deriv      src/basis/basis.cpp:169-224
 *   correction derivatives     src/basis/basis.cpp:314-379
 *   FROperators::initQuad      src/basis/basis.cpp:464-613
 *   shape functions, Jacobian  src/basis/basis.cpp:717-893
 *   Mesh::buildFaces           src/mesh/mesh.cpp:18-83
 *   areas, normals, centroids  src/mesh/mesh.cpp:109-194
 *   initGeometry               src/solver/fr_solver.cpp:85-129
 *   BC packing                 src/solver/fr_solver.cpp:432-494
 *   advance                    src/solver/fr_solver.cpp:305-333
 *   computeTimeStep            src/solver/fr_solver.cpp:784-816
 *   IdealGas                   include/physics/euler.hpp:16-129
 *   kernels K1,K4,K8,K9,K10,K13,K15,K17,K18  src/gpu/kernels.cu (see each fn)
 */
#include "fr_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

enum { BC_INTERIOR = 0, BC_WALL = 1, BC_SLIPWALL = 2, BC_SYMMETRY = 3,
       BC_FARFIELD = 4, BC_INFLOW = 5, BC_OUTFLOW = 6, BC_PERIODIC = 7 };

struct orc_ctx {
    int P, n1, nsp, nfp, nn, eorder;
    int64_t n_elem, n_nodes, n_faces;
    double gamma, rho_inf, u_inf, v_inf, p_inf;
    double* xy;       /* [n_nodes][2] */
    int64_t* conn;    /* [E][nn] */
    /* geometry */
    double *J, *Jinv, *area;
    /* faces */
    int *fle, *fll, *fre, *frl, *fbct, *ftag, *fbcmap;
    double *fn, *bc_data;
    /* operators */
    double *pts, *D1, *dxi, *deta, *interp, *corr;
    /* work */
    double *Fx, *Fy, *Ufp, *Fcom, *Fdiff, *U0, *U1;
    int nthreads;
    /* physics mode */
    int flux_type, riemann, viscous;
    double Re, Pr, T_inf;
    double gLp[16], gRp[16];
    int n_tags;
    int tag_ids[64];
    double tag_pt[64], tag_Tt[64], tag_dx[64], tag_dy[64], tag_Tw[64], tag_ps[64];
    double *flen;
    double *fpn;      /* curved meshes, physics mode: [nf][nfp][3] (nx, ny, s) per face point */
};

/* ---------------------------------------------------------------- basis -- */

/* basis.cpp:12-104 */
static void gl_points(int n, double* x, double* w) {
    switch (n) {
    case 1: x[0] = 0.0; w[0] = 2.0; break;
    case 2: x[0] = -1.0 / sqrt(3.0); x[1] = 1.0 / sqrt(3.0); w[0] = w[1] = 1.0; break;
    case 3:
        x[0] = -sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = sqrt(3.0 / 5.0);
        w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0; break;
    case 4:
        x[0] = -sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
        x[1] = -sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
        x[2] = sqrt(3.0 / 7.0 - 2.0 / 7.0 * sqrt(6.0 / 5.0));
        x[3] = sqrt(3.0 / 7.0 + 2.0 / 7.0 * sqrt(6.0 / 5.0));
        w[0] = w[3] = (18.0 - sqrt(30.0)) / 36.0;
        w[1] = w[2] = (18.0 + sqrt(30.0)) / 36.0; break;
    case 5:
        x[0] = -sqrt(5.0 + 2.0 * sqrt(10.0 / 7.0)) / 3.0;
        x[1] = -sqrt(5.0 - 2.0 * sqrt(10.0 / 7.0)) / 3.0;
        x[2] = 0.0;
        x[3] = sqrt(5.0 - 2.0 * sqrt(10.0 / 7.0)) / 3.0;
        x[4] = sqrt(5.0 + 2.0 * sqrt(10.0 / 7.0)) / 3.0;
        w[0] = w[4] = (322.0 - 13.0 * sqrt(70.0)) / 900.0;
        w[1] = w[3] = (322.0 + 13.0 * sqrt(70.0)) / 900.0;
        w[2] = 128.0 / 225.0; break;
    case 6: /* the reference's 15-digit table */
        x[0] = -0.932469514203152; x[1] = -0.661209386466265; x[2] = -0.238619186083197;
        x[3] = 0.238619186083197;  x[4] = 0.661209386466265;  x[5] = 0.932469514203152;
        w[0] = w[5] = 0.171324492379170; w[1] = w[4] = 0.360761573048139;
        w[2] = w[3] = 0.467913934572691; break;
    default:
        for (int i = 0; i < n; ++i) {
            double xx = cos(M_PI * (i + 0.75) / (n + 0.5));
            for (int it = 0; it < 20; ++it) {
                double P0 = 1.0, P1 = xx;
                for (int j = 2; j <= n; ++j) {
                    double Pn = ((2 * j - 1) * xx * P1 - (j - 1) * P0) / j;
                    P0 = P1; P1 = Pn;
                }
                double dP = n * (xx * P1 - P0) / (xx * xx - 1.0);
                double dx = P1 / dP;
                xx -= dx;
                if (fabs(dx) < 1e-15) break;
            }
            x[i] = xx;
            double P0 = 1.0, P1 = xx;
            for (int j = 2; j <= n; ++j) {
                double Pn = ((2 * j - 1) * xx * P1 - (j - 1) * P0) / j;
                P0 = P1; P1 = Pn;
            }
            double dP = n * (xx * P1 - P0) / (xx * xx - 1.0);
            w[i] = 2.0 / ((1.0 - xx * xx) * dP * dP);
        }
    }
}

/* basis.cpp:169-178 */
static double lag_eval(const double* nodes, int n, int j, double x) {
    double r = 1.0;
    for (int i = 0; i < n; ++i)
        if (i != j) r *= (x - nodes[i]) / (nodes[j] - nodes[i]);
    return r;
}

/* basis.cpp:180-196 */
static double lag_deriv(const double* nodes, int n, int j, double x) {
    double r = 0.0;
    for (int k = 0; k < n; ++k) {
        if (k == j) continue;
        double term = 1.0 / (nodes[j] - nodes[k]);
        for (int i = 0; i < n; ++i)
            if (i != j && i != k) term *= (x - nodes[i]) / (nodes[j] - nodes[i]);
        r += term;
    }
    return r;
}

static double legendre(int n, double x) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    double P0 = 1.0, P1 = x;
    for (int i = 2; i <= n; ++i) {
        double Pn = ((2 * i - 1) * x * P1 - (i - 1) * P0) / i;
        P0 = P1; P1 = Pn;
    }
    return P1;
}

static double legendre_deriv(int n, double x) {
    if (n == 0) return 0.0;
    double Pn = legendre(n, x), Pn1 = legendre(n - 1, x);
    if (fabs(x * x - 1.0) < 1e-14)
        return n * (n + 1) / 2.0 * ((x > 0) ? 1.0 : ((n % 2 == 0) ? 1.0 : -1.0));
    return n / (x * x - 1.0) * (x * Pn - Pn1);
}

/* basis.cpp:314-348 (Radau left; the reference ignores flux_type) */
static double gL_deriv(int p, double x) {
    double dPp = legendre_deriv(p, x), dPp1 = legendre_deriv(p + 1, x);
    double sign = (p % 2 == 0) ? 1.0 : -1.0;
    return sign * 0.5 * (dPp - dPp1);
}

/* basis.cpp:350-379 */
static double gR_deriv(int p, double x) {
    double dPp = legendre_deriv(p, x), dPp1 = legendre_deriv(p + 1, x);
    return 0.5 * (dPp + dPp1);
}

/* basis.cpp:464-613 */
static void build_operators(orc_ctx* c) {
    int p = c->P, n1 = c->n1, nsp = c->nsp;
    double w[16];
    gl_points(n1, c->pts, w);
    const double* pts = c->pts;
    for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n1; ++j) c->D1[i * n1 + j] = lag_deriv(pts, n1, j, pts[i]);
    memset(c->dxi, 0, sizeof(double) * nsp * nsp);
    memset(c->deta, 0, sizeof(double) * nsp * nsp);
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= p; ++i) {
            int row = j * n1 + i;
            for (int k = 0; k <= p; ++k) {
                c->dxi[row * nsp + j * n1 + k] = c->D1[i * n1 + k];
                c->deta[row * nsp + k * n1 + i] = c->D1[j * n1 + k];
            }
        }
    for (int e = 0; e < 4; ++e)
        for (int fp = 0; fp < n1; ++fp) {
            double s = pts[fp], xf, ef;
            if (e == 0) { xf = s; ef = -1.0; }
            else if (e == 1) { xf = 1.0; ef = s; }
            else if (e == 2) { xf = -s; ef = 1.0; }
            else { xf = -1.0; ef = -s; }
            double Lx[16], Le[16];
            for (int j = 0; j < n1; ++j) { Lx[j] = lag_eval(pts, n1, j, xf); Le[j] = lag_eval(pts, n1, j, ef); }
            for (int j = 0; j <= p; ++j)
                for (int i = 0; i <= p; ++i)
                    c->interp[(e * n1 + fp) * nsp + j * n1 + i] = Lx[i] * Le[j];
        }
    for (int e = 0; e < 4; ++e)
        for (int j = 0; j <= p; ++j)
            for (int i = 0; i <= p; ++i) {
                int sp = j * n1 + i;
                double xi = pts[i], eta = pts[j], v;
                if (e == 0) v = gL_deriv(p, eta) * lag_eval(pts, n1, i, xi);
                else if (e == 2) v = gR_deriv(p, eta) * lag_eval(pts, n1, i, xi);
                else if (e == 3) v = gL_deriv(p, xi) * lag_eval(pts, n1, j, eta);
                else v = gR_deriv(p, xi) * lag_eval(pts, n1, j, eta);
                c->corr[e * nsp + sp] = v;
            }
}

/* ------------------------------------------------------------- geometry -- */

static const int Q4_XI[25] = {0,4,4,0, 1,2,3, 4,4,4, 3,2,1, 0,0,0, 1,2,3,1,2,3,1,2,3};
static const int Q4_ETA[25] = {0,0,4,4, 0,0,0, 1,2,3, 4,4,4, 3,2,1, 1,1,1,2,2,2,3,3,3};

static void q4_lag(double t, double* L, double* dL) {
    static const double nd[5] = {-1.0, -0.5, 0.0, 0.5, 1.0};
    for (int i = 0; i < 5; ++i) {
        L[i] = 1.0;
        for (int j = 0; j < 5; ++j) if (j != i) L[i] *= (t - nd[j]) / (nd[i] - nd[j]);
        dL[i] = 0.0;
        for (int k = 0; k < 5; ++k) {
            if (k == i) continue;
            double pr = 1.0 / (nd[i] - nd[k]);
            for (int j = 0; j < 5; ++j) if (j != i && j != k) pr *= (t - nd[j]) / (nd[i] - nd[j]);
            dL[i] += pr;
        }
    }
}

/* basis.cpp:717-847: shape functions and derivatives of quads. */
static int shape_quad(int order, double xi, double eta, double* N, double* dNx, double* dNe) {
    if (order == 1) {
        N[0] = 0.25 * (1 - xi) * (1 - eta); N[1] = 0.25 * (1 + xi) * (1 - eta);
        N[2] = 0.25 * (1 + xi) * (1 + eta); N[3] = 0.25 * (1 - xi) * (1 + eta);
        dNx[0] = -0.25 * (1 - eta); dNe[0] = -0.25 * (1 - xi);
        dNx[1] = 0.25 * (1 - eta);  dNe[1] = -0.25 * (1 + xi);
        dNx[2] = 0.25 * (1 + eta);  dNe[2] = 0.25 * (1 + xi);
        dNx[3] = -0.25 * (1 + eta); dNe[3] = 0.25 * (1 - xi);
        return 4;
    }
    if (order == 2) {
        N[0] = 0.25 * xi * (xi - 1) * eta * (eta - 1);
        N[1] = 0.25 * xi * (xi + 1) * eta * (eta - 1);
        N[2] = 0.25 * xi * (xi + 1) * eta * (eta + 1);
        N[3] = 0.25 * xi * (xi - 1) * eta * (eta + 1);
        N[4] = 0.5 * (1 - xi * xi) * eta * (eta - 1);
        N[5] = 0.5 * xi * (xi + 1) * (1 - eta * eta);
        N[6] = 0.5 * (1 - xi * xi) * eta * (eta + 1);
        N[7] = 0.5 * xi * (xi - 1) * (1 - eta * eta);
        N[8] = (1 - xi * xi) * (1 - eta * eta);
        dNx[0] = 0.25 * (2 * xi - 1) * eta * (eta - 1); dNe[0] = 0.25 * xi * (xi - 1) * (2 * eta - 1);
        dNx[1] = 0.25 * (2 * xi + 1) * eta * (eta - 1); dNe[1] = 0.25 * xi * (xi + 1) * (2 * eta - 1);
        dNx[2] = 0.25 * (2 * xi + 1) * eta * (eta + 1); dNe[2] = 0.25 * xi * (xi + 1) * (2 * eta + 1);
        dNx[3] = 0.25 * (2 * xi - 1) * eta * (eta + 1); dNe[3] = 0.25 * xi * (xi - 1) * (2 * eta + 1);
        dNx[4] = -xi * eta * (eta - 1);               dNe[4] = 0.5 * (1 - xi * xi) * (2 * eta - 1);
        dNx[5] = 0.5 * (2 * xi + 1) * (1 - eta * eta); dNe[5] = -xi * (xi + 1) * eta;
        dNx[6] = -xi * eta * (eta + 1);               dNe[6] = 0.5 * (1 - xi * xi) * (2 * eta + 1);
        dNx[7] = 0.5 * (2 * xi - 1) * (1 - eta * eta); dNe[7] = -xi * (xi - 1) * eta;
        dNx[8] = -2 * xi * (1 - eta * eta);            dNe[8] = -2 * eta * (1 - xi * xi);
        return 9;
    }
    if (order == 4) {
        double Lx[5], Le[5], dLx[5], dLe[5];
        q4_lag(xi, Lx, dLx);
        q4_lag(eta, Le, dLe);
        for (int k = 0; k < 25; ++k) {
            N[k] = Lx[Q4_XI[k]] * Le[Q4_ETA[k]];
            dNx[k] = dLx[Q4_XI[k]] * Le[Q4_ETA[k]];
            dNe[k] = Lx[Q4_XI[k]] * dLe[Q4_ETA[k]];
        }
        return 25;
    }
    return 0;
}

/* fr_solver.cpp:85-129 with basis.cpp:849-863 */
static void build_geometry(orc_ctx* c) {
    int nsp = c->nsp, n1 = c->n1;
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int64_t* nd = c->conn + e * c->nn;
        for (int sp = 0; sp < nsp; ++sp) {
            double xi = c->pts[sp % n1], eta = c->pts[sp / n1];
            double N[25], dNx[25], dNe[25];
            int n = shape_quad(c->eorder, xi, eta, N, dNx, dNe);
            double dxdxi = 0.0, dxdeta = 0.0, dydxi = 0.0, dydeta = 0.0;
            for (int i = 0; i < n; ++i) {
                double x = c->xy[2 * nd[i]], y = c->xy[2 * nd[i] + 1];
                dxdxi += dNx[i] * x; dxdeta += dNe[i] * x;
                dydxi += dNx[i] * y; dydeta += dNe[i] * y;
            }
            double Jd = dxdxi * dydeta - dxdeta * dydxi;
            double invJ = 1.0 / Jd;
            c->J[e * nsp + sp] = Jd;
            double* Ji = c->Jinv + (e * nsp + sp) * 4;
            Ji[0] = dydeta * invJ; Ji[1] = -dxdeta * invJ;
            Ji[2] = -dydxi * invJ; Ji[3] = dxdxi * invJ;
        }
        /* mesh.cpp:122-146 (quad split into two triangles) */
        const double *p0 = c->xy + 2 * nd[0], *p1 = c->xy + 2 * nd[1];
        const double *p2 = c->xy + 2 * nd[2], *p3 = c->xy + 2 * nd[3];
        double a1 = 0.5 * fabs((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
        double a2 = 0.5 * fabs((p2[0] - p0[0]) * (p3[1] - p0[1]) - (p3[0] - p0[0]) * (p2[1] - p0[1]));
        c->area[e] = a1 + a2;
    }
}

/* ---------------------------------------------------------------- faces -- */

typedef struct { int64_t a, b, seq; int e, l; } edge_ent;

static int cmp_edge(const void* x, const void* y) {
    const edge_ent *p = (const edge_ent*)x, *q = (const edge_ent*)y;
    if (p->a != q->a) return p->a < q->a ? -1 : 1;
    if (p->b != q->b) return p->b < q->b ? -1 : 1;
    if (p->seq != q->seq) return p->seq < q->seq ? -1 : 1;
    return 0;
}

/* mesh.cpp:159-183 */
static void face_normal(const orc_ctx* c, int e, int lf, double* n) {
    const int64_t* nd = c->conn + (int64_t)e * c->nn;
    const double* v0 = c->xy + 2 * nd[lf];
    const double* v1 = c->xy + 2 * nd[(lf + 1) % 4];
    double tx = v1[0] - v0[0], ty = v1[1] - v0[1];
    double len = sqrt(tx * tx + ty * ty);
    double nx = ty / len, ny = -tx / len;
    double cx = 0.0, cy = 0.0;
    for (int i = 0; i < 4; ++i) { cx = cx + c->xy[2 * nd[i]]; cy = cy + c->xy[2 * nd[i] + 1]; }
    cx = cx / 4.0; cy = cy / 4.0;
    double fx = (v0[0] + v1[0]) * 0.5, fy = (v0[1] + v1[1]) * 0.5;
    double dx = fx - cx, dy = fy - cy;
    if (nx * dx + ny * dy < 0) { nx = nx * (-1.0); ny = ny * (-1.0); }
    n[0] = nx; n[1] = ny;
}

static int build_faces(orc_ctx* c, int64_t n_bnd, const int64_t* bnd,
                       int n_tags, const int* tag_ids, const int* tag_types,
                       const double* tag_ps) {
    int64_t ne = c->n_elem;
    edge_ent* ent = (edge_ent*)malloc(sizeof(edge_ent) * (size_t)(ne * 4 + 1));
    if (!ent) return -1;
    for (int64_t e = 0; e < ne; ++e)
        for (int l = 0; l < 4; ++l) {
            int64_t v0 = c->conn[e * c->nn + l], v1 = c->conn[e * c->nn + (l + 1) % 4];
            edge_ent* q = ent + e * 4 + l;
            q->a = v0 < v1 ? v0 : v1; q->b = v0 < v1 ? v1 : v0;
            q->seq = e * 4 + l; q->e = (int)e; q->l = l;
        }
    qsort(ent, (size_t)(ne * 4), sizeof(edge_ent), cmp_edge);
    /* boundary-edge tag lookup: last definition of a vertex pair wins */
    edge_ent* be = (edge_ent*)malloc(sizeof(edge_ent) * (size_t)(n_bnd + 1));
    int64_t nbe = 0;
    for (int64_t i = 0; i < n_bnd; ++i) {
        int64_t v0 = bnd[3 * i], v1 = bnd[3 * i + 1];
        int tag = (int)bnd[3 * i + 2];
        if (tag <= 0) continue;
        be[nbe].a = v0 < v1 ? v0 : v1; be[nbe].b = v0 < v1 ? v1 : v0;
        be[nbe].seq = i; be[nbe].e = tag; be[nbe].l = 0; ++nbe;
    }
    qsort(be, (size_t)nbe, sizeof(edge_ent), cmp_edge);

    int64_t cap = ne * 4, nf = 0, nbc = 0;
    c->fle = (int*)malloc(sizeof(int) * cap); c->fll = (int*)malloc(sizeof(int) * cap);
    c->fre = (int*)malloc(sizeof(int) * cap); c->frl = (int*)malloc(sizeof(int) * cap);
    c->fbct = (int*)malloc(sizeof(int) * cap); c->ftag = (int*)malloc(sizeof(int) * cap);
    c->fbcmap = (int*)malloc(sizeof(int) * cap);
    c->fn = (double*)malloc(sizeof(double) * 2 * cap);
    c->flen = (double*)malloc(sizeof(double) * cap);
    c->bc_data = (double*)calloc((size_t)(cap * 8 + 8), sizeof(double));
    double c_inf = sqrt(c->gamma * c->p_inf / c->rho_inf);
    (void)c_inf;
    int64_t i = 0, jb = 0;
    while (i < ne * 4) {
        int64_t j = i;
        while (j < ne * 4 && ent[j].a == ent[i].a && ent[j].b == ent[i].b) ++j;
        int64_t cnt = j - i;
        if (cnt == 1 || cnt == 2) {
            int f = (int)nf++;
            c->fle[f] = ent[i].e; c->fll[f] = ent[i].l;
            if (cnt == 1) {
                c->fre[f] = -1; c->frl[f] = -1;
                c->fbct[f] = BC_FARFIELD; c->ftag[f] = 0;
                /* mesh.cpp:48-57 default, then gmsh_reader.cpp:736-758 tagging */
                while (jb < nbe && (be[jb].a < ent[i].a || (be[jb].a == ent[i].a && be[jb].b < ent[i].b))) ++jb;
                int64_t k = jb, last = -1;
                while (k < nbe && be[k].a == ent[i].a && be[k].b == ent[i].b) last = k++;
                if (last >= 0) {
                    int tag = be[last].e;
                    c->ftag[f] = tag;
                    for (int t = 0; t < n_tags; ++t)
                        if (tag_ids[t] == tag) c->fbct[f] = tag_types[t];
                }
            } else {
                c->fre[f] = ent[i + 1].e; c->frl[f] = ent[i + 1].l;
                c->fbct[f] = BC_INTERIOR; c->ftag[f] = -1;
            }
            face_normal(c, c->fle[f], c->fll[f], c->fn + 2 * f);
            {   /* mesh.cpp:148-157 */
                const int64_t* nd = c->conn + (int64_t)c->fle[f] * c->nn;
                const double* v0 = c->xy + 2 * nd[c->fll[f]];
                const double* v1 = c->xy + 2 * nd[(c->fll[f] + 1) % 4];
                double tx = v1[0] - v0[0], ty = v1[1] - v0[1];
                c->flen[f] = sqrt(tx * tx + ty * ty);
            }
            /* fr_solver.cpp:432-482 BC packing, 8 values per boundary face */
            if (cnt == 1) {
                c->fbcmap[f] = (int)nbc;
                double* d = c->bc_data + 8 * nbc;
                if (c->fbct[f] == BC_FARFIELD) {
                    d[0] = c->rho_inf; d[1] = c->u_inf; d[2] = c->v_inf; d[3] = c->p_inf;
                } else if (c->fbct[f] == BC_OUTFLOW) {
                    double ps = c->p_inf;
                    for (int t = 0; t < n_tags; ++t)
                        if (c->ftag[f] > 0 && tag_ids[t] == c->ftag[f] && tag_ps[t] > 0) ps = tag_ps[t];
                    d[0] = ps;
                }
                ++nbc;
            } else {
                c->fbcmap[f] = -1;
            }
        }
        i = j;
    }
    c->n_faces = nf;
    free(ent);
    free(be);
    return 0;
}

/* ---------------------------------------------------------------- create -- */

orc_ctx* orc_create(int P, double gamma, double rho_inf, double p_inf,
                    double Mach, double AoA_deg,
                    int64_t n_nodes, const double* xy,
                    int64_t n_elem, int nn, int elem_order, const int64_t* conn,
                    int64_t n_bnd, const int64_t* bnd,
                    int n_tags, const int* tag_ids, const int* tag_types,
                    const double* tag_pstatic) {
    if (P < 0 || P > 8 || n_elem <= 0 || n_nodes <= 0) return NULL;
    if (!((elem_order == 1 && nn == 4) || (elem_order == 2 && nn == 9) || (elem_order == 4 && nn == 25)))
        return NULL;
    orc_ctx* c = (orc_ctx*)calloc(1, sizeof(orc_ctx));
    c->P = P; c->n1 = P + 1; c->nsp = (P + 1) * (P + 1); c->nfp = P + 1;
    c->nn = nn; c->eorder = elem_order;
    c->n_elem = n_elem; c->n_nodes = n_nodes;
    c->gamma = gamma; c->rho_inf = rho_inf; c->p_inf = p_inf;
    /* fr_solver.cpp:439-443 */
    double c_inf = sqrt(gamma * p_inf / rho_inf);
    double vel_inf = Mach * c_inf;
    c->u_inf = vel_inf * cos(AoA_deg * M_PI / 180.0);
    c->v_inf = vel_inf * sin(AoA_deg * M_PI / 180.0);
    c->xy = (double*)malloc(sizeof(double) * 2 * n_nodes);
    memcpy(c->xy, xy, sizeof(double) * 2 * n_nodes);
    c->conn = (int64_t*)malloc(sizeof(int64_t) * n_elem * nn);
    memcpy(c->conn, conn, sizeof(int64_t) * n_elem * nn);
    for (int64_t k = 0; k < n_elem * nn; ++k)
        if (conn[k] < 0 || conn[k] >= n_nodes) { orc_destroy(c); return NULL; }
    int nsp = c->nsp, n1 = c->n1;
    c->pts = (double*)malloc(sizeof(double) * n1);
    c->D1 = (double*)malloc(sizeof(double) * n1 * n1);
    c->dxi = (double*)malloc(sizeof(double) * nsp * nsp);
    c->deta = (double*)malloc(sizeof(double) * nsp * nsp);
    c->interp = (double*)malloc(sizeof(double) * 4 * n1 * nsp);
    c->corr = (double*)malloc(sizeof(double) * 4 * nsp);
    build_operators(c);
    c->J = (double*)malloc(sizeof(double) * n_elem * nsp);
    c->Jinv = (double*)malloc(sizeof(double) * n_elem * nsp * 4);
    c->area = (double*)malloc(sizeof(double) * n_elem);
    build_geometry(c);
    c->n_tags = n_tags < 64 ? n_tags : 64;
    for (int t = 0; t < c->n_tags; ++t) {
        c->tag_ids[t] = tag_ids[t]; c->tag_ps[t] = tag_pstatic[t];
        c->tag_pt[t] = 0.0; c->tag_Tt[t] = 0.0; c->tag_dx[t] = 1.0; c->tag_dy[t] = 0.0; c->tag_Tw[t] = 0.0;
    }
    c->flux_type = 2; c->riemann = 0; c->viscous = 0; c->Re = 1000.0; c->Pr = 0.72; c->T_inf = 300.0;
    if (build_faces(c, n_bnd, bnd, n_tags, tag_ids, tag_types, tag_pstatic) != 0) {
        orc_destroy(c); return NULL;
    }
    size_t sol = (size_t)n_elem * nsp * 4, fpn = (size_t)n_elem * 4 * n1 * 4;
    c->Fx = (double*)malloc(sizeof(double) * sol);
    c->Fy = (double*)malloc(sizeof(double) * sol);
    c->U0 = (double*)malloc(sizeof(double) * sol);
    c->U1 = (double*)malloc(sizeof(double) * sol);
    c->Ufp = (double*)malloc(sizeof(double) * fpn);
    c->Fdiff = (double*)malloc(sizeof(double) * fpn);
    c->Fcom = (double*)malloc(sizeof(double) * (size_t)(c->n_faces > 0 ? c->n_faces : 1) * n1 * 4);
    c->nthreads = 1;
    return c;
}

void orc_destroy(orc_ctx* c) {
    if (!c) return;
    void* ps[] = {c->xy, c->conn, c->J, c->Jinv, c->area, c->fle, c->fll, c->fre, c->frl,
                  c->fbct, c->ftag, c->fbcmap, c->fn, c->bc_data, c->pts, c->D1, c->dxi,
                  c->deta, c->interp, c->corr, c->Fx, c->Fy, c->Ufp, c->Fcom, c->Fdiff,
                  c->U0, c->U1, c->flen, c->fpn};
    for (size_t i = 0; i < sizeof(ps) / sizeof(ps[0]); ++i) free(ps[i]);
    free(c);
}

void orc_set_threads(orc_ctx* c, int n) { c->nthreads = n > 0 ? n : 1; }
int64_t orc_num_faces(const orc_ctx* c) { return c->n_faces; }
int orc_num_sp(const orc_ctx* c) { return c->nsp; }

void orc_faces(const orc_ctx* c, int* le, int* ll, int* re, int* rl, int* bct, int* tag, double* n) {
    size_t nf = (size_t)c->n_faces;
    memcpy(le, c->fle, nf * sizeof(int)); memcpy(ll, c->fll, nf * sizeof(int));
    memcpy(re, c->fre, nf * sizeof(int)); memcpy(rl, c->frl, nf * sizeof(int));
    memcpy(bct, c->fbct, nf * sizeof(int)); memcpy(tag, c->ftag, nf * sizeof(int));
    memcpy(n, c->fn, nf * 2 * sizeof(double));
}

void orc_geometry(const orc_ctx* c, double* J, double* Jinv) {
    memcpy(J, c->J, sizeof(double) * c->n_elem * c->nsp);
    memcpy(Jinv, c->Jinv, sizeof(double) * c->n_elem * c->nsp * 4);
}

void orc_operators(const orc_ctx* c, double* pts, double* D1, double* dxi, double* deta,
                   double* interp, double* corr) {
    int n1 = c->n1, nsp = c->nsp;
    memcpy(pts, c->pts, sizeof(double) * n1);
    memcpy(D1, c->D1, sizeof(double) * n1 * n1);
    memcpy(dxi, c->dxi, sizeof(double) * nsp * nsp);
    memcpy(deta, c->deta, sizeof(double) * nsp * nsp);
    memcpy(interp, c->interp, sizeof(double) * 4 * n1 * nsp);
    memcpy(corr, c->corr, sizeof(double) * 4 * nsp);
}

/* fr_solver.cpp:268-299 with basis.cpp:882-893 */
void orc_sp_coords(const orc_ctx* c, double* out) {
    int nsp = c->nsp, n1 = c->n1;
    for (int64_t e = 0; e < c->n_elem; ++e) {
        const int64_t* nd = c->conn + e * c->nn;
        for (int sp = 0; sp < nsp; ++sp) {
            double N[25], dNx[25], dNe[25];
            int n = shape_quad(c->eorder, c->pts[sp % n1], c->pts[sp / n1], N, dNx, dNe);
            double x = 0.0, y = 0.0;
            for (int i = 0; i < n; ++i) { x += N[i] * c->xy[2 * nd[i]]; y += N[i] * c->xy[2 * nd[i] + 1]; }
            out[(e * nsp + sp) * 2] = x;
            out[(e * nsp + sp) * 2 + 1] = y;
        }
    }
}

/* --------------------------------------------------------------- physics -- */

/* euler.hpp:16-23 */
static double pressure(const double* U, double g) {
    double rho = U[0], u = U[1] / rho, v = U[2] / rho, E = U[3] / rho;
    double ke = 0.5 * (u * u + v * v);
    return (g - 1.0) * rho * (E - ke);
}

/* euler.hpp:101-129 */
static void flux_xy(const double* U, double g, double* F, double* G) {
    double rho = U[0], u = U[1] / rho, v = U[2] / rho, p = pressure(U, g);
    F[0] = U[1]; F[1] = U[1] * u + p; F[2] = U[1] * v; F[3] = (U[3] + p) * u;
    G[0] = U[2]; G[1] = U[2] * u; G[2] = U[2] * v + p; G[3] = (U[3] + p) * v;
}

/* euler.hpp:81-88 */
static void prim2cons(double rho, double u, double v, double p, double g, double* U) {
    U[0] = rho; U[1] = rho * u; U[2] = rho * v;
    U[3] = p / (g - 1.0) + 0.5 * rho * (u * u + v * v);
}

/* kernels.cu:453-525 */
static void ghost_state(const double* Ui, double nx, double ny, int bct,
                        const double* bcd, int bci, double g, double* Ug) {
    switch (bct) {
    case BC_WALL: case BC_SLIPWALL: case BC_SYMMETRY: {
        double rho = Ui[0], u = Ui[1] / rho, v = Ui[2] / rho;
        double p = pressure(Ui, g);
        double vn = u * nx + v * ny;
        prim2cons(rho, u - 2.0 * vn * nx, v - 2.0 * vn * ny, p, g, Ug);
        break;
    }
    case BC_FARFIELD: {
        const double* d = bcd + bci * 8;
        double rho_inf = d[0], u_inf = d[1], v_inf = d[2], p_inf = d[3];
        double rho_i = fmax(Ui[0], 1e-10);
        double u_i = Ui[1] / rho_i, v_i = Ui[2] / rho_i;
        double p_i = fmax((g - 1.0) * (Ui[3] - 0.5 * rho_i * (u_i * u_i + v_i * v_i)), 1e-10);
        double vn_inf = u_inf * nx + v_inf * ny;
        double rb, ub, vb, pb;
        if (vn_inf > 0) { rb = rho_inf; ub = u_inf; vb = v_inf; pb = 0.5 * (p_inf + p_i); }
        else { rb = rho_i; ub = u_i; vb = v_i; pb = 0.5 * (p_inf + p_i); }
        rb = fmax(fmin(rb, 100.0), 0.01);
        ub = fmax(fmin(ub, 1000.0), -1000.0);
        vb = fmax(fmin(vb, 1000.0), -1000.0);
        pb = fmax(fmin(pb, 1e7), 1e3);
        prim2cons(rb, ub, vb, pb, g, Ug);
        break;
    }
    case BC_OUTFLOW: {
        double rho = Ui[0], u = Ui[1] / rho, v = Ui[2] / rho;
        prim2cons(rho, u, v, bcd[bci * 8], g, Ug);
        break;
    }
    default:
        Ug[0] = Ui[0]; Ug[1] = Ui[1]; Ug[2] = Ui[2]; Ug[3] = Ui[3];
    }
}

/* kernels.cu:597-669 (hard-coded Rusanov with floors; NaN/Inf -> 0) */
static void rusanov_compat(const double* UL, const double* UR, double nx, double ny,
                           double g, double* F) {
    double rhoL = fmax(UL[0], 1e-10), rhoR = fmax(UR[0], 1e-10);
    double uL = UL[1] / rhoL, vL = UL[2] / rhoL, uR = UR[1] / rhoR, vR = UR[2] / rhoR;
    double EL = UL[3] / rhoL, ER = UR[3] / rhoR;
    double pL = fmax((g - 1.0) * rhoL * (EL - 0.5 * (uL * uL + vL * vL)), 1e-10);
    double pR = fmax((g - 1.0) * rhoR * (ER - 0.5 * (uR * uR + vR * vR)), 1e-10);
    double cL = sqrt(fmax(g * pL / rhoL, 1e-10)), cR = sqrt(fmax(g * pR / rhoR, 1e-10));
    double vnL = uL * nx + vL * ny, vnR = uR * nx + vR * ny;
    double velL = sqrt(uL * uL + vL * vL), velR = sqrt(uR * uR + vR * vR);
    double smax = fmax(velL + cL, velR + cR);
    double HL = EL + pL / rhoL, HR = ER + pR / rhoR;
    double FL[4] = {rhoL * vnL, rhoL * uL * vnL + pL * nx, rhoL * vL * vnL + pL * ny, rhoL * HL * vnL};
    double FR[4] = {rhoR * vnR, rhoR * uR * vnR + pR * nx, rhoR * vR * vnR + pR * ny, rhoR * HR * vnR};
    for (int v = 0; v < 4; ++v) {
        F[v] = 0.5 * (FL[v] + FR[v]) - 0.5 * smax * (UR[v] - UL[v]);
        if (isnan(F[v]) || isinf(F[v])) F[v] = 0.0;
    }
}

/* ------------------------------------------------------------------- RHS -- */

void orc_rhs(orc_ctx* c, const double* U, double* R) {
    const int nsp = c->nsp, n1 = c->n1, nfp = c->nfp;
    const int64_t ne = c->n_elem, nf = c->n_faces;
    const double g = c->gamma;
    int nt = c->nthreads;
    (void)nt;
    /* K4 kernels.cu:157-194 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t idx = 0; idx < ne * nsp; ++idx)
        flux_xy(U + idx * 4, g, c->Fx + idx * 4, c->Fy + idx * 4);
    /* K1 kernels.cu:30-67 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t e = 0; e < ne; ++e)
        for (int t = 0; t < 4 * nfp; ++t) {
            int edge = t / nfp, fp = t % nfp;
            for (int v = 0; v < 4; ++v) {
                double val = 0.0;
                for (int sp = 0; sp < nsp; ++sp)
                    val += c->interp[edge * nfp * nsp + fp * nsp + sp] * U[e * nsp * 4 + sp * 4 + v];
                c->Ufp[(e * 4 + edge) * nfp * 4 + fp * 4 + v] = val;
            }
        }
    memset(c->Fdiff, 0, sizeof(double) * (size_t)ne * 4 * nfp * 4);
    /* K10 kernels.cu:528-701 then K8 kernels.cu:346-450 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t f = 0; f < nf; ++f) {
        int le = c->fle[f], ll = c->fll[f], re = c->fre[f], rl = c->frl[f];
        double nx = c->fn[2 * f], ny = c->fn[2 * f + 1];
        for (int fp = 0; fp < nfp; ++fp) {
            const double* UL = c->Ufp + ((int64_t)le * 4 + ll) * nfp * 4 + fp * 4;
            double UR[4];
            if (re >= 0) {
                const double* q = c->Ufp + ((int64_t)re * 4 + rl) * nfp * 4 + (nfp - 1 - fp) * 4;
                UR[0] = q[0]; UR[1] = q[1]; UR[2] = q[2]; UR[3] = q[3];
            } else {
                int bct = c->fbct[f], bci = c->fbcmap[f];
                if (bci < 0) { bct = BC_SLIPWALL; bci = 0; }
                ghost_state(UL, nx, ny, bct, c->bc_data, bci, g, UR);
            }
            rusanov_compat(UL, UR, nx, ny, g, c->Fcom + (f * nfp + fp) * 4);
        }
    }
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t f = 0; f < nf; ++f) {
        int le = c->fle[f], ll = c->fll[f], re = c->fre[f], rl = c->frl[f];
        double nx = c->fn[2 * f], ny = c->fn[2 * f + 1];
        for (int fp = 0; fp < nfp; ++fp) {
            const double* Fc = c->Fcom + (f * nfp + fp) * 4;
            int64_t lo = ((int64_t)le * 4 + ll) * nfp * 4 + fp * 4;
            double Fx[4], Fy[4];
            flux_xy(c->Ufp + lo, g, Fx, Fy);
            for (int v = 0; v < 4; ++v) c->Fdiff[lo + v] = Fc[v] - (Fx[v] * nx + Fy[v] * ny);
            if (re >= 0) {
                int64_t ro = ((int64_t)re * 4 + rl) * nfp * 4 + fp * 4;
                flux_xy(c->Ufp + ro, g, Fx, Fy);
                for (int v = 0; v < 4; ++v) c->Fdiff[ro + v] = -Fc[v] + (Fx[v] * nx + Fy[v] * ny);
            }
        }
    }
    /* K13 kernels.cu:813-872 then K15 kernels.cu:948-1034 */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t e = 0; e < ne; ++e)
        for (int sp = 0; sp < nsp; ++sp) {
            const double* Ji = c->Jinv + (e * nsp + sp) * 4;
            int si = sp / n1, sj = sp % n1;
            for (int v = 0; v < 4; ++v) {
                double a = 0.0, b = 0.0, cc = 0.0, d = 0.0;
                for (int k = 0; k < nsp; ++k) {
                    double fx = c->Fx[e * nsp * 4 + k * 4 + v], fy = c->Fy[e * nsp * 4 + k * 4 + v];
                    a += c->dxi[sp * nsp + k] * fx;
                    b += c->deta[sp * nsp + k] * fx;
                    cc += c->dxi[sp * nsp + k] * fy;
                    d += c->deta[sp * nsp + k] * fy;
                }
                double div = (a * Ji[0] + b * Ji[2]) + (cc * Ji[1] + d * Ji[3]);
                double r = -div;
                const double* Fd = c->Fdiff + e * 4 * nfp * 4;
                double corr = 0.0;
                corr += Fd[(0 * nfp + sj) * 4 + v] * c->corr[0 * nsp + sp];
                corr += Fd[(1 * nfp + si) * 4 + v] * c->corr[1 * nsp + sp];
                corr += Fd[(2 * nfp + sj) * 4 + v] * c->corr[2 * nsp + sp];
                corr += Fd[(3 * nfp + si) * 4 + v] * c->corr[3 * nsp + sp];
                r -= corr;
                R[e * nsp * 4 + sp * 4 + v] = r;
            }
        }
}

/* ------------------------------------------------------------ RK + clamp -- */

/* kernels.cu:1236-1288 */
static void positivity(double* U) {
    const double RHO_MIN = 0.01, RHO_MAX = 100.0, P_MIN = 100.0, P_MAX = 1e8;
    const double VEL_MAX = 2000.0, GPP = 1.4;
    double rho = U[0], rhou = U[1], rhov = U[2], rhoE = U[3];
    double rn = fmax(RHO_MIN, fmin(RHO_MAX, rho));
    double u = rhou / fmax(rn, 1e-10), v = rhov / fmax(rn, 1e-10);
    double vm = sqrt(u * u + v * v);
    if (vm > VEL_MAX) { double s = VEL_MAX / vm; u *= s; v *= s; }
    double ke = 0.5 * rn * (u * u + v * v);
    double p = (GPP - 1.0) * (rhoE - ke);
    p = fmax(P_MIN, fmin(P_MAX, p));
    double E = p / (GPP - 1.0) + ke;
    U[0] = rn; U[1] = rn * u; U[2] = rn * v; U[3] = E;
}

/* fr_solver.cpp:305-333 with kernels.cu:1297-1349 */
void orc_step(orc_ctx* c, double* U, double dt, int nsteps, double* R_last) {
    int64_t n = c->n_elem * c->nsp * 4, ns = c->n_elem * c->nsp;
    double* R = (double*)malloc(sizeof(double) * (size_t)n);
    int nt = c->nthreads;
    (void)nt;
    for (int s = 0; s < nsteps; ++s) {
        memcpy(c->U0, U, sizeof(double) * (size_t)n);
        orc_rhs(c, U, R);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < n; ++i) U[i] = c->U0[i] + dt * R[i];
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < ns; ++i) positivity(U + 4 * i);
        memcpy(c->U1, U, sizeof(double) * (size_t)n);
        orc_rhs(c, U, R);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < n; ++i) U[i] = 0.75 * c->U0[i] + 0.25 * c->U1[i] + 0.25 * dt * R[i];
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < ns; ++i) positivity(U + 4 * i);
        orc_rhs(c, U, R);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < n; ++i)
            U[i] = (1.0 / 3.0) * c->U0[i] + (2.0 / 3.0) * U[i] + (2.0 / 3.0) * dt * R[i];
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < ns; ++i) positivity(U + 4 * i);
    }
    if (R_last) memcpy(R_last, R, sizeof(double) * (size_t)n);
    free(R);
}

/* fr_solver.cpp:784-816 with euler.hpp:34-41,166-171 */
double orc_compute_dt(const orc_ctx* c, const double* U, double CFL) {
    double dt_min = 1e20;
    double cfl_factor = 2.0 * c->P + 1.0;
    for (int64_t e = 0; e < c->n_elem; ++e) {
        double h = sqrt(c->area[e]);
        for (int sp = 0; sp < c->nsp; ++sp) {
            const double* s = U + (e * c->nsp + sp) * 4;
            double u = s[1] / s[0], v = s[2] / s[0];
            double vel = sqrt(u * u + v * v);
            double p = fmax(pressure(s, c->gamma), 1e-10), rho = fmax(s[0], 1e-10);
            double ws = vel + sqrt(c->gamma * p / rho);
            double dl = CFL * h / (ws * cfl_factor);
            if (dl < dt_min) dt_min = dl;
        }
    }
    return dt_min;
}

double orc_l2(const double* R, int64_t n) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += R[i] * R[i];
    return sqrt(s);
}


/* ======================================================================= */
/* Physics mode: the conservative FR scheme the parameters ask for, restated  */
/* from the reference's formula sources (no reference residual exists):      */
/*   Riemann solvers      include/physics/euler.hpp:184-375                  */
/*   ghost states         include/bc/boundary_condition.hpp:42-311           */
/*   BC defaults          src/bc/boundary_condition.cpp:32-64                */
/*   VCJH corrections     Vincent, Castonguay & Jameson 2011 (README refs)   */
/* ======================================================================= */

static double pressure_raw(const double* U, double g) { return pressure(U, g); }

/* IdealGas::soundSpeed (euler.hpp:34-41) */
static double sound_speed(const double* U, double g) {
    double p = fmax(pressure_raw(U, g), 1e-10), rho = fmax(U[0], 1e-10);
    return sqrt(g * p / rho);
}

/* IdealGas::fluxNormal (euler.hpp:133-147) */
static void flux_normal_phys(const double* U, double nx, double ny, double g, double* Fn) {
    double rho = fmax(U[0], 1e-10);
    double u = U[1] / rho, v = U[2] / rho;
    double p = fmax(pressure_raw(U, g), 1e-10);
    double H = U[3] + pressure_raw(U, g);
    double vn = u * nx + v * ny;
    Fn[0] = rho * vn; Fn[1] = rho * u * vn + p * nx; Fn[2] = rho * v * vn + p * ny; Fn[3] = H * vn;
}

/* IdealGas::maxWaveSpeed (euler.hpp:166-171) */
static double max_wave_speed(const double* U, double g) {
    double u = U[1] / U[0], v = U[2] / U[0];
    return sqrt(u * u + v * v) + sound_speed(U, g);
}

/* RiemannSolvers::rusanov (euler.hpp:184-200) */
static void riemann_rusanov(const double* UL, const double* UR, double nx, double ny, double g, double* F) {
    double FL[4], FR[4];
    flux_normal_phys(UL, nx, ny, g, FL);
    flux_normal_phys(UR, nx, ny, g, FR);
    double smax = fmax(max_wave_speed(UL, g), max_wave_speed(UR, g));
    for (int i = 0; i < 4; ++i) F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * smax * (UR[i] - UL[i]);
}

/* RiemannSolvers::roe with Harten's entropy fix (euler.hpp:204-294) */
static void riemann_roe(const double* UL, const double* UR, double nx, double ny, double g, double* F) {
    double rhoL = fmax(UL[0], 1e-10), rhoR = fmax(UR[0], 1e-10);
    double uL = UL[1] / rhoL, vL = UL[2] / rhoL, uR = UR[1] / rhoR, vR = UR[2] / rhoR;
    double HL = (UL[3] + pressure_raw(UL, g)) / rhoL, HR = (UR[3] + pressure_raw(UR, g)) / rhoR;
    double sL = sqrt(rhoL), sR = sqrt(rhoR);
    double den = fmax(sL + sR, 1e-10);
    double rhoRoe = sL * sR;
    double uRoe = (sL * uL + sR * uR) / den, vRoe = (sL * vL + sR * vR) / den;
    double HRoe = (sL * HL + sR * HR) / den;
    double vnRoe = uRoe * nx + vRoe * ny, qsq = uRoe * uRoe + vRoe * vRoe;
    double c2 = fmax((g - 1.0) * (HRoe - 0.5 * qsq), 1e-10), cR = sqrt(c2);
    double l1 = fabs(vnRoe - cR), l2 = fabs(vnRoe), l3 = fabs(vnRoe), l4 = fabs(vnRoe + cR);
    double eps = 0.1 * cR;
    if (l1 < eps) l1 = (l1 * l1 + eps * eps) / (2.0 * eps);
    if (l4 < eps) l4 = (l4 * l4 + eps * eps) / (2.0 * eps);
    double drho = rhoR - rhoL, du = uR - uL, dv = vR - vL;
    double dp = pressure_raw(UR, g) - pressure_raw(UL, g);
    double dvn = du * nx + dv * ny;
    double cs = fmax(cR * cR, 1e-10);
    double a1 = (dp - rhoRoe * cR * dvn) / (2.0 * cs);
    double a2 = drho - dp / cs;
    double a3 = rhoRoe * (dv * nx - du * ny);
    double a4 = (dp + rhoRoe * cR * dvn) / (2.0 * cs);
    double FL[4], FR[4], dF[4];
    flux_normal_phys(UL, nx, ny, g, FL);
    flux_normal_phys(UR, nx, ny, g, FR);
    double tx = -ny, ty = nx;
    dF[0] = l1 * a1 * 1.0;
    dF[1] = l1 * a1 * (uRoe - cR * nx);
    dF[2] = l1 * a1 * (vRoe - cR * ny);
    dF[3] = l1 * a1 * (HRoe - cR * vnRoe);
    dF[0] += l2 * a2 * 1.0;
    dF[1] += l2 * a2 * uRoe;
    dF[2] += l2 * a2 * vRoe;
    dF[3] += l2 * a2 * 0.5 * qsq;
    dF[0] += l3 * a3 * 0.0;
    dF[1] += l3 * a3 * tx;
    dF[2] += l3 * a3 * ty;
    dF[3] += l3 * a3 * (uRoe * tx + vRoe * ty);
    dF[0] += l4 * a4 * 1.0;
    dF[1] += l4 * a4 * (uRoe + cR * nx);
    dF[2] += l4 * a4 * (vRoe + cR * ny);
    dF[3] += l4 * a4 * (HRoe + cR * vnRoe);
    for (int i = 0; i < 4; ++i) F[i] = 0.5 * (FL[i] + FR[i]) - 0.5 * dF[i];
}

static double clamp_away(double d) { return (fabs(d) < 1e-10) ? ((d >= 0) ? 1e-10 : -1e-10) : d; }

/* RiemannSolvers::hllc (euler.hpp:298-375) */
static void riemann_hllc(const double* UL, const double* UR, double nx, double ny, double g, double* F) {
    double rhoL = fmax(UL[0], 1e-10), rhoR = fmax(UR[0], 1e-10);
    double uL = UL[1] / rhoL, vL = UL[2] / rhoL, uR = UR[1] / rhoR, vR = UR[2] / rhoR;
    double pL = fmax(pressure_raw(UL, g), 1e-10), pR = fmax(pressure_raw(UR, g), 1e-10);
    double cL = sound_speed(UL, g), cR = sound_speed(UR, g);
    double vnL = uL * nx + vL * ny, vnR = uR * nx + vR * ny;
    double ps = 0.5 * (pL + pR) - 0.5 * (vnR - vnL) * 0.5 * (rhoL + rhoR) * 0.5 * (cL + cR);
    ps = fmax(ps, 1e-10);
    double qL = (ps <= pL) ? 1.0 : sqrt(1.0 + (g + 1.0) / (2.0 * g) * (ps / pL - 1.0));
    double qR = (ps <= pR) ? 1.0 : sqrt(1.0 + (g + 1.0) / (2.0 * g) * (ps / pR - 1.0));
    double SL = vnL - cL * qL, SR = vnR + cR * qR;
    double dSM = clamp_away(rhoL * (SL - vnL) - rhoR * (SR - vnR));
    double SM = (pR - pL + rhoL * vnL * (SL - vnL) - rhoR * vnR * (SR - vnR)) / dSM;
    if (SL >= 0.0) { flux_normal_phys(UL, nx, ny, g, F); return; }
    if (SR <= 0.0) { flux_normal_phys(UR, nx, ny, g, F); return; }
    const double *Uk; double rk, uk, vk, vnk, pk, Sk;
    if (SM >= 0.0) { Uk = UL; rk = rhoL; uk = uL; vk = vL; vnk = vnL; pk = pL; Sk = SL; }
    else { Uk = UR; rk = rhoR; uk = uR; vk = vR; vnk = vnR; pk = pR; Sk = SR; }
    double dK = clamp_away(Sk - SM);
    double dvn = clamp_away(Sk - vnk);
    double fac = rk * dvn / dK;
    double Us[4];
    Us[0] = fac;
    Us[1] = fac * (uk + (SM - vnk) * nx);
    Us[2] = fac * (vk + (SM - vnk) * ny);
    Us[3] = fac * (Uk[3] / rk + (SM - vnk) * (SM + pk / (rk * dvn)));
    double Fk[4];
    flux_normal_phys(Uk, nx, ny, g, Fk);
    for (int i = 0; i < 4; ++i) F[i] = Fk[i] + Sk * (Us[i] - Uk[i]);
}

void orc_riemann_point(int which, const double* UL, const double* UR, double nx, double ny,
                       double g, double* F) {
    if (which == 1) riemann_roe(UL, UR, nx, ny, g, F);
    else if (which == 2) riemann_hllc(UL, UR, nx, ny, g, F);
    else riemann_rusanov(UL, UR, nx, ny, g, F);
}

static int tag_slot(const orc_ctx* c, int tag) {
    int hit = -1;
    for (int t = 0; t < c->n_tags; ++t) if (c->tag_ids[t] == tag) hit = t;
    return hit;
}

/* BoundaryCondition::ghostState of each class (boundary_condition.hpp:42-311),
 * with the parameters createBCFromSpec gives them (boundary_condition.cpp:32-64). */
void orc_ghost_point(const orc_ctx* c, int bct, int tag, const double* Ui, double nx, double ny,
                     double* Ug) {
    const double g = c->gamma;
    int t = tag > 0 ? tag_slot(c, tag) : -1;
    switch (bct) {
    case BC_WALL: {
        double rho = Ui[0], u = Ui[1] / rho, v = Ui[2] / rho;
        double Tw = (t >= 0) ? c->tag_Tw[t] : 0.0;
        double p = (Tw > 0) ? rho * Tw : pressure_raw(Ui, g);
        prim2cons(rho, -u, -v, p, g, Ug);
        break;
    }
    case BC_SLIPWALL: case BC_SYMMETRY: {
        double rho = Ui[0], u = Ui[1] / rho, v = Ui[2] / rho, p = pressure_raw(Ui, g);
        double vn = u * nx + v * ny;
        prim2cons(rho, u - 2.0 * vn * nx, v - 2.0 * vn * ny, p, g, Ug);
        break;
    }
    case BC_FARFIELD: {
        double Uinf[4];
        prim2cons(c->rho_inf, c->u_inf, c->v_inf, c->p_inf, g, Uinf);
        double c_inf = sound_speed(Uinf, g);
        double rho_i = Ui[0], u_i = Ui[1] / rho_i, v_i = Ui[2] / rho_i;
        double p_i = pressure_raw(Ui, g), c_i = sound_speed(Ui, g);
        double vn_i = u_i * nx + v_i * ny, vn_inf = c->u_inf * nx + c->v_inf * ny;
        double Rp = vn_i + 2.0 * c_i / (g - 1.0), Rm = vn_inf - 2.0 * c_inf / (g - 1.0);
        double vn_b = 0.5 * (Rp + Rm), c_b = 0.25 * (g - 1.0) * (Rp - Rm);
        double rho_b, p_b, u_b, v_b;
        if (vn_b >= 0) {
            double vt = u_i * (-ny) + v_i * nx, s_i = p_i / pow(rho_i, g);
            rho_b = pow(c_b * c_b / (g * s_i), 1.0 / (g - 1.0));
            p_b = rho_b * c_b * c_b / g;
            u_b = vn_b * nx - vt * ny; v_b = vn_b * ny + vt * nx;
        } else {
            double vt = c->u_inf * (-ny) + c->v_inf * nx, s_inf = c->p_inf / pow(c->rho_inf, g);
            rho_b = pow(c_b * c_b / (g * s_inf), 1.0 / (g - 1.0));
            p_b = rho_b * c_b * c_b / g;
            u_b = vn_b * nx - vt * ny; v_b = vn_b * ny + vt * nx;
        }
        prim2cons(rho_b, u_b, v_b, p_b, g, Ug);
        break;
    }
    case BC_INFLOW: {
        double pt = (t >= 0 && c->tag_pt[t] > 0) ? c->tag_pt[t] : c->p_inf * 1.2;
        double Tt = (t >= 0 && c->tag_Tt[t] > 0) ? c->tag_Tt[t] : c->T_inf;
        double dx = (t >= 0) ? c->tag_dx[t] : 1.0, dy = (t >= 0) ? c->tag_dy[t] : 0.0;
        double mag = sqrt(dx * dx + dy * dy);
        dx /= mag; dy /= mag;
        double p_int = pressure_raw(Ui, g);
        double ratio = p_int / pt;
        double M2 = 2.0 / (g - 1.0) * (pow(ratio, -(g - 1.0) / g) - 1.0);
        M2 = fmax(M2, 0.0);
        double M = sqrt(M2);
        double T = Tt / (1.0 + 0.5 * (g - 1.0) * M2);
        double rho = p_int / T;
        double cc = sqrt(g * p_int / rho);
        double vel = M * cc;
        prim2cons(rho, vel * dx, vel * dy, p_int, g, Ug);
        break;
    }
    case BC_OUTFLOW: {
        double ps = (t >= 0 && c->tag_ps[t] > 0) ? c->tag_ps[t] : c->p_inf;
        double rho = Ui[0], u = Ui[1] / rho, v = Ui[2] / rho;
        prim2cons(rho, u, v, ps, g, Ug);
        break;
    }
    default:
        Ug[0] = Ui[0]; Ug[1] = Ui[1]; Ug[2] = Ui[2]; Ug[3] = Ui[3];
    }
}

/* VCJH g_L', g_R' at the solution points, from the reference's Legendre
 * derivative formula (basis.cpp:332-341) -- an independent evaluation of the
 * same functions the product builds with a recurrence. */
void orc_vcjh(int P, int flux_type, const double* x, double* gL, double* gR) {
    int p = P;
    double fp = 1.0, f2p = 1.0;
    for (int i = 2; i <= p; ++i) fp *= i;
    for (int i = 2; i <= 2 * p; ++i) f2p *= i;
    double ap = f2p / (pow(2.0, p) * fp);
    double ap2 = ap * ap, cc = 0.0;
    if (flux_type == 1) cc = 2.0 * p / ((2.0 * p + 1.0) * (p + 1.0) * ap2);
    else if (flux_type == 2) cc = 2.0 * (p + 1.0) / ((2.0 * p + 1.0) * p * ap2);
    else if (flux_type == 3) cc = 2.0 * (p + 1.0) * fp * fp / (f2p * (2.0 * p + 1.0));
    double eta = cc * (2.0 * p + 1.0) * ap2 / 2.0;
    for (int j = 0; j <= p; ++j) {
        double t = x[j];
        double dR = 0.5 * (legendre_deriv(p, t) + (eta * legendre_deriv(p - 1, t) + legendre_deriv(p + 1, t)) / (1.0 + eta));
        double tn = -t;
        double dRm = 0.5 * (legendre_deriv(p, tn) + (eta * legendre_deriv(p - 1, tn) + legendre_deriv(p + 1, tn)) / (1.0 + eta));
        gR[j] = dR;
        gL[j] = -dRm;
    }
}

void orc_set_physics(orc_ctx* c, int flux_type, int riemann, int viscous, double Re, double Pr,
                     double T_inf) {
    c->flux_type = flux_type; c->riemann = riemann; c->viscous = viscous;
    c->Re = Re; c->Pr = Pr; c->T_inf = T_inf;
    orc_vcjh(c->P, flux_type, c->pts, c->gLp, c->gRp);
}

void orc_set_bc_extra(orc_ctx* c, int n, const int* ids, const double* pt, const double* Tt,
                      const double* dx, const double* dy, const double* Tw) {
    for (int k = 0; k < n; ++k) {
        int t = tag_slot(c, ids[k]);
        if (t < 0) continue;
        c->tag_pt[t] = pt[k]; c->tag_Tt[t] = Tt[k]; c->tag_dx[t] = dx[k]; c->tag_dy[t] = dy[k];
        c->tag_Tw[t] = Tw[k];
    }
}

void orc_get_vcjh(const orc_ctx* c, double* gL, double* gR) {
    for (int j = 0; j < c->n1; ++j) { gL[j] = c->gLp[j]; gR[j] = c->gRp[j]; }
}

/* Viscous flux at one state with conservative gradients dx, dy: velocity
 * and temperature gradients from the conservative ones
 * (ViscousFlux::velocityGradients / temperatureGradient, navierstokes.hpp:
 * 115-158, the same formulas as computeViscousFluxSPKernel,
 * kernels.cu:742-760), Stokes stresses (navierstokes.hpp:36-46), and one of
 * the reference's two viscosity laws:
 *   law 0: the kernel's mu = T^0.7/Re, k = mu gamma/((gamma-1) Pr)
 *          (kernels.cu:762-764) -- the law of every residual here;
 *   law 1: the header's Sutherland law mu = (T^1.5 (1+S)/(T+S))/Re,
 *          S = 110.4, and k = (mu cp/Pr)/Re (ViscousFlux::fluxX,
 *          navierstokes.hpp:17-33, 52-96), kept for its pointwise pin. */
void orc_viscous_flux_law(int law, const double* s, const double* dx, const double* dy, double g,
                          double Re, double Pr, double* Fv, double* Gv) {
    double rho = s[0], u = s[1] / rho, v = s[2] / rho;
    double dudx = (dx[1] - u * dx[0]) / rho, dudy = (dy[1] - u * dy[0]) / rho;
    double dvdx = (dx[2] - v * dx[0]) / rho, dvdy = (dy[2] - v * dy[0]) / rho;
    double p = pressure_raw(s, g), T = p / rho;
    double dpdx = (g - 1.0) * (dx[3] - 0.5 * dx[0] * (u * u + v * v) - rho * (u * dudx + v * dvdx));
    double dpdy = (g - 1.0) * (dy[3] - 0.5 * dy[0] * (u * u + v * v) - rho * (u * dudy + v * dvdy));
    double dTdx = (dpdx - T * dx[0]) / rho, dTdy = (dpdy - T * dy[0]) / rho;
    double mu, k;
    if (law == 1) {
        const double S = 110.4 / 1.0, Tn = T / 1.0;
        mu = 1.0 * pow(Tn, 1.5) * (1.0 + S) / (Tn + S) / Re;
        const double cp = g / (g - 1.0);
        k = mu * cp / Pr / Re;
    } else {
        mu = pow(T, 0.7) / Re;
        k = mu * g / ((g - 1.0) * Pr);
    }
    double div = dudx + dvdy, lam = -2.0 / 3.0 * mu;
    double txx = 2.0 * mu * dudx + lam * div, tyy = 2.0 * mu * dvdy + lam * div;
    double txy = mu * (dudy + dvdx);
    Fv[0] = 0.0; Fv[1] = txx; Fv[2] = txy; Fv[3] = u * txx + v * txy + k * dTdx;
    Gv[0] = 0.0; Gv[1] = txy; Gv[2] = tyy; Gv[3] = u * txy + v * tyy + k * dTdy;
}

/* The kernel law (law 0), the viscous flux of every residual here. */
void orc_viscous_flux(const double* s, const double* dx, const double* dy, double g, double Re,
                      double Pr, double* Fv, double* Gv) {
    orc_viscous_flux_law(0, s, dx, dy, g, Re, Pr, Fv, Gv);
}

/* Common normal viscous flux of a face point (BR2Scheme::commonFlux,
 * navierstokes.hpp:166-201): average state and average gradients, the
 * viscous flux there, dotted with the normal. */
void orc_common_viscous_law(int law, const double* UL, const double* UR, const double* dxL,
                            const double* dyL, const double* dxR, const double* dyR, double nx,
                            double ny, double g, double Re, double Pr, double* Fvn) {
    double Ua[4], dxa[4], dya[4], Fv[4], Gv[4];
    for (int v = 0; v < 4; ++v) {
        Ua[v] = 0.5 * (UL[v] + UR[v]);
        dxa[v] = 0.5 * (dxL[v] + dxR[v]);
        dya[v] = 0.5 * (dyL[v] + dyR[v]);
    }
    orc_viscous_flux_law(law, Ua, dxa, dya, g, Re, Pr, Fv, Gv);
    for (int v = 0; v < 4; ++v) Fvn[v] = Fv[v] * nx + Gv[v] * ny;
}

/* Neumann data of the walls on the common normal viscous flux Fvn of a
 * boundary face (the conditions the wall classes state,
 * boundary_condition.hpp:60-67 and 146-155): slip and symmetry walls carry
 * no shear stress and no heat flux (Fvn keeps tau_nn n), an adiabatic
 * no-slip wall (T_wall = 0) no heat flux. */
void orc_wall_viscous_closure(const orc_ctx* c, int bct, int tag, double nx, double ny, double* Fvn) {
    if (bct == BC_SLIPWALL || bct == BC_SYMMETRY) {
        double tnn = Fvn[1] * nx + Fvn[2] * ny;
        Fvn[1] = tnn * nx;
        Fvn[2] = tnn * ny;
        Fvn[3] = 0.0;
    } else if (bct == BC_WALL) {
        int t = tag > 0 ? tag_slot(c, tag) : -1;
        double Tw = (t >= 0) ? c->tag_Tw[t] : 0.0;
        if (!(Tw > 0)) Fvn[3] = 0.0;
    }
}

/* Curved elements (geometric order 2 or 4) in physics mode: the unit normal
 * and the edge Jacobian s = |dx/dt| at every point of every face, from the
 * face's left element's mapping (basis.cpp:717-847 shape functions).  The
 * left element's edge ll runs counter-clockwise with t the 1-D flux points:
 * (t,-1), (1,t), (-t,1), (-1,-t) for edges 0..3; the outward normal is the
 * tangent turned clockwise.  On a straight edge s = length/2 and n is the
 * face normal. */
static void build_face_point_normals(orc_ctx* c) {
    const int nfp = c->nfp;
    c->fpn = (double*)malloc(sizeof(double) * (size_t)c->n_faces * nfp * 3);
    for (int64_t f = 0; f < c->n_faces; ++f) {
        const int le = c->fle[f], ll = c->fll[f];
        const int64_t* nd = c->conn + (int64_t)le * c->nn;
        for (int fp = 0; fp < nfp; ++fp) {
            const double t = c->pts[fp];
            double xi, eta, dxi, deta;
            if (ll == 0) { xi = t; eta = -1.0; dxi = 1.0; deta = 0.0; }
            else if (ll == 1) { xi = 1.0; eta = t; dxi = 0.0; deta = 1.0; }
            else if (ll == 2) { xi = -t; eta = 1.0; dxi = -1.0; deta = 0.0; }
            else { xi = -1.0; eta = -t; dxi = 0.0; deta = -1.0; }
            double N[25], dNx[25], dNe[25];
            const int n = shape_quad(c->eorder, xi, eta, N, dNx, dNe);
            double tx = 0.0, ty = 0.0;
            for (int i = 0; i < n; ++i) {
                const double w = dNx[i] * dxi + dNe[i] * deta;
                tx += w * c->xy[2 * nd[i]];
                ty += w * c->xy[2 * nd[i] + 1];
            }
            const double len = sqrt(tx * tx + ty * ty);
            double* q = c->fpn + ((size_t)f * nfp + fp) * 3;
            q[0] = ty / len; q[1] = -tx / len; q[2] = len;
        }
    }
}

/* (nx, ny, s) of point fp of face f: per point on curved meshes, else the
 * face's normal and half its length. */
static void face_point(const orc_ctx* c, int64_t f, int fp, double* nx, double* ny, double* s) {
    if (c->fpn) {
        const double* q = c->fpn + ((size_t)f * c->nfp + fp) * 3;
        *nx = q[0]; *ny = q[1]; *s = q[2];
    } else {
        *nx = c->fn[2 * f]; *ny = c->fn[2 * f + 1]; *s = 0.5 * c->flen[f];
    }
}

void orc_rhs_phys(orc_ctx* c, const double* U, double* R) {
    const int nsp = c->nsp, n1 = c->n1, nfp = c->nfp;
    const int64_t ne = c->n_elem, nf = c->n_faces;
    const double g = c->gamma;
    int nt = c->nthreads;
    (void)nt;
    size_t fpn = (size_t)ne * 4 * nfp * 4;
    double* Ft = c->Fx; double* Gt = c->Fy;          /* transformed fluxes at sp */
    double* FnD = (double*)malloc(sizeof(double) * fpn);
    if (c->eorder > 1 && !c->fpn) build_face_point_normals(c);
    /* traces of the state (dense interp) */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t e = 0; e < ne; ++e)
        for (int t = 0; t < 4 * nfp; ++t) {
            const double* w = c->interp + t * nsp;
            for (int v = 0; v < 4; ++v) {
                double su = 0.0;
                for (int sp = 0; sp < nsp; ++sp) su += w[sp] * U[(e * nsp + sp) * 4 + v];
                c->Ufp[((e * 4) * nfp + t) * 4 + v] = su;
            }
        }
    /* Navier-Stokes: corrected gradient with the common solution
     * U_c = (U_L + U_R)/2 at every face point (ghost state on boundaries),
     * Q = grad U at the solution points, and its traces. */
    double *Q = NULL, *Qfp = NULL;
    if (c->viscous) {
        double* dU = (double*)calloc(fpn, sizeof(double));
        Q = (double*)malloc(sizeof(double) * (size_t)ne * nsp * 8);
        Qfp = (double*)malloc(sizeof(double) * fpn * 2);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t f = 0; f < nf; ++f) {
            int le = c->fle[f], ll = c->fll[f], re = c->fre[f], rl = c->frl[f];
            for (int fp = 0; fp < nfp; ++fp) {
                double nx, ny, s;
                face_point(c, f, fp, &nx, &ny, &s);
                (void)s;
                int64_t lo = (((int64_t)le * 4 + ll) * nfp + fp) * 4;
                const double* UL = c->Ufp + lo;
                double UR[4];
                int64_t ro = -1;
                if (re >= 0) {
                    ro = (((int64_t)re * 4 + rl) * nfp + (nfp - 1 - fp)) * 4;
                    for (int v = 0; v < 4; ++v) UR[v] = c->Ufp[ro + v];
                } else {
                    orc_ghost_point(c, c->fbct[f], c->ftag[f], UL, nx, ny, UR);
                }
                for (int v = 0; v < 4; ++v) {
                    double uc = 0.5 * (UL[v] + UR[v]);
                    dU[lo + v] = uc - UL[v];
                    if (ro >= 0) dU[ro + v] = uc - UR[v];
                }
            }
        }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t e = 0; e < ne; ++e)
            for (int sp = 0; sp < nsp; ++sp) {
                int i = sp % n1, j = sp / n1;
                const double* D = dU + e * 4 * nfp * 4;
                const double* Ji = c->Jinv + (e * nsp + sp) * 4;
                for (int v = 0; v < 4; ++v) {
                    double dxi = 0.0, deta = 0.0;
                    for (int k = 0; k < nsp; ++k) {
                        dxi += c->dxi[sp * nsp + k] * U[(e * nsp + k) * 4 + v];
                        deta += c->deta[sp * nsp + k] * U[(e * nsp + k) * 4 + v];
                    }
                    dxi += c->gRp[i] * D[(1 * nfp + j) * 4 + v] + c->gLp[i] * D[(3 * nfp + (nfp - 1 - j)) * 4 + v];
                    deta += c->gLp[j] * D[(0 * nfp + i) * 4 + v] + c->gRp[j] * D[(2 * nfp + (nfp - 1 - i)) * 4 + v];
                    Q[(e * nsp + sp) * 8 + v] = Ji[0] * dxi + Ji[2] * deta;
                    Q[(e * nsp + sp) * 8 + 4 + v] = Ji[1] * dxi + Ji[3] * deta;
                }
            }
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t e = 0; e < ne; ++e)
            for (int t = 0; t < 4 * nfp; ++t) {
                const double* w = c->interp + t * nsp;
                for (int v = 0; v < 8; ++v) {
                    double sq = 0.0;
                    for (int sp = 0; sp < nsp; ++sp) sq += w[sp] * Q[(e * nsp + sp) * 8 + v];
                    Qfp[((e * 4) * nfp + t) * 8 + v] = sq;
                }
            }
        free(dU);
    }
    /* transformed total fluxes F~ = J (xi_x (F - Fv) + xi_y (G - Gv)), G~ likewise */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t idx = 0; idx < ne * nsp; ++idx) {
        double F[4], G[4];
        flux_xy(U + idx * 4, g, F, G);
        if (c->viscous) {
            double Fv[4], Gv[4];
            orc_viscous_flux(U + idx * 4, Q + idx * 8, Q + idx * 8 + 4, g, c->Re, c->Pr, Fv, Gv);
            for (int v = 0; v < 4; ++v) { F[v] -= Fv[v]; G[v] -= Gv[v]; }
        }
        const double* Ji = c->Jinv + idx * 4;
        double J = c->J[idx];
        for (int v = 0; v < 4; ++v) {
            Ft[idx * 4 + v] = J * (Ji[0] * F[v] + Ji[1] * G[v]);
            Gt[idx * 4 + v] = J * (Ji[2] * F[v] + Ji[3] * G[v]);
        }
    }
    /* outward reference-normal extrapolated transformed flux, dense interp */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t e = 0; e < ne; ++e)
        for (int t = 0; t < 4 * nfp; ++t) {
            int edge = t / nfp;
            const double* w = c->interp + t * nsp;
            for (int v = 0; v < 4; ++v) {
                double sf = 0.0, sg = 0.0;
                for (int sp = 0; sp < nsp; ++sp) {
                    sf += w[sp] * Ft[(e * nsp + sp) * 4 + v];
                    sg += w[sp] * Gt[(e * nsp + sp) * 4 + v];
                }
                FnD[((e * 4) * nfp + t) * 4 + v] = (edge == 0) ? -sg : (edge == 1) ? sf : (edge == 2) ? sg : -sf;
            }
        }
    memset(c->Fdiff, 0, sizeof(double) * fpn);
    /* common fluxes, computed once per face from the left side's view */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t f = 0; f < nf; ++f) {
        int le = c->fle[f], ll = c->fll[f], re = c->fre[f], rl = c->frl[f];
        for (int fp = 0; fp < nfp; ++fp) {
            double nx, ny, s;
            face_point(c, f, fp, &nx, &ny, &s);
            int64_t lo = (((int64_t)le * 4 + ll) * nfp + fp) * 4;
            const double* UL = c->Ufp + lo;
            double UR[4], Fc[4];
            int64_t ro = -1;
            if (re >= 0) {
                ro = (((int64_t)re * 4 + rl) * nfp + (nfp - 1 - fp)) * 4;
                for (int v = 0; v < 4; ++v) UR[v] = c->Ufp[ro + v];
            } else {
                orc_ghost_point(c, c->fbct[f], c->ftag[f], UL, nx, ny, UR);
            }
            orc_riemann_point(c->riemann, UL, UR, nx, ny, g, Fc);
            if (c->viscous) {
                /* BR2Scheme::commonFlux (navierstokes.hpp:177-204): average state
                 * and gradients; boundaries copy the interior gradient
                 * (BoundaryCondition::ghostGradient), walls impose their
                 * Neumann data */
                const double* QL = Qfp + (lo / 4) * 8;
                const double* QR = (ro >= 0) ? Qfp + (ro / 4) * 8 : QL;
                double Fvn[4];
                orc_common_viscous_law(0, UL, UR, QL, QL + 4, QR, QR + 4, nx, ny, g, c->Re, c->Pr, Fvn);
                if (re < 0) orc_wall_viscous_closure(c, c->fbct[f], c->ftag[f], nx, ny, Fvn);
                for (int v = 0; v < 4; ++v) Fc[v] -= Fvn[v];
            }
            for (int v = 0; v < 4; ++v) c->Fdiff[lo + v] = s * Fc[v] - FnD[lo + v];
            if (ro >= 0)
                for (int v = 0; v < 4; ++v) c->Fdiff[ro + v] = s * (-Fc[v]) - FnD[ro + v];
        }
    }
    /* divergence + VCJH correction, divided by J */
#pragma omp parallel for num_threads(nt) schedule(static)
    for (int64_t e = 0; e < ne; ++e)
        for (int sp = 0; sp < nsp; ++sp) {
            int i = sp % n1, j = sp / n1;
            const double* D = c->Fdiff + e * 4 * nfp * 4;
            for (int v = 0; v < 4; ++v) {
                double div = 0.0;
                for (int k = 0; k < nsp; ++k)
                    div += c->dxi[sp * nsp + k] * Ft[(e * nsp + k) * 4 + v] +
                           c->deta[sp * nsp + k] * Gt[(e * nsp + k) * 4 + v];
                double corr = c->gRp[i] * D[(1 * nfp + j) * 4 + v] - c->gLp[i] * D[(3 * nfp + (nfp - 1 - j)) * 4 + v] +
                              c->gRp[j] * D[(2 * nfp + (nfp - 1 - i)) * 4 + v] - c->gLp[j] * D[(0 * nfp + i) * 4 + v];
                R[(e * nsp + sp) * 4 + v] = -(div + corr) / c->J[e * nsp + sp];
            }
        }
    free(FnD);
    free(Q);
    free(Qfp);
}

void orc_step_phys(orc_ctx* c, double* U, double dt, int nsteps, double* R_last) {
    int64_t n = c->n_elem * c->nsp * 4;
    double* R = (double*)malloc(sizeof(double) * (size_t)n);
    int nt = c->nthreads;
    (void)nt;
    for (int st = 0; st < nsteps; ++st) {
        memcpy(c->U0, U, sizeof(double) * (size_t)n);
        orc_rhs_phys(c, U, R);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < n; ++i) U[i] = c->U0[i] + dt * R[i];
        memcpy(c->U1, U, sizeof(double) * (size_t)n);
        orc_rhs_phys(c, U, R);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < n; ++i) U[i] = 0.75 * c->U0[i] + 0.25 * c->U1[i] + 0.25 * dt * R[i];
        orc_rhs_phys(c, U, R);
#pragma omp parallel for num_threads(nt) schedule(static)
        for (int64_t i = 0; i < n; ++i)
            U[i] = (1.0 / 3.0) * c->U0[i] + (2.0 / 3.0) * U[i] + (2.0 / 3.0) * dt * R[i];
    }
    if (R_last) memcpy(R_last, R, sizeof(double) * (size_t)n);
    free(R);
}
