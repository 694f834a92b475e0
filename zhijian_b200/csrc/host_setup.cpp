// host_setup.cpp -- one-time host work of zj_solver_create: 1D operators,
// face topology, normals, metric terms, boundary data and config parsing.
// Compiled with -ffp-contract=off so the metric terms and normals round
// exactly like the reference host code they must reproduce.
#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>
#include <string>

#include "zj_internal.h"

namespace zj {

// ---------------------------------------------------------------------------
// Gauss-Legendre nodes.  Orders up to 5 use the same closed forms as the
// reference and 6 points use its 15-digit table (src/basis/basis.cpp:12-67),
// because reference parity at P5 depends on those exact values; beyond that a
// Newton iteration on the Legendre recurrence.
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
    x.assign(n, 0.0);
    w.assign(n, 0.0);
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; return; }
    if (n == 2) { x[0] = -1.0 / std::sqrt(3.0); x[1] = 1.0 / std::sqrt(3.0); w[0] = w[1] = 1.0; return; }
    if (n == 3) {
        x[0] = -std::sqrt(3.0 / 5.0); x[1] = 0.0; x[2] = std::sqrt(3.0 / 5.0);
        w[0] = w[2] = 5.0 / 9.0; w[1] = 8.0 / 9.0; return;
    }
    if (n == 4) {
        const double a = std::sqrt(3.0 / 7.0 + 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
        const double b = std::sqrt(3.0 / 7.0 - 2.0 / 7.0 * std::sqrt(6.0 / 5.0));
        x[0] = -a; x[1] = -b; x[2] = b; x[3] = a;
        w[0] = w[3] = (18.0 - std::sqrt(30.0)) / 36.0;
        w[1] = w[2] = (18.0 + std::sqrt(30.0)) / 36.0; return;
    }
    if (n == 5) {
        const double a = std::sqrt(5.0 + 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
        const double b = std::sqrt(5.0 - 2.0 * std::sqrt(10.0 / 7.0)) / 3.0;
        x[0] = -a; x[1] = -b; x[2] = 0.0; x[3] = b; x[4] = a;
        w[0] = w[4] = (322.0 - 13.0 * std::sqrt(70.0)) / 900.0;
        w[1] = w[3] = (322.0 + 13.0 * std::sqrt(70.0)) / 900.0;
        w[2] = 128.0 / 225.0; return;
    }
    if (n == 6) {
        static const double t[3] = {0.932469514203152, 0.661209386466265, 0.238619186083197};
        static const double tw[3] = {0.171324492379170, 0.360761573048139, 0.467913934572691};
        for (int i = 0; i < 3; ++i) {
            x[i] = -t[i]; x[5 - i] = t[i]; w[i] = w[5 - i] = tw[i];
        }
        return;
    }
    for (int i = 0; i < n; ++i) {
        double r = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double P0 = 1.0, P1 = r;
        for (int it = 0; it < 100; ++it) {
            P0 = 1.0; P1 = r;
            for (int j = 2; j <= n; ++j) { double Pn = ((2 * j - 1) * r * P1 - (j - 1) * P0) / j; P0 = P1; P1 = Pn; }
            double dP = n * (r * P1 - P0) / (r * r - 1.0);
            double dx = P1 / dP;
            r -= dx;
            if (std::fabs(dx) < 1e-16) break;
        }
        P0 = 1.0; P1 = r;
        for (int j = 2; j <= n; ++j) { double Pn = ((2 * j - 1) * r * P1 - (j - 1) * P0) / j; P0 = P1; P1 = Pn; }
        double dP = n * (r * P1 - P0) / (r * r - 1.0);
        x[i] = r;
        w[i] = 2.0 / ((1.0 - r * r) * dP * dP);
    }
}

// Lagrange cardinal function and derivative on arbitrary nodes, in the
// product order of src/basis/basis.cpp:169-196 (the compat residual's trace
// weights and derivative matrix must round identically).
double lagrange_eval(const std::vector<double>& nodes, int j, double x) {
    double r = 1.0;
    for (size_t i = 0; i < nodes.size(); ++i)
        if ((int)i != j) r *= (x - nodes[i]) / (nodes[j] - nodes[i]);
    return r;
}

double lagrange_deriv(const std::vector<double>& nodes, int j, double x) {
    double r = 0.0;
    const int n = (int)nodes.size();
    for (int k = 0; k < n; ++k) {
        if (k == j) continue;
        double term = 1.0 / (nodes[j] - nodes[k]);
        for (int i = 0; i < n; ++i)
            if (i != j && i != k) term *= (x - nodes[i]) / (nodes[j] - nodes[i]);
        r += term;
    }
    return r;
}

namespace {

double legendre(int n, double x) {
    if (n == 0) return 1.0;
    if (n == 1) return x;
    double P0 = 1.0, P1 = x;
    for (int i = 2; i <= n; ++i) { double Pn = ((2 * i - 1) * x * P1 - (i - 1) * P0) / i; P0 = P1; P1 = Pn; }
    return P1;
}

// The reference's P_n'(x) = n (x P_n - P_{n-1}) / (x^2 - 1) away from the
// end points (basis.cpp:332-341); solution points never sit on them.
double legendre_deriv_compat(int n, double x) {
    if (n == 0) return 0.0;
    double Pn = legendre(n, x), Pn1 = legendre(n - 1, x);
    if (std::fabs(x * x - 1.0) < 1e-14)
        return n * (n + 1) / 2.0 * ((x > 0) ? 1.0 : ((n % 2 == 0) ? 1.0 : -1.0));
    return n / (x * x - 1.0) * (x * Pn - Pn1);
}

// P_n'(x) from the recurrence P_{n+1}' = P_{n-1}' + (2n+1) P_n, valid on
// the whole interval.
double legendre_deriv(int n, double x) {
    if (n == 0) return 0.0;
    double dm1 = 0.0, d0 = 1.0;        // P_0', P_1'
    double Pm1 = 1.0, P0 = x;          // P_0, P_1
    for (int k = 1; k < n; ++k) {
        double d1 = dm1 + (2 * k + 1) * P0;
        double P1 = ((2 * k + 1) * x * P0 - k * Pm1) / (k + 1);
        dm1 = d0; d0 = d1; Pm1 = P0; P0 = P1;
    }
    return d0;
}

double factorial(int n) { double f = 1.0; for (int i = 2; i <= n; ++i) f *= i; return f; }

}  // namespace

static void fill_common(int P, Operators1D& ops) {
    ops.P = P;
    ops.n1 = P + 1;
    gauss_legendre(P + 1, ops.pts, ops.wts);
    const int n1 = ops.n1;
    ops.D1.assign(n1 * n1, 0.0);
    for (int i = 0; i < n1; ++i)
        for (int k = 0; k < n1; ++k) ops.D1[i * n1 + k] = lagrange_deriv(ops.pts, k, ops.pts[i]);
    ops.Lm.assign(n1, 0.0);
    ops.Lp.assign(n1, 0.0);
    for (int j = 0; j < n1; ++j) {
        ops.Lm[j] = lagrange_eval(ops.pts, j, -1.0);
        ops.Lp[j] = lagrange_eval(ops.pts, j, 1.0);
    }
}

void build_operators_compat(int P, Operators1D& ops) {
    fill_common(P, ops);
    const int n1 = ops.n1;
    ops.gL.assign(n1, 0.0);
    ops.gR.assign(n1, 0.0);
    const double sign = (P % 2 == 0) ? 1.0 : -1.0;
    for (int j = 0; j < n1; ++j) {
        double x = ops.pts[j];
        double dPp = legendre_deriv_compat(P, x), dPp1 = legendre_deriv_compat(P + 1, x);
        ops.gL[j] = sign * 0.5 * (dPp - dPp1);           // basis.cpp:343-347
        ops.gR[j] = 0.5 * (dPp + dPp1);                  // basis.cpp:375-378
    }
}

// VCJH correction derivatives (Vincent, Castonguay & Jameson 2011):
//   g_R = 1/2 [P_p + (eta P_{p-1} + P_{p+1}) / (1 + eta)],  g_L(x) = g_R(-x),
//   eta = c (2p+1) (a_p p!)^2 / 2,  a_p = (2p)! / (2^p (p!)^2).
// c: DG 0; SD c_SD = 2p / ((2p+1)(p+1)(a_p p!)^2); HU (Huynh g2)
// c_HU = 2(p+1) / ((2p+1) p (a_p p!)^2); GA the reference's "Gauss" value
// 2(p+1)(p!)^2 / ((2p)! (2p+1)) (src/basis/basis.cpp:250-256).
void build_operators_vcjh(int P, int flux_type, Operators1D& ops) {
    fill_common(P, ops);
    const int n1 = ops.n1, p = P;
    const double fp = factorial(p), f2p = factorial(2 * p);
    const double ap_pf = f2p / (std::pow(2.0, p) * fp);   // a_p p!
    const double ap2 = ap_pf * ap_pf;
    double c = 0.0;
    switch (flux_type) {
        case ZJ_FLUX_DG: c = 0.0; break;
        case ZJ_FLUX_SD: c = 2.0 * p / ((2.0 * p + 1.0) * (p + 1.0) * ap2); break;
        case ZJ_FLUX_HU: c = 2.0 * (p + 1.0) / ((2.0 * p + 1.0) * p * ap2); break;
        case ZJ_FLUX_GA: c = 2.0 * (p + 1.0) * fp * fp / (f2p * (2.0 * p + 1.0)); break;
        default: c = 0.0;
    }
    const double eta = c * (2.0 * p + 1.0) * ap2 / 2.0;
    ops.gL.assign(n1, 0.0);
    ops.gR.assign(n1, 0.0);
    for (int j = 0; j < n1; ++j) {
        const double x = ops.pts[j];
        auto dgR = [&](double t) {
            double dPm = (p >= 1) ? legendre_deriv(p - 1, t) : 0.0;
            return 0.5 * (legendre_deriv(p, t) + (eta * dPm + legendre_deriv(p + 1, t)) / (1.0 + eta));
        };
        ops.gR[j] = dgR(x);
        ops.gL[j] = -dgR(-x);   // g_L(x) = g_R(-x)  =>  g_L'(x) = -g_R'(-x)
    }
}

// ---------------------------------------------------------------------------
// Mesh topology.

namespace {

struct EdgeKey {
    int64_t a, b, seq;
    int32_t e, l;
};
bool key_less(const EdgeKey& p, const EdgeKey& q) {
    if (p.a != q.a) return p.a < q.a;
    if (p.b != q.b) return p.b < q.b;
    return p.seq < q.seq;
}

const zj_bc_spec* find_bc(const zj_params* p, int tag) {
    if (!p) return nullptr;
    const zj_bc_spec* hit = nullptr;
    for (int i = 0; i < p->n_bc && i < ZJ_MAX_BC; ++i)
        if (p->bc[i].tag == tag) hit = &p->bc[i];
    return hit;
}

// mesh.cpp:159-183
void face_normal(const HostMesh& m, int e, int lf, double& nx, double& ny, double& len) {
    const int64_t* nd = &m.conn[(size_t)e * m.nn];
    const int nve = m.nv(e);
    const double* v0 = &m.xy[2 * nd[lf]];
    const double* v1 = &m.xy[2 * nd[(lf + 1) % nve]];
    double tx = v1[0] - v0[0], ty = v1[1] - v0[1];
    len = std::sqrt(tx * tx + ty * ty);
    nx = ty / len;
    ny = -tx / len;
    double cx = 0.0, cy = 0.0;
    for (int i = 0; i < nve; ++i) { cx = cx + m.xy[2 * nd[i]]; cy = cy + m.xy[2 * nd[i] + 1]; }
    cx = cx / (double)nve;
    cy = cy / (double)nve;
    double fx = (v0[0] + v1[0]) * 0.5, fy = (v0[1] + v1[1]) * 0.5;
    if (nx * (fx - cx) + ny * (fy - cy) < 0) { nx = nx * (-1.0); ny = ny * (-1.0); }
}

}  // namespace

bool build_mesh(const zj_mesh_desc* d, const zj_params* p, HostMesh& m, std::string& msg) {
    if (!d || d->n_nodes <= 0 || d->n_elem <= 0 || !d->xy || !d->conn || !d->conn_offsets) {
        msg = "mesh descriptor: empty mesh or null array";
        return false;
    }
    m.n_nodes = d->n_nodes;
    m.n_elem = d->n_elem;
    int order = d->elem_order ? d->elem_order[0] : 1;
    int nn = (order == 1) ? 4 : (order == 2) ? 9 : (order == 4) ? 25 : -1;
    if (nn < 0) { msg = "element order must be 1, 2 or 4"; return false; }
    m.etype.assign((size_t)d->n_elem, (int8_t)ZJ_ELEM_QUAD);
    m.n_tri = 0;
    for (int64_t e = 0; e < d->n_elem; ++e) {
        const bool tri = d->elem_type && d->elem_type[e] == ZJ_ELEM_TRI;
        if (d->elem_type && d->elem_type[e] != ZJ_ELEM_TRI && d->elem_type[e] != ZJ_ELEM_QUAD) {
            msg = "element " + std::to_string(e) + " has an unknown type";
            return false;
        }
        if (d->elem_order && d->elem_order[e] != order) {
            msg = "mixed geometric orders are not supported";
            return false;
        }
        if (tri && order != 1) {
            msg = "element " + std::to_string(e) + " is a curved triangle: only straight-sided triangles are supported";
            return false;
        }
        if (d->conn_offsets[e + 1] - d->conn_offsets[e] != (tri ? 3 : nn)) {
            msg = "element " + std::to_string(e) + " has a node count that does not match its order";
            return false;
        }
        if (tri) { m.etype[(size_t)e] = (int8_t)ZJ_ELEM_TRI; ++m.n_tri; }
    }
    m.nn = nn;
    m.order = order;
    m.xy.assign(d->xy, d->xy + 2 * d->n_nodes);
    m.conn.assign((size_t)m.n_elem * nn, -1);
    for (int64_t e = 0; e < m.n_elem; ++e) {
        const int k_n = (int)(d->conn_offsets[e + 1] - d->conn_offsets[e]);
        for (int k = 0; k < k_n; ++k) {
            int64_t v = d->conn[d->conn_offsets[e] + k];
            if (v < 0 || v >= m.n_nodes) { msg = "element " + std::to_string(e) + " references a bad node"; return false; }
            m.conn[(size_t)e * nn + k] = v;
        }
    }
    for (double v : m.xy)
        if (!std::isfinite(v)) { msg = "non-finite node coordinate"; return false; }

    // Edge map keyed by the sorted vertex pair, first-seen element is the
    // left side (mesh.cpp:18-83).
    std::vector<EdgeKey> ent;
    ent.reserve((size_t)m.n_elem * 4);
    for (int64_t e = 0; e < m.n_elem; ++e) {
        const int nve = m.nv(e);
        for (int l = 0; l < nve; ++l) {
            int64_t v0 = m.conn[(size_t)e * nn + l], v1 = m.conn[(size_t)e * nn + (l + 1) % nve];
            EdgeKey k;
            k.a = std::min(v0, v1); k.b = std::max(v0, v1); k.seq = e * 4 + l;
            k.e = (int32_t)e; k.l = l;
            ent.push_back(k);
        }
    }
    std::sort(ent.begin(), ent.end(), key_less);
    std::vector<EdgeKey> bk;
    for (int64_t i = 0; i < d->n_bnd_edges; ++i) {
        int64_t v0 = d->bnd_edges[3 * i], v1 = d->bnd_edges[3 * i + 1], tag = d->bnd_edges[3 * i + 2];
        if (tag <= 0) continue;
        EdgeKey k;
        k.a = std::min(v0, v1); k.b = std::max(v0, v1); k.seq = i; k.e = (int32_t)tag; k.l = 0;
        bk.push_back(k);
    }
    std::sort(bk.begin(), bk.end(), key_less);

    size_t i = 0, jb = 0;
    const size_t ne4 = ent.size();
    m.n_bnd_faces = 0;
    m.n_orphan_edges = 0;
    while (i < ne4) {
        size_t j = i;
        while (j < ne4 && ent[j].a == ent[i].a && ent[j].b == ent[i].b) ++j;
        const size_t cnt = j - i;
        if (cnt > 2) { m.n_orphan_edges += (int64_t)cnt; i = j; continue; }
        const int32_t f = (int32_t)m.fle.size();
        m.fle.push_back(ent[i].e); m.fll.push_back(ent[i].l);
        if (cnt == 1) {
            m.fre.push_back(-1); m.frl.push_back(-1);
            int32_t bct = ZJ_BC_FARFIELD, tag = 0;
            while (jb < bk.size() && (bk[jb].a < ent[i].a || (bk[jb].a == ent[i].a && bk[jb].b < ent[i].b))) ++jb;
            size_t k = jb;
            int64_t last = -1;
            while (k < bk.size() && bk[k].a == ent[i].a && bk[k].b == ent[i].b) last = (int64_t)(k++);
            if (last >= 0) {
                tag = bk[(size_t)last].e;
                const zj_bc_spec* s = find_bc(p, tag);
                if (s) bct = s->type;
            }
            m.fbct.push_back(bct); m.ftag.push_back(tag);
            m.fslot.push_back((int32_t)m.n_bnd_faces++);
        } else {
            m.fre.push_back(ent[i + 1].e); m.frl.push_back(ent[i + 1].l);
            m.fbct.push_back(ZJ_BC_INTERIOR); m.ftag.push_back(-1); m.fslot.push_back(-1);
        }
        double nx, ny, len;
        face_normal(m, m.fle[f], m.fll[f], nx, ny, len);
        m.fnx.push_back(nx); m.fny.push_back(ny); m.flen.push_back(len);
        i = j;
    }
    m.n_faces = (int64_t)m.fle.size();
    return true;
}

// ---------------------------------------------------------------------------
// Geometry: shape functions of Q1/Q2/Q4 quads (src/basis/basis.cpp:717-847).

namespace {
const int kQ4Xi[25] = {0,4,4,0, 1,2,3, 4,4,4, 3,2,1, 0,0,0, 1,2,3,1,2,3,1,2,3};
const int kQ4Eta[25] = {0,0,4,4, 0,0,0, 1,2,3, 4,4,4, 3,2,1, 1,1,1,2,2,2,3,3,3};

void q4_lagrange(double t, double* L, double* dL) {
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

int shape(int order, double xi, double eta, double* N, double* dNx, double* dNe) {
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
        dNx[4] = -xi * eta * (eta - 1);                dNe[4] = 0.5 * (1 - xi * xi) * (2 * eta - 1);
        dNx[5] = 0.5 * (2 * xi + 1) * (1 - eta * eta);  dNe[5] = -xi * (xi + 1) * eta;
        dNx[6] = -xi * eta * (eta + 1);                dNe[6] = 0.5 * (1 - xi * xi) * (2 * eta + 1);
        dNx[7] = 0.5 * (2 * xi - 1) * (1 - eta * eta);  dNe[7] = -xi * (xi - 1) * eta;
        dNx[8] = -2 * xi * (1 - eta * eta);             dNe[8] = -2 * eta * (1 - xi * xi);
        return 9;
    }
    double Lx[5], Le[5], dLx[5], dLe[5];
    q4_lagrange(xi, Lx, dLx);
    q4_lagrange(eta, Le, dLe);
    for (int k = 0; k < 25; ++k) {
        N[k] = Lx[kQ4Xi[k]] * Le[kQ4Eta[k]];
        dNx[k] = dLx[kQ4Xi[k]] * Le[kQ4Eta[k]];
        dNe[k] = Lx[kQ4Xi[k]] * dLe[kQ4Eta[k]];
    }
    return 25;
}
}  // namespace

// Normals of a curved mesh at every flux point: [E][4][n1][4] = (nx, ny,
// 2 s, 0) with s = |dx/dt| the edge Jacobian at the point and n the face's
// unit normal there, both from the left element's mapping (shape functions of
// basis.cpp:717-847).  Edge k of the reference square runs counter-clockwise
// with t = the 1-D flux points: edge 0 (t, -1), edge 1 (1, t), edge 2
// (-t, 1), edge 3 (-1, -t); the outward normal of a positively oriented
// element is the tangent dx/dt turned clockwise.  The face's right element
// gets the same (face) normal at its coinciding point n1-1-fp, as the
// per-edge records of straight meshes do.  The 2 s slot keeps the kernels'
// s = 0.5 * length of a straight edge (for which 2 s is the length).
void build_point_normals(const HostMesh& m, const Operators1D& ops, std::vector<double>& nrm) {
    const int n1 = ops.n1;
    nrm.assign((size_t)m.n_elem * 4 * n1 * 4, 0.0);
    for (int64_t f = 0; f < m.n_faces; ++f) {
        const int64_t le = m.fle[(size_t)f];
        const int ll = m.fll[(size_t)f];
        const int64_t* nd = &m.conn[(size_t)le * m.nn];
        for (int fp = 0; fp < n1; ++fp) {
            const double t = ops.pts[(size_t)fp];
            double xi, eta, sx, se;
            switch (ll) {
                case 0: xi = t; eta = -1.0; sx = 1.0; se = 0.0; break;
                case 1: xi = 1.0; eta = t; sx = 0.0; se = 1.0; break;
                case 2: xi = -t; eta = 1.0; sx = -1.0; se = 0.0; break;
                default: xi = -1.0; eta = -t; sx = 0.0; se = -1.0; break;
            }
            double N[25], dNx[25], dNe[25];
            const int n = shape(m.order, xi, eta, N, dNx, dNe);
            double tx = 0.0, ty = 0.0;
            for (int i = 0; i < n; ++i) {
                const double dn = dNx[i] * sx + dNe[i] * se;
                tx += dn * m.xy[2 * nd[i]];
                ty += dn * m.xy[2 * nd[i] + 1];
            }
            const double len = std::sqrt(tx * tx + ty * ty);
            const double rec[4] = {ty / len, -tx / len, 2.0 * len, 0.0};
            std::memcpy(&nrm[(((size_t)le * 4 + ll) * n1 + fp) * 4], rec, sizeof(rec));
            if (m.fre[(size_t)f] >= 0) {
                const size_t r = ((size_t)m.fre[(size_t)f] * 4 + m.frl[(size_t)f]) * n1 + (n1 - 1 - fp);
                std::memcpy(&nrm[r * 4], rec, sizeof(rec));
            }
        }
    }
}

// Affine map of a triangle: x_r = (v1 - v0)/2, x_s = (v2 - v0)/2.
static void tri_jacobian(const HostMesh& m, int64_t e, double& a, double& b, double& c, double& d) {
    const int64_t* nd = &m.conn[(size_t)e * m.nn];
    const double *p0 = &m.xy[2 * nd[0]], *p1 = &m.xy[2 * nd[1]], *p2 = &m.xy[2 * nd[2]];
    a = 0.5 * (p1[0] - p0[0]); b = 0.5 * (p2[0] - p0[0]);   // x_r, x_s
    c = 0.5 * (p1[1] - p0[1]); d = 0.5 * (p2[1] - p0[1]);   // y_r, y_s
}

bool build_metrics(const HostMesh& m, const Operators1D& ops, std::vector<double>& J,
                   std::vector<double>& Jinv, std::string& msg, const TriOperators* tri) {
    const int n1 = ops.n1, nsp = n1 * n1;
    J.assign((size_t)m.n_elem * nsp, 0.0);
    Jinv.assign((size_t)m.n_elem * nsp * 4, 0.0);
    for (int64_t e = 0; e < m.n_elem; ++e) {
        if (m.etype[(size_t)e] == ZJ_ELEM_TRI) {
            if (!tri) { msg = "triangle without triangle operators"; return false; }
            double a, b, c, dd;
            tri_jacobian(m, e, a, b, c, dd);
            const double Jd = a * dd - b * c;
            if (!(Jd > 0.0) || !std::isfinite(Jd)) {
                msg = "element " + std::to_string(e) + " has a non-positive Jacobian (check node order: CCW)";
                return false;
            }
            const double inv = 1.0 / Jd;
            for (int sp = 0; sp < tri->nt; ++sp) {
                J[(size_t)e * nsp + sp] = Jd;
                double* Ji = &Jinv[((size_t)e * nsp + sp) * 4];
                Ji[0] = dd * inv; Ji[1] = -b * inv; Ji[2] = -c * inv; Ji[3] = a * inv;
            }
            continue;
        }
        const int64_t* nd = &m.conn[(size_t)e * m.nn];
        for (int sp = 0; sp < nsp; ++sp) {
            double N[25], dNx[25], dNe[25];
            int n = shape(m.order, ops.pts[sp % n1], ops.pts[sp / n1], N, dNx, dNe);
            double a = 0.0, b = 0.0, c = 0.0, dd = 0.0;   // x_xi, x_eta, y_xi, y_eta
            for (int i = 0; i < n; ++i) {
                double x = m.xy[2 * nd[i]], y = m.xy[2 * nd[i] + 1];
                a += dNx[i] * x; b += dNe[i] * x; c += dNx[i] * y; dd += dNe[i] * y;
            }
            double Jd = a * dd - b * c;
            if (!(Jd > 0.0) || !std::isfinite(Jd)) {
                msg = "element " + std::to_string(e) + " has a non-positive Jacobian (check node order: CCW)";
                return false;
            }
            double inv = 1.0 / Jd;
            J[(size_t)e * nsp + sp] = Jd;
            double* Ji = &Jinv[((size_t)e * nsp + sp) * 4];
            Ji[0] = dd * inv; Ji[1] = -b * inv; Ji[2] = -c * inv; Ji[3] = a * inv;
        }
    }
    return true;
}

void sp_coords(const HostMesh& m, const Operators1D& ops, std::vector<double>& out, const TriOperators* tri) {
    const int n1 = ops.n1, nsp = n1 * n1;
    out.assign((size_t)m.n_elem * nsp * 2, 0.0);
    for (int64_t e = 0; e < m.n_elem; ++e) {
        const int64_t* nd = &m.conn[(size_t)e * m.nn];
        if (m.etype[(size_t)e] == ZJ_ELEM_TRI) {
            if (!tri) continue;
            const double *p0 = &m.xy[2 * nd[0]], *p1 = &m.xy[2 * nd[1]], *p2 = &m.xy[2 * nd[2]];
            for (int sp = 0; sp < tri->nt; ++sp) {
                const double r = tri->r[sp], s = tri->s[sp];
                const double w0 = -0.5 * (r + s), w1 = 0.5 * (1.0 + r), w2 = 0.5 * (1.0 + s);
                out[((size_t)e * nsp + sp) * 2] = w0 * p0[0] + w1 * p1[0] + w2 * p2[0];
                out[((size_t)e * nsp + sp) * 2 + 1] = w0 * p0[1] + w1 * p1[1] + w2 * p2[1];
            }
            continue;
        }
        for (int sp = 0; sp < nsp; ++sp) {
            double N[25], dNx[25], dNe[25];
            int n = shape(m.order, ops.pts[sp % n1], ops.pts[sp / n1], N, dNx, dNe);
            double x = 0.0, y = 0.0;
            for (int i = 0; i < n; ++i) { x += N[i] * m.xy[2 * nd[i]]; y += N[i] * m.xy[2 * nd[i] + 1]; }
            out[((size_t)e * nsp + sp) * 2] = x;
            out[((size_t)e * nsp + sp) * 2 + 1] = y;
        }
    }
}

// mesh.cpp:122-146
void element_areas(const HostMesh& m, std::vector<double>& area) {
    area.assign((size_t)m.n_elem, 0.0);
    for (int64_t e = 0; e < m.n_elem; ++e) {
        const int64_t* nd = &m.conn[(size_t)e * m.nn];
        const double *p0 = &m.xy[2 * nd[0]], *p1 = &m.xy[2 * nd[1]], *p2 = &m.xy[2 * nd[2]];
        double a1 = 0.5 * std::fabs((p1[0] - p0[0]) * (p2[1] - p0[1]) - (p2[0] - p0[0]) * (p1[1] - p0[1]));
        if (m.etype[(size_t)e] == ZJ_ELEM_TRI) { area[(size_t)e] = a1; continue; }
        const double* p3 = &m.xy[2 * nd[3]];
        double a2 = 0.5 * std::fabs((p2[0] - p0[0]) * (p3[1] - p0[1]) - (p3[0] - p0[0]) * (p2[1] - p0[1]));
        area[(size_t)e] = a1 + a2;
    }
}

// Eight doubles per boundary slot.  Compat layout follows fr_solver.cpp:438-482
// (far-field: rho, u, v, p at infinity; outflow: p_static); the physics mode
// adds inflow (p_total, T_total, dir) and the isothermal wall temperature.
void build_bc_data(const HostMesh& m, const zj_params* p, std::vector<double>& bc) {
    bc.assign((size_t)std::max<int64_t>(m.n_bnd_faces, 1) * 8, 0.0);
    const double rho_inf = p->rho_inf;
    const double c_inf = std::sqrt(p->gamma * p->p_inf / rho_inf);
    const double vel_inf = p->Mach * c_inf;
    const double u_inf = vel_inf * std::cos(p->AoA * M_PI / 180.0);
    const double v_inf = vel_inf * std::sin(p->AoA * M_PI / 180.0);
    for (int64_t f = 0; f < m.n_faces; ++f) {
        if (m.fslot[f] < 0) continue;
        double* d = &bc[(size_t)m.fslot[f] * 8];
        const zj_bc_spec* s = (m.ftag[f] > 0) ? find_bc(p, m.ftag[f]) : nullptr;
        switch (m.fbct[f]) {
            case ZJ_BC_FARFIELD:
                d[0] = rho_inf; d[1] = u_inf; d[2] = v_inf; d[3] = p->p_inf;
                break;
            case ZJ_BC_OUTFLOW:
                d[0] = (s && s->p_static > 0) ? s->p_static : p->p_inf;
                break;
            case ZJ_BC_INFLOW: {
                d[0] = (s && s->p_total > 0) ? s->p_total : p->p_inf * 1.2;
                d[1] = (s && s->T_total > 0) ? s->T_total : p->T_inf;
                double dx = s ? s->dir_x : 1.0, dy = s ? s->dir_y : 0.0;
                double mag = std::sqrt(dx * dx + dy * dy);
                if (!(mag > 0)) { dx = 1.0; dy = 0.0; mag = 1.0; }
                d[2] = dx / mag; d[3] = dy / mag;
                break;
            }
            case ZJ_BC_WALL:
                d[0] = s ? s->T_wall : 0.0;
                break;
            default:
                break;
        }
    }
}

void build_edge_records(const HostMesh& m, std::vector<EdgeRec>& rec, std::vector<double>& nrm) {
    rec.assign((size_t)m.n_elem * 4, EdgeRec{-1, 0, kEdgeOrphan, 0});
    nrm.assign((size_t)m.n_elem * 4 * 4, 0.0);   // nx, ny, edge length, pad
    for (int64_t f = 0; f < m.n_faces; ++f) {
        const int64_t lo = (int64_t)m.fle[f] * 4 + m.fll[f];
        if (m.fre[f] < 0) {
            rec[lo] = EdgeRec{-1, m.fslot[f], kEdgeBoundary | (m.fbct[f] << 8), 0};
        } else {
            const int64_t ro = (int64_t)m.fre[f] * 4 + m.frl[f];
            rec[lo] = EdgeRec{m.fre[f], m.frl[f], 0, 0};
            rec[ro] = EdgeRec{m.fle[f], m.fll[f], kEdgeRight, 0};
            nrm[ro * 4] = m.fnx[f]; nrm[ro * 4 + 1] = m.fny[f]; nrm[ro * 4 + 2] = m.flen[f];
        }
        nrm[lo * 4] = m.fnx[f]; nrm[lo * 4 + 1] = m.fny[f]; nrm[lo * 4 + 2] = m.flen[f];
    }
}

}  // namespace zj

// ---------------------------------------------------------------------------
// Config parsing with the reference grammar (src/main.cpp:78-170).

extern "C" void zj_params_default(zj_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma = 1.4; p->Pr = 0.72; p->Re = 1000.0; p->Mach = 0.5; p->T_inf = 300.0;
    p->p_inf = 101325.0; p->rho_inf = 1.225; p->AoA = 0.0;
    p->poly_order = 3; p->flux_type = ZJ_FLUX_HU; p->riemann = ZJ_RIEMANN_ROE;
    p->CFL = 0.5; p->dt = 0.0; p->t_final = 1.0; p->max_iter = 100000;
    p->viscous = 1; p->output_freq = 100; p->restart_freq = 1000;
    std::snprintf(p->case_name, sizeof(p->case_name), "%s", "simulation");
    p->compat = 1; p->precision = ZJ_FP64; p->n_bc = 0;
}

namespace {

std::string lower(std::string s) {
    std::transform(s.begin(), s.end(), s.begin(), [](unsigned char c) { return (char)std::tolower(c); });
    return s;
}

// createBCFromSpec's type strings (src/bc/boundary_condition.cpp:32-64).
int bc_type_from_string(const std::string& t) {
    if (t == "wall" || t == "noslip" || t == "no_slip" || t == "no-slip") return ZJ_BC_WALL;
    if (t == "slipwall" || t == "slip_wall" || t == "slip" || t == "inviscid_wall") return ZJ_BC_SLIPWALL;
    if (t == "symmetry" || t == "sym") return ZJ_BC_SYMMETRY;
    if (t == "farfield" || t == "far_field" || t == "far-field" || t == "freestream") return ZJ_BC_FARFIELD;
    if (t == "inflow" || t == "inlet") return ZJ_BC_INFLOW;
    if (t == "outflow" || t == "outlet" || t == "exit") return ZJ_BC_OUTFLOW;
    if (t == "periodic") return ZJ_BC_PERIODIC;
    return ZJ_BC_SLIPWALL;   // unknown strings default to a slip wall
}

void parse_stream(std::istream& in, zj_params* p) {
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream iss(line);
        std::string key;
        iss >> key;
        if (key == "gamma") iss >> p->gamma;
        else if (key == "Pr") iss >> p->Pr;
        else if (key == "Re") iss >> p->Re;
        else if (key == "Mach") iss >> p->Mach;
        else if (key == "AoA") iss >> p->AoA;
        else if (key == "T_inf") iss >> p->T_inf;
        else if (key == "p_inf") iss >> p->p_inf;
        else if (key == "rho_inf") iss >> p->rho_inf;
        else if (key == "poly_order") iss >> p->poly_order;
        else if (key == "CFL") iss >> p->CFL;
        else if (key == "dt") iss >> p->dt;
        else if (key == "t_final") iss >> p->t_final;
        else if (key == "max_iter") iss >> p->max_iter;
        else if (key == "viscous") { std::string v; iss >> v; p->viscous = (v == "true" || v == "1"); }
        else if (key == "output_freq") iss >> p->output_freq;
        else if (key == "restart_freq") iss >> p->restart_freq;
        else if (key == "case_name") {
            std::string v; iss >> v;
            std::snprintf(p->case_name, sizeof(p->case_name), "%s", v.c_str());
        } else if (key == "flux_type") {
            std::string t; iss >> t;
            if (t == "DG") p->flux_type = ZJ_FLUX_DG;
            else if (t == "SD") p->flux_type = ZJ_FLUX_SD;
            else if (t == "HU") p->flux_type = ZJ_FLUX_HU;
            else if (t == "GA") p->flux_type = ZJ_FLUX_GA;
        } else if (key == "riemann") {
            std::string t; iss >> t;
            if (t == "Rusanov") p->riemann = ZJ_RIEMANN_RUSANOV;
            else if (t == "Roe") p->riemann = ZJ_RIEMANN_ROE;
            else if (t == "HLLC") p->riemann = ZJ_RIEMANN_HLLC;
        } else if (key == "compat") {
            std::string t; iss >> t; t = lower(t);
            p->compat = (t == "on" || t == "1" || t == "true");
        } else if (key == "precision") {
            std::string t; iss >> t; t = lower(t);
            if (t == "fp64") p->precision = ZJ_FP64;
            else if (t == "mixed" || t == "fp32") p->precision = ZJ_MIXED;
            else if (t == "split_bf16") p->precision = ZJ_SPLIT_BF16;
        } else if (key == "bc") {
            int tag = 0;
            std::string type;
            iss >> tag >> type;
            zj_bc_spec s;
            std::memset(&s, 0, sizeof(s));
            s.tag = tag;
            s.type = bc_type_from_string(lower(type));
            s.dir_x = 1.0; s.dir_y = 0.0;
            std::string k;
            while (iss >> k) {
                k = lower(k);
                if (k == "p_static") iss >> s.p_static;
                else if (k == "p_total") iss >> s.p_total;
                else if (k == "t_total") iss >> s.T_total;
                else if (k == "t_wall") iss >> s.T_wall;
                else if (k == "direction") iss >> s.dir_x >> s.dir_y;
            }
            int slot = -1;   // a repeated tag overwrites (std::map semantics)
            for (int i = 0; i < p->n_bc; ++i) if (p->bc[i].tag == tag) slot = i;
            if (slot < 0 && p->n_bc < ZJ_MAX_BC) slot = p->n_bc++;
            if (slot >= 0) p->bc[slot] = s;
        }
    }
}

}  // namespace

extern "C" zj_status zj_params_parse_file(const char* path, zj_params* p) {
    if (!path || !p) return ZJ_ERR_ARG;
    std::ifstream f(path);
    if (!f.is_open()) return ZJ_ERR_IO;
    parse_stream(f, p);
    return ZJ_OK;
}

extern "C" zj_status zj_params_parse_string(const char* text, zj_params* p) {
    if (!text || !p) return ZJ_ERR_ARG;
    std::istringstream in(text);
    parse_stream(in, p);
    return ZJ_OK;
}
