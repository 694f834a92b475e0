// tri_setup.cpp -- FR operators of the straight-sided triangle, physics mode.
//
// Reference element T = {(r,s): r >= -1, s >= -1, r + s <= 0}, vertices
// (-1,-1), (1,-1), (-1,1) (the reference's (0,0), (1,0), (0,1) triangle with
// r = 2 xi - 1, s = 2 eta - 1).  Solution points: the reference's collapsed
// Gauss-Legendre set (SolutionPoints::getTriangle, src/basis/basis.cpp:391-416):
// row j = 0..p at t_j, points i = 0..p-j at s_i, (xi, eta) = (s_i (1 - t_j), t_j)
// with s, t the Gauss-Legendre nodes mapped to [0, 1]; unisolvent for P_p
// (p+1-j distinct points on each of p+1 distinct horizontal lines).  Flux
// points: p+1 Gauss-Legendre points per edge, counter-clockwise
// (FROperators::initTriangle, basis.cpp:629-640): edge 0 (r, -1), edge 1
// (-sigma, sigma), edge 2 (-1, -sigma), sigma ascending.
//
// The reference leaves the triangle's interpolation, differentiation and
// correction operators at zero (basis.cpp:642-668); they are built here from
// the literature:
//  * nodal operators from the orthonormal Proriol-Koornwinder-Dubiner basis
//    psi_ij = sqrt(2) P_i(a) P_j^(2i+1,0)(b) (1-b)^i, a = 2(1+r)/(1-s) - 1,
//    b = s (Hesthaven & Warburton, Nodal Discontinuous Galerkin Methods,
//    2008, sec. 6.1): V = psi(x_n), Dr = V_r V^-1, Ds = V_s V^-1, edge
//    interpolation L = psi(x_f) V^-1;
//  * VCJH correction fields (Castonguay, Vincent & Jameson, J. Sci. Comput.
//    50, 2012): phi_{f,j} in P_p with
//      (phi, v)_T + c sum_m C(p,m) (d^p phi / dr^m ds^(p-m), d^p v / ...)_T
//        = int_{edge f} l_j v dGamma      for all v in P_p,
//    solved in the orthonormal modal basis, (I + c K) phi^ = b; c = 0 is the
//    nodal DG lifting.  The c of each flux type is the one-dimensional value
//    of build_operators_vcjh (the 1D SD / HU / GA schemes' c) -- an energy
//    stable member of the triangle family, not a triangle "SD" scheme.
// The residual of a triangle then reads, at solution point n,
//    R_n = -(1/J) [ sum_k Dr_nk F~_k + Ds_nk G~_k + sum_{f,j} phi_{f,j}(x_n) dF_{f,j} ],
//    dF_{f,j} = (|edge_f| / |ref edge_f|) F_common . n - F~(x_fj) . n^_f,
// with n^_f the unit outward normal of the reference edge.
#include <cmath>
#include <string>
#include <vector>

#include "zj_internal.h"

namespace zj {

namespace {

// Orthonormal Jacobi polynomial P_n^(alpha,beta)(x) and its derivative
// (normalised on [-1,1] with weight (1-x)^alpha (1+x)^beta; three-term
// recurrence, Hesthaven & Warburton, Appendix A).
double jacobi(int n, double alpha, double beta, double x) {
    const double g0 = std::pow(2.0, alpha + beta + 1.0) / (alpha + beta + 1.0) * std::tgamma(alpha + 1.0) *
                      std::tgamma(beta + 1.0) / std::tgamma(alpha + beta + 1.0);
    double pm1 = 1.0 / std::sqrt(g0);
    if (n == 0) return pm1;
    const double g1 = (alpha + 1.0) * (beta + 1.0) / (alpha + beta + 3.0) * g0;
    double p = ((alpha + beta + 2.0) * x / 2.0 + (alpha - beta) / 2.0) / std::sqrt(g1);
    if (n == 1) return p;
    double aold = 2.0 / (2.0 + alpha + beta) * std::sqrt((alpha + 1.0) * (beta + 1.0) / (alpha + beta + 3.0));
    for (int i = 1; i < n; ++i) {
        const double h1 = 2.0 * i + alpha + beta;
        const double anew = 2.0 / (h1 + 2.0) *
                            std::sqrt((i + 1.0) * (i + 1.0 + alpha + beta) * (i + 1.0 + alpha) * (i + 1.0 + beta) /
                                      (h1 + 1.0) / (h1 + 3.0));
        const double bnew = -(alpha * alpha - beta * beta) / h1 / (h1 + 2.0);
        const double pn = 1.0 / anew * (-aold * pm1 + (x - bnew) * p);
        pm1 = p;
        p = pn;
        aold = anew;
    }
    return p;
}

double jacobi_deriv(int n, double alpha, double beta, double x) {
    if (n == 0) return 0.0;
    return std::sqrt(n * (n + alpha + beta + 1.0)) * jacobi(n - 1, alpha + 1.0, beta + 1.0, x);
}

// psi_ij and its r, s derivatives at (r, s).
void pkd(int i, int j, double r, double s, double& f, double& fr, double& fs) {
    const double a = (s != 1.0) ? 2.0 * (1.0 + r) / (1.0 - s) - 1.0 : -1.0;
    const double b = s;
    const double fa = jacobi(i, 0, 0, a), dfa = jacobi_deriv(i, 0, 0, a);
    const double gb = jacobi(j, 2.0 * i + 1.0, 0, b), dgb = jacobi_deriv(j, 2.0 * i + 1.0, 0, b);
    const double h = 0.5 * (1.0 - b);
    f = std::sqrt(2.0) * fa * gb * std::pow(1.0 - b, i);
    // Hesthaven & Warburton GradSimplex2DP, with their 2^(i+1/2) normalisation
    double dr = dfa * gb;
    if (i > 0) dr *= std::pow(h, i - 1);
    double ds = dfa * (gb * (0.5 * (1.0 + a)));
    if (i > 0) ds *= std::pow(h, i - 1);
    double tmp = dgb * std::pow(h, i);
    if (i > 0) tmp -= 0.5 * i * gb * std::pow(h, i - 1);
    ds += fa * tmp;
    const double sc = std::pow(2.0, i + 0.5);
    fr = dr * sc;
    fs = ds * sc;
}

// A^-1 of a dense n x n matrix (row-major), Gauss-Jordan with partial pivoting.
bool invert(int n, std::vector<double> A, std::vector<double>& inv) {
    inv.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; ++c) {
        int piv = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
        if (std::fabs(A[(size_t)piv * n + c]) < 1e-300) return false;
        if (piv != c)
            for (int k = 0; k < n; ++k) {
                std::swap(A[(size_t)c * n + k], A[(size_t)piv * n + k]);
                std::swap(inv[(size_t)c * n + k], inv[(size_t)piv * n + k]);
            }
        const double d = 1.0 / A[(size_t)c * n + c];
        for (int k = 0; k < n; ++k) { A[(size_t)c * n + k] *= d; inv[(size_t)c * n + k] *= d; }
        for (int r = 0; r < n; ++r) {
            if (r == c) continue;
            const double f = A[(size_t)r * n + c];
            if (f == 0.0) continue;
            for (int k = 0; k < n; ++k) {
                A[(size_t)r * n + k] -= f * A[(size_t)c * n + k];
                inv[(size_t)r * n + k] -= f * inv[(size_t)c * n + k];
            }
        }
    }
    return true;
}

void matmul(int m, int k, int n, const std::vector<double>& A, const std::vector<double>& B,
            std::vector<double>& C) {
    C.assign((size_t)m * n, 0.0);
    for (int i = 0; i < m; ++i)
        for (int l = 0; l < k; ++l) {
            const double a = A[(size_t)i * k + l];
            for (int j = 0; j < n; ++j) C[(size_t)i * n + j] += a * B[(size_t)l * n + j];
        }
}

double factorial(int n) {
    double f = 1.0;
    for (int i = 2; i <= n; ++i) f *= i;
    return f;
}

}  // namespace

double vcjh_c(int P, int flux_type) {
    const int p = P;
    const double fp = factorial(p), f2p = factorial(2 * p);
    const double ap_pf = f2p / (std::pow(2.0, p) * fp);
    const double ap2 = ap_pf * ap_pf;
    switch (flux_type) {
        case ZJ_FLUX_SD: return 2.0 * p / ((2.0 * p + 1.0) * (p + 1.0) * ap2);
        case ZJ_FLUX_HU: return 2.0 * (p + 1.0) / ((2.0 * p + 1.0) * p * ap2);
        case ZJ_FLUX_GA: return 2.0 * (p + 1.0) * fp * fp / (f2p * (2.0 * p + 1.0));
        default: return 0.0;
    }
}

bool build_operators_tri(int P, int flux_type, TriOperators& t, std::string& msg) {
    const int p = P, n1 = P + 1, nt = (P + 1) * (P + 2) / 2, nf = 3 * n1;
    t = TriOperators();
    t.P = P; t.n1 = n1; t.nt = nt;
    std::vector<double> g, gw;
    gauss_legendre(n1, g, gw);
    // solution points (basis.cpp:391-416), as (r, s)
    for (int j = 0; j <= p; ++j)
        for (int i = 0; i <= p - j; ++i) {
            const double sc = 0.5 * (1.0 + g[i]), tc = 0.5 * (1.0 + g[j]);
            t.r.push_back(2.0 * sc * (1.0 - tc) - 1.0);
            t.s.push_back(2.0 * tc - 1.0);
        }
    // modal basis order (i, j), i + j <= p
    std::vector<std::pair<int, int>> modes;
    for (int i = 0; i <= p; ++i)
        for (int j = 0; j <= p - i; ++j) modes.push_back({i, j});
    auto vander = [&](const std::vector<double>& rr, const std::vector<double>& ss, std::vector<double>& V,
                      std::vector<double>& Vr, std::vector<double>& Vs) {
        const int n = (int)rr.size();
        V.assign((size_t)n * nt, 0.0); Vr = V; Vs = V;
        for (int q = 0; q < n; ++q)
            for (int k = 0; k < nt; ++k)
                pkd(modes[k].first, modes[k].second, rr[q], ss[q], V[(size_t)q * nt + k], Vr[(size_t)q * nt + k],
                    Vs[(size_t)q * nt + k]);
    };
    std::vector<double> V, Vr, Vs, Vinv;
    vander(t.r, t.s, V, Vr, Vs);
    if (!invert(nt, V, Vinv)) { msg = "triangle Vandermonde is singular"; return false; }
    matmul(nt, nt, nt, Vr, Vinv, t.Dr);
    matmul(nt, nt, nt, Vs, Vinv, t.Ds);
    // flux points, edge-major, counter-clockwise
    std::vector<double> fr, fs;
    for (int f = 0; f < 3; ++f)
        for (int j = 0; j < n1; ++j) {
            const double sg = g[j];
            if (f == 0) { fr.push_back(sg); fs.push_back(-1.0); }
            else if (f == 1) { fr.push_back(-sg); fs.push_back(sg); }
            else { fr.push_back(-1.0); fs.push_back(-sg); }
        }
    std::vector<double> Vf, Vfr, Vfs;
    vander(fr, fs, Vf, Vfr, Vfs);
    matmul(nf, nt, nt, Vf, Vinv, t.L);
    // p-th derivatives of the modes: monomial coefficients of each mode
    std::vector<std::pair<int, int>> mono;          // (a, b): r^a s^b
    for (int a = 0; a <= p; ++a)
        for (int b = 0; b <= p - a; ++b) mono.push_back({a, b});
    std::vector<double> M((size_t)nt * nt), Minv;
    for (int q = 0; q < nt; ++q)
        for (int k = 0; k < nt; ++k) M[(size_t)q * nt + k] = std::pow(t.r[q], mono[k].first) * std::pow(t.s[q], mono[k].second);
    if (!invert(nt, M, Minv)) { msg = "triangle monomial Vandermonde is singular"; return false; }
    std::vector<double> coef;                        // [mono][mode]
    matmul(nt, nt, nt, Minv, V, coef);
    const double c = vcjh_c(P, flux_type);
    std::vector<double> A((size_t)nt * nt, 0.0);     // I + c K
    for (int k = 0; k < nt; ++k) A[(size_t)k * nt + k] = 1.0;
    if (c != 0.0) {
        for (int m = 0; m <= p; ++m) {
            int q = -1;
            for (int k = 0; k < nt; ++k) if (mono[k].first == m && mono[k].second == p - m) q = k;
            const double fac = factorial(m) * factorial(p - m);
            const double binom = factorial(p) / (factorial(m) * factorial(p - m));
            for (int i = 0; i < nt; ++i)
                for (int k = 0; k < nt; ++k)
                    A[(size_t)i * nt + k] += c * binom * 2.0 * (fac * coef[(size_t)q * nt + i]) * (fac * coef[(size_t)q * nt + k]);
        }
    }
    std::vector<double> Ainv;
    if (!invert(nt, A, Ainv)) { msg = "triangle correction system is singular"; return false; }
    // phi_{f,j} at the solution points: V Ainv b, b_k = |ref edge|/2 w_j psi_k(x_fj)
    const double elen[3] = {2.0, 2.0 * std::sqrt(2.0), 2.0};
    t.Phi.assign((size_t)nt * nf, 0.0);
    for (int f = 0; f < 3; ++f)
        for (int j = 0; j < n1; ++j) {
            const int q = f * n1 + j;
            std::vector<double> b(nt), ph(nt, 0.0);
            for (int k = 0; k < nt; ++k) b[k] = 0.5 * elen[f] * gw[j] * Vf[(size_t)q * nt + k];
            for (int i = 0; i < nt; ++i)
                for (int k = 0; k < nt; ++k) ph[i] += Ainv[(size_t)i * nt + k] * b[k];
            for (int n = 0; n < nt; ++n) {
                double v = 0.0;
                for (int k = 0; k < nt; ++k) v += V[(size_t)n * nt + k] * ph[k];
                t.Phi[(size_t)n * nf + q] = v;
            }
        }
    // quadrature weights at the solution points: the integrals of the nodal
    // basis, w_n = sum_k Vinv[k][n] int psi_k = sqrt(2) Vinv[0][n] (psi_00 = 1/sqrt(2))
    t.w.assign(nt, 0.0);
    for (int n = 0; n < nt; ++n) t.w[n] = std::sqrt(2.0) * Vinv[(size_t)0 * nt + n];
    return true;
}

}  // namespace zj
