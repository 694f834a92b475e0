"""Oracle (test infrastructure) of the physics-mode residual on meshes of
straight-sided quadrilaterals and triangles, in numpy, for small meshes.

The reference has no working triangle FR (FROperators::initTriangle,
src/basis/basis.cpp:615-668, leaves every triangle operator at zero), so the
triangle part is parity unpinned against the reference; this oracle states
the scheme the CUDA kernels implement, from the same definitions but an
independent construction:

* triangle solution points: the reference's collapsed Gauss-Legendre set
  (SolutionPoints::getTriangle, basis.cpp:391-416); flux points: p+1
  Gauss-Legendre points per edge, counter-clockwise (basis.cpp:629-640);
* nodal operators from a MONOMIAL basis (the kernels' setup uses the
  orthonormal Dubiner basis): Dr = V_r V^-1, Ds = V_s V^-1, L = V_f V^-1;
* VCJH correction fields from (M + c K) phi^ = b in the monomial basis with
  the mass matrix M by a collapsed (Duffy) Gauss-Legendre quadrature,
  K_ii = C(p,m) (m! (p-m)!)^2 |T| for the top-degree monomial r^m s^(p-m),
  b_i = int_edge l_j m_i; c of the flux type as in one dimension;
* quadrilaterals: tensor-product Gauss-Legendre operators with the pinned
  VCJH derivatives of the C oracle (orc_vcjh);
* pointwise physics -- Riemann fluxes, ghost states, viscous flux -- from the
  C oracle, which is pinned to the reference's functions.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

try:
    from . import oracle as O
except ImportError:          # imported as a top-level module
    import oracle as O

SQ2 = math.sqrt(2.0)
TRI_NREF = np.array([[0.0, -1.0], [1.0 / SQ2, 1.0 / SQ2], [-1.0, 0.0]])
TRI_REFLEN = np.array([2.0, 2.0 * SQ2, 2.0])


def vcjh_c(P, flux_type):
    p = P
    fp, f2p = math.factorial(p), math.factorial(2 * p)
    ap2 = (f2p / (2.0 ** p * fp)) ** 2
    if flux_type == 1:
        return 2.0 * p / ((2.0 * p + 1.0) * (p + 1.0) * ap2)
    if flux_type == 2:
        return 2.0 * (p + 1.0) / ((2.0 * p + 1.0) * p * ap2)
    if flux_type == 3:
        return 2.0 * (p + 1.0) * fp * fp / (f2p * (2.0 * p + 1.0))
    return 0.0


def tri_points(P):
    g, _ = np.polynomial.legendre.leggauss(P + 1)
    r, s = [], []
    for j in range(P + 1):
        for i in range(P + 1 - j):
            sc, tc = 0.5 * (1 + g[i]), 0.5 * (1 + g[j])
            r.append(2 * sc * (1 - tc) - 1)
            s.append(2 * tc - 1)
    return np.array(r), np.array(s)


def tri_flux_points(P):
    g, w = np.polynomial.legendre.leggauss(P + 1)
    fr = np.concatenate([g, -g, -np.ones_like(g)])
    fs = np.concatenate([-np.ones_like(g), g, -g])
    return fr, fs, g, w


def tri_operators(P, flux_type):
    """Dr, Ds [nt][nt], L [3(P+1)][nt], Phi [nt][3(P+1)], w [nt]."""
    mono = [(a, b) for a in range(P + 1) for b in range(P + 1 - a)]
    nt = len(mono)
    r, s = tri_points(P)

    def mv(rr, ss):
        return np.stack([rr ** a * ss ** b for a, b in mono], axis=-1)

    def mvr(rr, ss):
        return np.stack([a * rr ** max(a - 1, 0) * ss ** b if a else 0 * rr for a, b in mono], axis=-1)

    def mvs(rr, ss):
        return np.stack([b * rr ** a * ss ** max(b - 1, 0) if b else 0 * rr for a, b in mono], axis=-1)
    V = mv(r, s)
    Vi = np.linalg.inv(V)
    Dr = mvr(r, s) @ Vi
    Ds = mvs(r, s) @ Vi
    fr, fs, g, w = tri_flux_points(P)
    L = mv(fr, fs) @ Vi
    # mass matrix of the monomials on the reference triangle (Duffy map)
    xq, wq = np.polynomial.legendre.leggauss(2 * P + 3)
    A, B = np.meshgrid(xq, xq, indexing="ij")
    WA, WB = np.meshgrid(wq, wq, indexing="ij")
    rq = 0.5 * (1 + A) * (1 - B) - 1
    sq = B
    wt = (WA * WB * 0.5 * (1 - B)).ravel()
    Mq = mv(rq.ravel(), sq.ravel())
    M = (Mq * wt[:, None]).T @ Mq
    K = np.zeros((nt, nt))
    c = vcjh_c(P, flux_type)
    for i, (a, b) in enumerate(mono):
        if a + b == P:
            K[i, i] = math.comb(P, a) * (math.factorial(a) * math.factorial(b)) ** 2 * 2.0
    Phi = np.zeros((nt, 3 * (P + 1)))
    Mf = mv(fr, fs)
    for f in range(3):
        for j in range(P + 1):
            q = f * (P + 1) + j
            bq = 0.5 * TRI_REFLEN[f] * w[j] * Mf[q]
            coef = np.linalg.solve(M + c * K, bq)
            Phi[:, q] = V @ coef
    integ = Mq.T @ wt          # int m_i over the triangle
    w_nodes = Vi.T @ integ     # nodal quadrature weights
    return Dr, Ds, L, Phi, w_nodes


def quad_operators(P, flux_type):
    """1D GL nodes, D1, Lm, Lp, gL', gR' (pinned VCJH of the C oracle)."""
    n1 = P + 1
    x, w = np.polynomial.legendre.leggauss(n1)
    D1 = np.zeros((n1, n1))
    for k in range(n1):
        ck = np.zeros(n1)
        ck[k] = 1.0
        poly = np.polynomial.polynomial.Polynomial.fit(x, ck, n1 - 1, domain=[-1, 1], window=[-1, 1])
        D1[:, k] = poly.deriv()(x)
        if k == 0:
            Lm, Lp = np.zeros(n1), np.zeros(n1)
        Lm[k], Lp[k] = poly(-1.0), poly(1.0)
    gL, gR = np.empty(n1), np.empty(n1)
    O.lib().orc_vcjh(P, flux_type, O._d(np.ascontiguousarray(x)), O._d(gL), O._d(gR))
    return x, w, D1, Lm, Lp, gL, gR


def viscous_point(U, dx, dy, g, Re, Pr):
    h = O.lib()
    if not getattr(h, "_vf_set", False):
        dp = C.POINTER(C.c_double)
        h.orc_viscous_flux.argtypes = [dp, dp, dp, C.c_double, C.c_double, C.c_double, dp, dp]
        h._vf_set = True
    Fv, Gv = np.empty(4), np.empty(4)
    h.orc_viscous_flux(O._d(np.ascontiguousarray(U, dtype=np.float64)),
                       O._d(np.ascontiguousarray(dx, dtype=np.float64)),
                       O._d(np.ascontiguousarray(dy, dtype=np.float64)), g, Re, Pr, O._d(Fv), O._d(Gv))
    return Fv, Gv


class MixedOracle:
    """Physics-mode residual R(U) on a meshgen.MixedMesh (or QuadMesh)."""

    def __init__(self, mesh, P, gamma=1.4, rho_inf=1.0, p_inf=1.0 / 1.4, Mach=0.5, AoA=0.0,
                 flux_type=2, riemann=1, viscous=False, Re=1000.0, Pr=0.72, T_inf=300.0, tags=None):
        self.P, self.n1, self.g = P, P + 1, gamma
        self.nsp = (P + 1) ** 2
        self.nt = (P + 1) * (P + 2) // 2
        self.riemann, self.viscous, self.Re, self.Pr = riemann, viscous, Re, Pr
        xy = np.asarray(mesh.xy, dtype=np.float64)
        if hasattr(mesh, "offsets"):
            self.etype = np.asarray(mesh.etype)
            self.elems = [np.asarray(mesh.element(e)) for e in range(mesh.n_elem)]
        else:
            self.etype = np.ones(mesh.n_elem, dtype=np.int32)
            self.elems = [np.asarray(c[:4]) for c in mesh.conn]
        self.E = len(self.elems)
        self.xy = xy
        # pointwise ghost states through a C oracle context with these tags
        if tags is None:
            tags = [(t, O.BC_TYPES[n], 0.0) for t, n in sorted(mesh.tag_names.items())]
        self.tagtype = {t: ty for t, ty, *_ in tags}
        dummy = type("M", (), {})()
        dummy.xy = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], dtype=np.float64)
        dummy.conn = np.array([[0, 1, 2, 3]], dtype=np.int64)
        dummy.bnd = np.array([[0, 1, tags[0][0] if tags else 1]], dtype=np.int64)
        self._ctx = O.Oracle(dummy, P, gamma, rho_inf, p_inf, Mach, AoA, tags=tags)
        self._ctx.set_physics(flux_type, riemann, viscous, Re, Pr, T_inf)
        self.q = quad_operators(P, flux_type)
        self.t = tri_operators(P, flux_type)
        self._faces(mesh)
        self._geometry()

    # -- topology ----------------------------------------------------------
    def _faces(self, mesh):
        tag = {}
        for v0, v1, t in np.asarray(mesh.bnd):
            if t > 0:
                tag[(min(v0, v1), max(v0, v1))] = int(t)
        first = {}
        self.nbr = {}        # (e, edge) -> (e2, edge2) or ("bnd", type, tag, slot)
        for e, nd in enumerate(self.elems):
            nv = len(nd)
            for l in range(nv):
                a, b = int(nd[l]), int(nd[(l + 1) % nv])
                k = (min(a, b), max(a, b))
                if k in first:
                    e0, l0 = first.pop(k)
                    self.nbr[(e0, l0)] = (e, l, False)
                    self.nbr[(e, l)] = (e0, l0, True)
                else:
                    first[k] = (e, l)
        for k, (e, l) in first.items():
            t = tag.get(k, 0)
            self.nbr[(e, l)] = ("bnd", self.tagtype.get(t, 4), t)

    def _geometry(self):
        P, n1 = self.P, self.n1
        x1, w1, D1, Lm, Lp, gL, gR = self.q
        self.Ji, self.Jd, self.w = [], [], []
        for e, nd in enumerate(self.elems):
            p = self.xy[nd]
            if len(nd) == 3:
                xr, xs = 0.5 * (p[1] - p[0]), 0.5 * (p[2] - p[0])
                J = xr[0] * xs[1] - xs[0] * xr[1]
                Ji = np.array([xs[1], -xs[0], -xr[1], xr[0]]) / J
                self.Ji.append(np.tile(Ji, (self.nt, 1)))
                self.Jd.append(np.full(self.nt, J))
                self.w.append(self.t[4] * J)
            else:
                Jis, Js = [], []
                for jj in range(n1):
                    for ii in range(n1):
                        xi, eta = x1[ii], x1[jj]
                        dNx = 0.25 * np.array([-(1 - eta), (1 - eta), (1 + eta), -(1 + eta)])
                        dNe = 0.25 * np.array([-(1 - xi), -(1 + xi), (1 + xi), (1 - xi)])
                        a, b = dNx @ p[:, 0], dNe @ p[:, 0]
                        c, d = dNx @ p[:, 1], dNe @ p[:, 1]
                        J = a * d - b * c
                        Jis.append(np.array([d, -b, -c, a]) / J)
                        Js.append(J)
                self.Ji.append(np.array(Jis))
                self.Jd.append(np.array(Js))
                self.w.append(np.outer(w1, w1).ravel() * np.array(Js))

    def edge_geom(self, e, l):
        nd = self.elems[e]
        nv = len(nd)
        a, b = self.xy[nd[l]], self.xy[nd[(l + 1) % nv]]
        t = b - a
        ln = math.hypot(*t)
        n = np.array([t[1], -t[0]]) / ln
        cen = self.xy[nd].mean(axis=0)
        if n @ (0.5 * (a + b) - cen) < 0:
            n = -n
        return n, ln

    # -- element operators -------------------------------------------------
    def traces(self, e, F):
        """[edges][n1][...] traces of the nodal field F [nsp or nt][...]."""
        n1 = self.n1
        if self.etype[e] == 0:
            L = self.t[2]
            return (L @ F[:self.nt]).reshape(3, n1, *F.shape[1:])
        _, _, _, Lm, Lp, _, _ = self.q
        Fg = F[:self.nsp].reshape(n1, n1, *F.shape[1:])           # [j][i]
        t0 = np.einsum("j,ji...->i...", Lm, Fg)                    # eta = -1, along xi
        t1 = np.einsum("i,ji...->j...", Lp, Fg)                    # xi = +1, along eta
        t2 = np.einsum("j,ji...->i...", Lp, Fg)[::-1]              # eta = +1, reversed
        t3 = np.einsum("i,ji...->j...", Lm, Fg)[::-1]              # xi = -1, reversed
        return np.stack([t0, t1, t2, t3])

    def states_of(self, U):
        return [U[e, :(self.nt if self.etype[e] == 0 else self.nsp)] for e in range(self.E)]

    def face_partner(self, e, l, fp, tr, own):
        """Neighbour value at the point coinciding with (e, l, fp), or the ghost."""
        nb = self.nbr[(e, l)]
        if nb[0] == "bnd":
            return None
        e2, l2, _ = nb
        return tr[e2][l2][self.n1 - 1 - fp]

    def gradient(self, e, Ue, jumps):
        """Corrected physical gradient (Qx, Qy) [npt][4] from face jumps [edges][n1][4]."""
        Ji = self.Ji[e]
        if self.etype[e] == 0:
            Dr, Ds, L, Phi, _ = self.t
            dr = Dr @ Ue
            ds = Ds @ Ue
            jf = jumps.reshape(-1, 4)
            qn = np.repeat(TRI_NREF, self.n1, axis=0)
            dr = dr + Phi @ (jf * qn[:, :1])
            ds = ds + Phi @ (jf * qn[:, 1:])
        else:
            n1 = self.n1
            _, _, D1, _, _, gL, gR = self.q
            Ug = Ue.reshape(n1, n1, 4)
            dr = np.einsum("im,jmv->jiv", D1, Ug)
            ds = np.einsum("jm,miv->jiv", D1, Ug)
            d1, d3, d0, d2 = jumps[1], jumps[3], jumps[0], jumps[2]
            dr = dr + gR[None, :, None] * d1[:, None, :] + gL[None, :, None] * d3[::-1][:, None, :]
            ds = ds + gL[:, None, None] * d0[None, :, :] + gR[:, None, None] * d2[::-1][None, :, :]
            dr, ds = dr.reshape(-1, 4), ds.reshape(-1, 4)
        Qx = Ji[:, 0:1] * dr + Ji[:, 2:3] * ds
        Qy = Ji[:, 1:2] * dr + Ji[:, 3:4] * ds
        return Qx, Qy

    def rhs(self, U):
        g, n1 = self.g, self.n1
        U = np.asarray(U, dtype=np.float64)
        Us = self.states_of(U)
        tr = [self.traces(e, Us[e]) for e in range(self.E)]
        # ghost states / neighbour values per flux point
        other = {}
        for (e, l), nb in self.nbr.items():
            n, ln = self.edge_geom(e, l)
            for fp in range(n1):
                if nb[0] == "bnd":
                    other[(e, l, fp)] = self._ctx.ghost(nb[1], nb[2], tr[e][l][fp], n[0], n[1])
                else:
                    other[(e, l, fp)] = tr[nb[0]][nb[1]][n1 - 1 - fp]
        Q = None
        if self.viscous:
            Q, TQ = [], []
            for e in range(self.E):
                nv = len(self.elems[e])
                jumps = np.array([[0.5 * (other[(e, l, fp)] - tr[e][l][fp]) for fp in range(n1)]
                                  for l in range(nv)])
                Qx, Qy = self.gradient(e, Us[e], jumps)
                Q.append((Qx, Qy))
                TQ.append((self.traces(e, Qx), self.traces(e, Qy)))
        R = np.zeros_like(U)
        for e in range(self.E):
            nv = len(self.elems[e])
            Ue, Ji, Jd = Us[e], self.Ji[e], self.Jd[e]
            rho = Ue[:, 0]
            u, v = Ue[:, 1] / rho, Ue[:, 2] / rho
            p = (g - 1) * (Ue[:, 3] - 0.5 * rho * (u * u + v * v))
            F = np.stack([Ue[:, 1], Ue[:, 1] * u + p, Ue[:, 1] * v, (Ue[:, 3] + p) * u], axis=1)
            G = np.stack([Ue[:, 2], Ue[:, 2] * u, Ue[:, 2] * v + p, (Ue[:, 3] + p) * v], axis=1)
            if self.viscous:
                for k in range(Ue.shape[0]):
                    Fv, Gv = viscous_point(Ue[k], Q[e][0][k], Q[e][1][k], g, self.Re, self.Pr)
                    F[k] -= Fv
                    G[k] -= Gv
            Ft = Jd[:, None] * (Ji[:, 0:1] * F + Ji[:, 1:2] * G)
            Gt = Jd[:, None] * (Ji[:, 2:3] * F + Ji[:, 3:4] * G)
            trF, trG = self.traces(e, Ft), self.traces(e, Gt)
            dF = np.zeros((nv, n1, 4))
            for l in range(nv):
                nb = self.nbr[(e, l)]
                n, ln = self.edge_geom(e, l)
                right = nb[0] != "bnd" and nb[2]
                if right:
                    n = -n          # the face normal: the left element's outward normal
                for fp in range(n1):
                    qo, qn = tr[e][l][fp], other[(e, l, fp)]
                    UL, UR = (qn, qo) if right else (qo, qn)
                    Fc = O.riemann_point(self.riemann, UL, UR, n[0], n[1], g)
                    if self.viscous:
                        Qo = (TQ[e][0][l][fp], TQ[e][1][l][fp])
                        if nb[0] == "bnd":
                            Qn = Qo
                        else:
                            e2, l2, _ = nb
                            Qn = (TQ[e2][0][l2][n1 - 1 - fp], TQ[e2][1][l2][n1 - 1 - fp])
                        Fv, Gv = viscous_point(0.5 * (UL + UR), 0.5 * (Qo[0] + Qn[0]), 0.5 * (Qo[1] + Qn[1]),
                                               g, self.Re, self.Pr)
                        Fvn = Fv * n[0] + Gv * n[1]
                        if nb[0] == "bnd":
                            Fvn = self._ctx.wall_closure(nb[1], nb[2], n[0], n[1], Fvn)
                        Fc = Fc - Fvn
                    if nv == 3:
                        sf = ln / TRI_REFLEN[l]
                        Fn = trF[l][fp] * TRI_NREF[l, 0] + trG[l][fp] * TRI_NREF[l, 1]
                    else:
                        sf = 0.5 * ln
                        Fn = [-trG[0][fp], trF[1][fp], trG[2][fp], -trF[3][fp]][l]
                    dF[l, fp] = (-sf if right else sf) * Fc - Fn
            if nv == 3:
                Dr, Ds, L, Phi, _ = self.t
                div = Dr @ Ft + Ds @ Gt + Phi @ dF.reshape(-1, 4)
                R[e, :self.nt] = -div / Jd[:, None]
            else:
                _, _, D1, _, _, gL, gR = self.q
                Fg, Gg = Ft.reshape(n1, n1, 4), Gt.reshape(n1, n1, 4)
                div = np.einsum("im,jmv->jiv", D1, Fg) + np.einsum("jm,miv->jiv", D1, Gg)
                d1, d3, d2, d0 = dF[1], dF[3], dF[2], dF[0]
                corr = (gR[None, :, None] * d1[:, None, :] - gL[None, :, None] * d3[::-1][:, None, :]
                        + gR[:, None, None] * d2[::-1][None, :, :] - gL[:, None, None] * d0[None, :, :])
                R[e, :self.nsp] = (-(div + corr) / Jd.reshape(n1, n1)[..., None]).reshape(-1, 4)
        return R

    def quadrature_weights(self):
        """[E][nsp] integration weights (w |J|; 0 on unused triangle slots)."""
        W = np.zeros((self.E, self.nsp))
        for e in range(self.E):
            W[e, :len(self.w[e])] = self.w[e]
        return W
