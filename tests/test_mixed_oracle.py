"""The numpy oracle of meshes with triangles (oracle/mixed_oracle.py), on the
CPU: its quadrilateral path equals the C physics oracle, its triangle
operators are exact on polynomials of degree P, its correction fields
conserve, and the residual preserves a free stream on a mixed mesh."""
import math
import os

import numpy as np
import pytest

from oracle import mixed_oracle as MO
from tests import _util as T
from zhijian_b200 import meshgen as M

BCS = [(1, "farfield")]


def small_mixed(n=4, seed=11, frac=0.5):
    q = M.structured_quads(n, n, 0.0, 1.0, 0.0, 1.0, 0.15, 5, (1, 1, 1, 1), {1: "farfield"})
    return M.split_quads(q, frac, seed)


GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
def test_triangle_points_pinned_to_reference(P):
    """The triangle solution points are the reference's
    (SolutionPoints::getTriangle, basis.cpp:391-417, recorded from its own
    build in ref_triangle.npz): the collapsed map of the (P+1)-point
    Gauss-Legendre rule, row j taking the first P+1-j points.  The
    reference's triangle interpolation, differentiation and correction
    operators (FROperators::initTriangle, basis.cpp:615-668) are all zero:
    there is no reference triangle residual to pin against, so the
    operators here are checked by exactness and conservation instead."""
    ref = np.load(os.path.join(GOLDEN, "ref_triangle.npz"))
    gl = np.load(os.path.join(GOLDEN, "ref_operators.npz"))[f"P{P}_pts"]
    xi, eta = [], []
    for j in range(P + 1):
        for i in range(P + 1 - j):
            sc, tc = 0.5 * (1.0 + gl[i]), 0.5 * (1.0 + gl[j])
            xi.append(sc * (1.0 - tc))
            eta.append(tc)
    assert np.array_equal(np.array(xi), ref[f"P{P}_xi"])
    assert np.array_equal(np.array(eta), ref[f"P{P}_eta"])
    r, s = MO.tri_points(P)
    assert np.abs(0.5 * (r + 1.0) - ref[f"P{P}_xi"]).max() <= 1e-15      # numpy leggauss rounding
    assert np.abs(0.5 * (s + 1.0) - ref[f"P{P}_eta"]).max() <= 1e-15
    for e in range(3):
        assert np.array_equal(ref[f"P{P}_fp_loc"][e], 0.5 * (1.0 + gl))
    for k in ("interp", "diff_xi", "diff_eta", "corr"):
        assert not ref[f"P{P}_{k}"].any()


@pytest.mark.parametrize("P", [1, 2, 3, 4])
def test_triangle_operators_exact(P):
    Dr, Ds, L, Phi, w = MO.tri_operators(P, 2)
    r, s = MO.tri_points(P)
    fr, fs, g, gw = MO.tri_flux_points(P)
    for a in range(P + 1):
        for b in range(P + 1 - a):
            f = r ** a * s ** b
            assert np.allclose(Dr @ f, a * r ** max(a - 1, 0) * s ** b if a else 0 * r, atol=1e-11)
            assert np.allclose(Ds @ f, b * r ** a * s ** max(b - 1, 0) if b else 0 * r, atol=1e-11)
            assert np.allclose(L @ f, fr ** a * fs ** b, atol=1e-11)
    assert abs(w.sum() - 2.0) < 1e-13                      # area of the reference triangle
    # conservation of the correction fields: int phi_{f,j} = |edge_f|/2 w_j
    for f in range(3):
        for j in range(P + 1):
            assert abs(w @ Phi[:, f * (P + 1) + j] - 0.5 * MO.TRI_REFLEN[f] * gw[j]) < 1e-12


@pytest.mark.parametrize("viscous", [False, True], ids=["euler", "ns"])
def test_quad_path_equals_c_oracle(oracle_mod, viscous):
    mesh = M.structured_quads(4, 3, 0.0, 1.0, 0.0, 0.8, 0.15, 3, (1, 1, 1, 1), {1: "farfield"})
    P = 3
    mo = MO.MixedOracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 10.0, flux_type=1, riemann=1, viscous=viscous,
                        Re=50.0, Pr=0.72, T_inf=8.5e4)
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 10.0)
    orc.set_physics(1, 1, viscous, 50.0, 0.72, 8.5e4)
    U = M.random_state(mesh.n_elem, 16, 3, 1.4, 1.2, 1.0e5, 0.05)
    Ro = orc.rhs_phys(U)
    Rm = mo.rhs(U)
    assert T.rel_err(Rm, Ro, T.euler_flux_scale(U, orc.geometry()[1])) <= 1e-12


@pytest.mark.parametrize("P", [1, 2, 3])
def test_mixed_free_stream(P):
    mesh = small_mixed()
    c = math.sqrt(1.4 * 1.0e5 / 1.2)
    mo = MO.MixedOracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 25.0, flux_type=2, riemann=1)
    u = 0.4 * c * math.cos(math.radians(25.0)), 0.4 * c * math.sin(math.radians(25.0))
    U = np.broadcast_to(M.prim_to_cons(1.2, u[0], u[1], 1.0e5, 1.4), (mesh.n_elem, (P + 1) ** 2, 4)).copy()
    R = mo.rhs(U)
    assert np.abs(R).max() <= 1e-10 * (1.0e5 + U[0, 0, 3]) * c


def vortex_and_rate(xy, gamma=1.4, beta=5.0, u_inf=0.5):
    """Exact advecting vortex (p_inf = 1) and its time derivative
    dU/dt = -u_inf dU/dx (pure translation), by complex-step differences."""
    def state(x):
        r2 = x[..., 0] ** 2 + x[..., 1] ** 2
        f = beta / (2 * math.pi) * np.exp(0.5 * (1 - r2))
        Tm = 1 - (gamma - 1) * beta ** 2 / (8 * gamma * math.pi ** 2) * np.exp(1 - r2)
        rho = Tm ** (1 / (gamma - 1))
        u, v, p = u_inf - f * x[..., 1], f * x[..., 0], rho ** gamma
        return np.stack([rho, rho * u, rho * v, p / (gamma - 1) + 0.5 * rho * (u * u + v * v)], axis=-1)
    h = 1e-20
    xc = xy.astype(complex)
    xc[..., 0] += 1j * h
    dUdx = state(xc).imag / h
    return state(xy), -u_inf * dUdx


@pytest.mark.parametrize("P", [2, 3])
def test_mixed_vortex_consistency_order(P):
    errs = []
    for n in (4, 8, 16):
        q = M.structured_quads(n, n, -5.0, 5.0, -5.0, 5.0, 0.1, 7, (1, 1, 1, 1), {1: "farfield"})
        mesh = M.split_quads(q, 0.5, 13)
        mo = MO.MixedOracle(mesh, P, 1.4, 1.0, 1.0, 0.5 / math.sqrt(1.4), 0.0, flux_type=2, riemann=1)
        xy = np.zeros((mesh.n_elem, (P + 1) ** 2, 2))
        rr, ss = MO.tri_points(P)
        g, _ = np.polynomial.legendre.leggauss(P + 1)
        for e in range(mesh.n_elem):
            nd = mesh.xy[mesh.element(e)]
            if len(nd) == 3:
                w0, w1, w2 = -0.5 * (rr + ss), 0.5 * (1 + rr), 0.5 * (1 + ss)
                xy[e, :len(rr)] = np.outer(w0, nd[0]) + np.outer(w1, nd[1]) + np.outer(w2, nd[2])
            else:
                xi, eta = np.meshgrid(g, g)
                xi, eta = xi.ravel(), eta.ravel()
                N = 0.25 * np.stack([(1 - xi) * (1 - eta), (1 + xi) * (1 - eta), (1 + xi) * (1 + eta),
                                     (1 - xi) * (1 + eta)], axis=1)
                xy[e] = N @ nd
        U, dUdt = vortex_and_rate(xy)
        R = mo.rhs(U)
        W = mo.quadrature_weights()
        # interior elements only (the far-field ghost of a vortex is not exact)
        cen = np.array([mesh.xy[mesh.element(e)].mean(axis=0) for e in range(mesh.n_elem)])
        inner = np.abs(cen).max(axis=1) < 3.5
        d = (R - dUdt)[inner]
        errs.append(math.sqrt(float(np.sum(W[inner][..., None] * d * d))))
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    print("P", P, "errors", errs, "rates", rates)
    assert rates[-1] >= P - 0.6
