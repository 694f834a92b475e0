"""The physics-mode oracle (conservative FR, VCJH, the reference's Riemann
solvers and ghost states).  No reference residual exists for this mode
(parity unpinned at the residual level); its pieces are pinned pointwise to
the reference's own header code and the assembled scheme is checked for the
properties FR must have: freestream preservation on jittered meshes, discrete
conservation, VCJH identities and the design order of accuracy."""
import math
import os

import numpy as np
import pytest

from tests.golden import make_golden as G
from zhijian_b200 import meshgen as M

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def phys():
    return np.load(os.path.join(GOLD, "ref_physics.npz"))


@pytest.mark.parametrize("which", [0, 1, 2])
def test_riemann_solvers_bitwise_vs_reference(oracle_mod, phys, which):
    smp, ref = phys["samples"], phys["out"]
    g = G.PHYS_PARAMS["g"]
    got = np.array([oracle_mod.riemann_point(which, s[:4], s[4:8], s[8], s[9], g) for s in smp])
    assert np.array_equal(got, ref[:, which])


def _ghost_oracle(oracle_mod):
    P_ = G.PHYS_PARAMS
    tags = [(1, 1, 0.0), (2, 1, 0.0), (3, 2, 0.0), (4, 3, 0.0), (5, 4, 0.0), (6, 5, 0.0),
            (7, 6, P_["p_static"])]
    orc = oracle_mod.Oracle(G.mixed_mesh(), 3, P_["g"], P_["rho_inf"], P_["p_inf"], P_["mach"],
                            P_["aoa"], tags=tags)
    orc.set_physics(2, 0, False, 1000.0, 0.72, 300.0)
    orc.set_bc_extra([(2, 0.0, 0.0, 1.0, 0.0, P_["T_wall"]),
                      (6, P_["p_total"], P_["T_total"], P_["dx"], P_["dy"], 0.0)])
    return orc


@pytest.mark.parametrize("k,bct,tag", [(0, 1, 1), (1, 1, 2), (2, 2, 3), (3, 3, 4), (4, 4, 5),
                                       (5, 5, 6), (6, 6, 7)])
def test_ghost_states_bitwise_vs_reference(oracle_mod, phys, k, bct, tag):
    smp, ref = phys["samples"], phys["out"]
    orc = _ghost_oracle(oracle_mod)
    got = np.array([orc.ghost(bct, tag, s[:4], s[8], s[9]) for s in smp])
    assert np.array_equal(got, ref[:, 3 + k])


@pytest.fixture(scope="module")
def visc():
    return np.load(os.path.join(GOLD, "ref_viscous.npz"))


def test_viscous_flux_bitwise_vs_reference_header(oracle_mod, visc):
    """The oracle's viscous arithmetic (velocity and temperature gradients,
    Stokes stresses, heat flux, the average-state common flux) under the
    header's Sutherland law against ViscousFlux::fluxX / fluxY and
    BR2Scheme::commonFlux (navierstokes.hpp:52-96, 166-201) compiled from the
    reference: bit for bit on 256 states (both temperature regimes)."""
    smp, ref = visc["samples"], visc["out"]
    V = G.VISC_PARAMS
    for q, r in zip(smp, ref):
        F, Gv = oracle_mod.viscous_point(1, q[0:4], q[4:8], q[8:12], V["g"], V["Re"], V["Pr"])
        C = oracle_mod.common_viscous_point(1, q[0:4], q[12:16], q[4:8], q[8:12], q[16:20], q[20:24],
                                            q[24], q[25], V["g"], V["Re"], V["Pr"])
        assert np.array_equal(F, r[0]) and np.array_equal(Gv, r[1]) and np.array_equal(C, r[2])


def test_viscous_flux_vs_reference_kernel(oracle_mod):
    """The oracle's viscous flux under the kernel's law (mu = T^0.7/Re, the
    law of every residual here) against the reference's own
    computeViscousFluxSPKernel (kernels.cu:719-807) run on a B200
    (tests/golden/make_golden.py gpu): within 1e-13 of each record's flux
    scale -- the reference kernel is compiled with FMA contraction, the
    oracle without."""
    d = np.load(os.path.join(GOLD, "ref_viscous_kernel.npz"))
    smp = d["samples"]
    assert np.array_equal(smp, G.visc_samples())
    V = G.VISC_PARAMS
    worst = 0.0
    for q, fr, gr in zip(smp, d["Fv"], d["Gv"]):
        F, Gv = oracle_mod.viscous_point(0, q[0:4], q[4:8], q[8:12], V["g"], V["Re"], V["Pr"])
        scale = max(np.abs(fr).max(), np.abs(gr).max())
        worst = max(worst, np.abs(F - fr).max() / scale, np.abs(Gv - gr).max() / scale)
    assert worst <= 1e-13


def _legendre(n, x):
    return np.polynomial.legendre.legval(x, [0] * n + [1])


def _dlegendre(n, x):
    return np.polynomial.legendre.legval(x, np.polynomial.legendre.legder([0] * n + [1]))


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
def test_vcjh_identities(oracle_mod, P):
    orc = oracle_mod.Oracle(M.vortex_mesh(2), P)
    pts = orc.operators()["pts"]
    w = np.polynomial.legendre.leggauss(P + 1)[1]
    ref_corr = np.load(os.path.join(GOLD, "ref_operators.npz"))[f"P{P}_corr"]
    for ft in range(4):
        orc.set_physics(ft)
        gL, gR = orc.vcjh()
        # g_R rises from 0 to 1 and g_L falls from 1 to 0 on [-1, 1]
        assert abs(np.dot(w, gR) - 1.0) < 1e-13 and abs(np.dot(w, gL) + 1.0) < 1e-13
        if ft == 0:   # DG = the right/left Radau polynomials the reference always uses
            assert np.array_equal(gR, ref_corr[1][:P + 1])
            assert np.array_equal(gL, ref_corr[3][:P + 1])
        if ft == 1:   # SD: g_R = (1+x)/2 P_p(x)  (Huynh's g_Ga)
            d = 0.5 * _legendre(P, pts) + 0.5 * (1 + pts) * _dlegendre(P, pts)
            assert np.allclose(gR, d, atol=1e-12)
        if ft == 2:   # Huynh g2 = (p R_{R,p+1} + (p+1) R_{R,p}) / (2p+1)
            RR = lambda k, x: 0.5 * (_dlegendre(k, x) + _dlegendre(k - 1, x))
            d = (P * RR(P + 1, pts) + (P + 1) * RR(P, pts)) / (2 * P + 1)
            assert np.allclose(gR, d, atol=1e-12)


def _farfield_box(n, jitter, seed, P, rho=1.2, p=1.0e5, mach=0.4, aoa=25.0):
    mesh = M.structured_quads(n, n, -1.0, 1.0, -1.0, 1.0, jitter, seed, (1, 1, 1, 1),
                              {1: "farfield"})
    return mesh, dict(gamma=1.4, rho_inf=rho, p_inf=p, Mach=mach, AoA=aoa)


@pytest.mark.parametrize("riemann", [0, 1, 2])
@pytest.mark.parametrize("P", [1, 3, 5])
def test_freestream_preserved_on_jittered_mesh(oracle_mod, P, riemann):
    mesh, kw = _farfield_box(6, 0.2, 4, P)
    orc = oracle_mod.Oracle(mesh, P, **kw)
    orc.set_physics(2, riemann)
    c = math.sqrt(1.4 * kw["p_inf"] / kw["rho_inf"])
    u = kw["Mach"] * c * math.cos(math.radians(kw["AoA"]))
    v = kw["Mach"] * c * math.sin(math.radians(kw["AoA"]))
    U = np.broadcast_to(M.prim_to_cons(kw["rho_inf"], u, v, kw["p_inf"], 1.4),
                        (orc.n_elem, orc.nsp, 4)).copy()
    R = orc.rhs_phys(U)
    flux = (kw["p_inf"] + U[0, 0, 3]) * c
    assert np.abs(R).max() <= 1e-11 * flux


@pytest.mark.parametrize("riemann", [0, 1, 2])
def test_mass_and_energy_conserved_in_slip_wall_box(oracle_mod, riemann):
    P = 3
    mesh = M.tgv_mesh(8, seed=5)
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.0, 1.0 / (1.4 * 0.09), 0.3, 0.0)
    orc.set_physics(2, riemann)
    U = M.taylor_green(orc.sp_coords())
    R = orc.rhs_phys(U)
    J, _ = orc.geometry()
    w1 = np.polynomial.legendre.leggauss(P + 1)[1]
    w = np.outer(w1, w1).ravel()           # sp = j*(P+1) + i
    tot = np.einsum("s,es,esv->v", w, J, R)
    scale = np.einsum("s,es,esv->", w, J, np.abs(R))   # all variables: a flux-sized scale
    assert abs(tot[0]) <= 1e-13 * scale
    assert abs(tot[3]) <= 1e-13 * scale


@pytest.mark.parametrize("P", [2, 3])
def test_design_order_on_the_isentropic_vortex(oracle_mod, P):
    """Residual error against the exact dU/dt = -u_inf dU/dx of the advected
    (exact) isentropic vortex, in the vortex core, on two uniform meshes:
    observed order >= P - 0.5."""
    errs = []
    for n in (16, 32):
        mesh = M.structured_quads(n, n, -5.0, 5.0, -5.0, 5.0, 0.0, 0, (1, 1, 1, 1),
                                  {1: "farfield"})
        orc = oracle_mod.Oracle(mesh, P, 1.4, 1.0, 1.0, 0.5 / math.sqrt(1.4), 0.0)
        orc.set_physics(2, 1)
        xy = orc.sp_coords()
        U = M.shu_vortex(xy, 1.4)
        R = orc.rhs_phys(U)
        h = 1e-5
        dUdx = (M.shu_vortex(xy + [h, 0.0], 1.4) - M.shu_vortex(xy - [h, 0.0], 1.4)) / (2 * h)
        exact = -0.5 * dUdx
        core = (np.hypot(xy[..., 0], xy[..., 1]) < 2.5)
        errs.append(np.abs(R - exact)[core].max())
    order = math.log2(errs[0] / errs[1])
    assert order >= P - 0.5, (errs, order)


# ------------------------------------------------------------ curved elements --

def _uniform_state(orc, rho=1.2, p=1.0e5, mach=0.4, aoa=25.0):
    c = math.sqrt(1.4 * p / rho)
    u, v = mach * c * math.cos(math.radians(aoa)), mach * c * math.sin(math.radians(aoa))
    U = np.broadcast_to(M.prim_to_cons(rho, u, v, p, 1.4), (orc.n_elem, orc.nsp, 4)).copy()
    return U, (p + U[0, 0, 3]) * c


@pytest.mark.parametrize("order,P", [(2, 2), (2, 3), (2, 5), (4, 4), (4, 5)])
def test_freestream_preserved_on_curved_mesh(oracle_mod, order, P):
    """Curved quads (every interior edge bent, far field all round): the
    per-flux-point normals and edge Jacobians keep a uniform flow steady when
    the solution order reaches the geometric order (the metric terms J xi_x =
    y_eta ... are then polynomials the operators differentiate exactly)."""
    mesh = M.curved_quads(5, 5, order, -1.0, 1.0, -1.0, 1.0, 0.04)
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 25.0)
    orc.set_physics(2, 1)
    U, flux = _uniform_state(orc)
    assert np.abs(orc.rhs_phys(U)).max() <= 1e-12 * flux


def test_freestream_not_preserved_below_the_geometric_order(oracle_mod):
    """Q4 geometry at P3: the metric terms are not degree-3 polynomials, so a
    uniform flow is not steady (the expected limit of any FR scheme)."""
    mesh = M.curved_quads(5, 5, 4, -1.0, 1.0, -1.0, 1.0, 0.04)
    orc = oracle_mod.Oracle(mesh, 3, 1.4, 1.2, 1.0e5, 0.4, 25.0)
    orc.set_physics(2, 1)
    U, flux = _uniform_state(orc)
    assert np.abs(orc.rhs_phys(U)).max() > 1e-6 * flux


@pytest.mark.parametrize("name,P", [("quad2_v41", 2), ("quad2_v41", 3), ("quad2_v41", 4), ("quad2_v41", 5)])
def test_freestream_on_curved_gmsh_fixtures(oracle_mod, name, P):
    """The curved Q2 Gmsh fixture (bent and jittered, read by the library's
    reader, which matches the reference's) with far field on every boundary
    group: a uniform flow stays steady in physics mode.  (The Q4 fixture,
    quad4_v22, jitters its 25 nodes per element independently, which turns
    its Jacobian negative at some solution points; the library refuses it
    for computation, and it serves the reader tests only.)"""
    from zhijian_b200.gmsh import read_gmsh
    mesh = read_gmsh(os.path.join(GOLD, "gmsh", name + ".msh")).to_quad_mesh()
    tags = [(t, 4, 0.0) for t in sorted(mesh.tag_names)]
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 25.0, tags=tags)
    orc.set_physics(2, 1)
    U, flux = _uniform_state(orc)
    assert np.abs(orc.rhs_phys(U)).max() <= 1e-12 * flux


@pytest.mark.parametrize("P", [2, 3])
def test_design_order_on_curved_mesh(oracle_mod, P):
    """The exact isentropic vortex on curved Q2 meshes of [-5, 5]^2 (16^2 and
    32^2 elements): the residual error in the core converges at order
    >= P - 0.5 (measured 1.8 at P2, 2.7 at P3, 3.8 at P4)."""
    errs = []
    for n in (16, 32):
        mesh = M.curved_quads(n, n, 2, -5.0, 5.0, -5.0, 5.0, 0.03)
        orc = oracle_mod.Oracle(mesh, P, 1.4, 1.0, 1.0, 0.5 / math.sqrt(1.4), 0.0, threads=os.cpu_count() or 1)
        orc.set_physics(2, 1)
        xy = orc.sp_coords()
        R = orc.rhs_phys(M.shu_vortex(xy, 1.4))
        h = 1e-5
        exact = -0.5 * (M.shu_vortex(xy + [h, 0.0], 1.4) - M.shu_vortex(xy - [h, 0.0], 1.4)) / (2 * h)
        core = (np.hypot(xy[..., 0], xy[..., 1]) < 2.5)
        errs.append(np.abs(R - exact)[core].max())
    order = math.log2(errs[0] / errs[1])
    assert order >= P - 0.5, (errs, order)


# ---------------------------------------------------------------- Navier-Stokes --

def _mms_prim(x, y):
    rho = 1.0 + 0.1 * np.sin(2.0 * x + y)
    u = 0.3 + 0.1 * np.cos(3.0 * y)
    v = 0.2 * np.sin(2.0 * x)
    p = (1.0 + 0.1 * np.cos(x - 2.0 * y)) / 1.4
    return rho, u, v, p


def _mms_U(x, y):
    rho, u, v, p = _mms_prim(x, y)
    # conserved variables; complex inputs stay complex (complex-step derivatives)
    return np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)], axis=-1)


def _grad_U(x, y):
    """Exact gradients by complex step."""
    h = 1e-30
    dx = np.imag(_mms_U(x + 1j * h, y + 0j)) / h
    dy = np.imag(_mms_U(x + 0j, y + 1j * h)) / h
    return dx, dy


def _total_flux(oracle_mod, x, y, Re, Pr):
    import ctypes as C
    U = _mms_U(x, y)
    dx, dy = _grad_U(x, y)
    F = np.empty(U.shape)
    G = np.empty(U.shape)
    lib = oracle_mod.lib()
    lib.orc_viscous_flux.argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_double] * 3 + \
        [C.POINTER(C.c_double)] * 2
    d = oracle_mod._d
    flat = U.reshape(-1, 4)
    for k in range(flat.shape[0]):
        s = np.ascontiguousarray(flat[k])
        a = np.ascontiguousarray(dx.reshape(-1, 4)[k])
        b = np.ascontiguousarray(dy.reshape(-1, 4)[k])
        fv, gv = np.empty(4), np.empty(4)
        lib.orc_viscous_flux(d(s), d(a), d(b), 1.4, Re, Pr, d(fv), d(gv))
        rho, u, v = s[0], s[1] / s[0], s[2] / s[0]
        pr = 0.4 * (s[3] - 0.5 * rho * (u * u + v * v))
        Fi = np.array([s[1], s[1] * u + pr, s[1] * v, (s[3] + pr) * u])
        Gi = np.array([s[2], s[2] * u, s[2] * v + pr, (s[3] + pr) * v])
        F.reshape(-1, 4)[k] = Fi - fv
        G.reshape(-1, 4)[k] = Gi - gv
    return F, G


def _exact_ns_rhs(oracle_mod, xy, Re, Pr, h=1e-3):
    x, y = xy[..., 0], xy[..., 1]
    c = [(-2, 1.0 / 12.0), (-1, -8.0 / 12.0), (1, 8.0 / 12.0), (2, -1.0 / 12.0)]
    div = 0.0
    for k, w in c:
        F, _ = _total_flux(oracle_mod, x + k * h, y, Re, Pr)
        _, G = _total_flux(oracle_mod, x, y + k * h, Re, Pr)
        div = div + w * (F + G) / h
    return -div


@pytest.mark.parametrize("P", [2, 3])
def test_navier_stokes_design_order(oracle_mod, P):
    Re, Pr = 20.0, 0.72
    errs = []
    for n in (6, 12):
        mesh = M.structured_quads(n, n, 0.0, 1.0, 0.0, 1.0, 0.0, 0, (1, 1, 1, 1), {1: "farfield"})
        orc = oracle_mod.Oracle(mesh, P, 1.4, 1.0, 1.0 / 1.4, 0.3, 0.0)
        orc.set_physics(2, 1, True, Re, Pr, 300.0)
        xy = orc.sp_coords()
        R = orc.rhs_phys(_mms_U(xy[..., 0], xy[..., 1]))
        ex = _exact_ns_rhs(oracle_mod, xy, Re, Pr)
        cx, cy = xy[..., 0].mean(1), xy[..., 1].mean(1)
        inner = (cx > 0.3) & (cx < 0.7) & (cy > 0.3) & (cy < 0.7)
        errs.append(np.abs(R - ex)[inner].max())
    # the central (BR1-type) viscous flux of navierstokes.hpp:177-204 makes the
    # pointwise residual error O(h^(P-1)) for second derivatives
    order = math.log2(errs[0] / errs[1])
    assert order >= P - 1.3, (errs, order)


def test_navier_stokes_freestream_and_mass(oracle_mod):
    mesh, kw = _farfield_box(6, 0.2, 4, 3)
    orc = oracle_mod.Oracle(mesh, 3, **kw)
    orc.set_physics(2, 1, True, 50.0, 0.72, 300.0)
    c = math.sqrt(1.4 * kw["p_inf"] / kw["rho_inf"])
    U = np.broadcast_to(M.prim_to_cons(kw["rho_inf"], kw["Mach"] * c * math.cos(math.radians(25.0)),
                                       kw["Mach"] * c * math.sin(math.radians(25.0)), kw["p_inf"], 1.4),
                        (orc.n_elem, orc.nsp, 4)).copy()
    assert np.abs(orc.rhs_phys(U)).max() <= 1e-11 * (kw["p_inf"] + U[0, 0, 3]) * c
    box = M.tgv_mesh(8, seed=5)
    orc = oracle_mod.Oracle(box, 3, 1.4, 1.0, 1.0 / (1.4 * 0.09), 0.3, 0.0)
    orc.set_physics(2, 1, True, 100.0, 0.72, 300.0)
    R = orc.rhs_phys(M.taylor_green(orc.sp_coords()))
    J, _ = orc.geometry()
    w1 = np.polynomial.legendre.leggauss(4)[1]
    w = np.outer(w1, w1).ravel()
    tot = np.einsum("s,es,esv->v", w, J, R)
    scale = np.einsum("s,es,esv->", w, J, np.abs(R))
    assert abs(tot[0]) <= 1e-13 * scale
