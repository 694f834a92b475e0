"""Physics mode (compat off) on the GPU against the physics oracle: the
conservative FR residual with VCJH corrections, the reference's
Rusanov/Roe/HLLC and every boundary class, FP64.  Bar: 1e-12 relative to the
flux scale, as the compat parity tests."""
import math

import numpy as np
import pytest

from tests import _util as T
from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu
TOL = 1e-12
RIEMANN = ["Rusanov", "Roe", "HLLC"]
FLUX = ["DG", "SD", "HU", "GA"]

# one boundary class per side and tag: bottom slip wall, right outflow,
# top inflow, left isothermal no-slip wall; a symmetry/far-field/adiabatic
# wall variant on a second mesh
BCS_A = [dict(tag=1, type="slipwall"), dict(tag=2, type="outflow", p_static=0.95e5),
         dict(tag=3, type="inflow", p_total=1.2e5, T_total=9.0e4, dir_x=0.6, dir_y=-0.8),
         dict(tag=4, type="wall", T_wall=8.0e4)]
BCS_B = [dict(tag=1, type="symmetry"), dict(tag=2, type="farfield"),
         dict(tag=3, type="wall"), dict(tag=4, type="farfield")]


def case_mesh(bcs, seed=7, n=6):
    names = {b["tag"]: b["type"] for b in bcs}
    return M.structured_quads(n, n, 0.0, 1.0, 0.0, 1.0, 0.15, seed, (1, 2, 3, 4), names)


def make_pair(oracle_mod, mesh, bcs, P, flux, riem, rho=1.2, p=1.0e5, mach=0.4, aoa=10.0):
    prm = make_params(poly_order=P, rho_inf=rho, p_inf=p, Mach=mach, AoA=aoa, flux_type=flux,
                      riemann=riem, compat=False, bcs=bcs, T_inf=8.5e4)
    s = FRSolver(mesh, prm)
    tags = [(b["tag"], L.BC_TYPES[b["type"]], b.get("p_static", 0.0)) for b in bcs]
    orc = oracle_mod.Oracle(mesh, P, 1.4, rho, p, mach, aoa, tags=tags)
    orc.set_physics(FLUX.index(flux), RIEMANN.index(riem), False, 1000.0, 0.72, 8.5e4)
    orc.set_bc_extra([(b["tag"], b.get("p_total", 0.0), b.get("T_total", 0.0), b.get("dir_x", 1.0),
                       b.get("dir_y", 0.0), b.get("T_wall", 0.0)) for b in bcs])
    return s, orc


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("bcs", [BCS_A, BCS_B], ids=["A", "B"])
def test_rhs_matches_physics_oracle(zjlib, oracle_mod, P, riem, bcs):
    mesh = case_mesh(bcs)
    flux = FLUX[(P + RIEMANN.index(riem)) % 4]
    s, orc = make_pair(oracle_mod, mesh, bcs, P, flux, riem)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 31 + P, 1.4, 1.2, 1.0e5, 0.1)
    R = s.rhs(U)
    Ro = orc.rhs_phys(U)
    scale = T.euler_flux_scale(U, orc.geometry()[1])
    assert T.rel_err(R, Ro, scale) <= TOL


@pytest.mark.parametrize("flux", FLUX)
def test_steps_match_physics_oracle(zjlib, oracle_mod, flux):
    mesh = case_mesh(BCS_A)
    s, orc = make_pair(oracle_mod, mesh, BCS_A, 3, flux, "Roe")
    U = M.random_state(mesh.n_elem, 16, 77, 1.4, 1.2, 1.0e5, 0.05)
    s.copyToDevice(U)
    s.advance(2e-8, 3)
    Uo, Ro = orc.step_phys(U, 2e-8, 3)
    assert T.rel_err(s.copyToHost(), Uo, T.euler_flux_scale(Uo)) <= TOL
    no = float(np.sqrt(np.sum(Ro * Ro)))
    assert abs(s.computeResidual() - no) <= 1e-11 * no


@pytest.mark.parametrize("riem", RIEMANN)
def test_freestream_preserved(zjlib, riem):
    mesh = M.structured_quads(8, 8, -1.0, 1.0, -1.0, 1.0, 0.2, 4, (1, 1, 1, 1), {1: "farfield"})
    prm = make_params(poly_order=4, rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=25.0, riemann=riem,
                      compat=False, bcs=[(1, "farfield")])
    s = FRSolver(mesh, prm)
    c = math.sqrt(1.4 * 1.0e5 / 1.2)
    U = np.broadcast_to(M.prim_to_cons(1.2, 0.4 * c * math.cos(math.radians(25.0)),
                                       0.4 * c * math.sin(math.radians(25.0)), 1.0e5, 1.4),
                        s.shape).copy()
    R = s.rhs(U)
    assert np.abs(R).max() <= 1e-11 * (1.0e5 + U[0, 0, 3]) * c


def test_full_size_tgv_roe(zjlib, oracle_mod):
    import os
    mesh = M.tgv_mesh(256, seed=1)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3,
                      riemann="Roe", compat=False, bcs=[(1, "slipwall")])
    s = FRSolver(mesh, prm)
    orc = oracle_mod.Oracle(mesh, 3, 1.4, 1.0, 1.0 / (1.4 * 0.09), 0.3, 0.0,
                            threads=os.cpu_count() or 1)
    orc.set_physics(2, 1)
    U = M.taylor_green(s.solution_point_coords())
    R = s.rhs(U)
    Ro = orc.rhs_phys(U)
    assert T.rel_err(R, Ro, T.euler_flux_scale(U, orc.geometry()[1])) <= TOL
    # discrete conservation of mass and energy in the slip-wall box
    J, _ = orc.geometry()
    w1 = np.polynomial.legendre.leggauss(4)[1]
    w = np.outer(w1, w1).ravel()
    tot = np.einsum("s,es,esv->v", w, J, R)
    scale = np.einsum("s,es,esv->", w, J, np.abs(R))
    assert abs(tot[0]) <= 1e-12 * scale and abs(tot[3]) <= 1e-12 * scale


def test_physics_mode_takes_straight_q2_elements_like_q1(zjlib):
    """A Q2 mesh whose edge and centre nodes sit at the midpoints (straight
    edges) gives the Q1 mesh's physics-mode residual to rounding: the
    per-flux-point normals of the curved-element path reduce to the per-edge
    ones."""
    fine = M.structured_quads(4, 4, -10.0, 10.0, -10.0, 10.0, 0.0, 0, (1, 1, 1, 1), {1: "farfield"})
    q1 = M.structured_quads(2, 2, -10.0, 10.0, -10.0, 10.0, 0.0, 0, (1, 1, 1, 1), {1: "farfield"})
    conn = []
    for ej in range(2):
        for ei in range(2):
            n = lambda i, j: (2 * ej + j) * 5 + (2 * ei + i)
            conn.append([n(0, 0), n(2, 0), n(2, 2), n(0, 2), n(1, 0), n(2, 1), n(1, 2), n(0, 1), n(1, 1)])
    bnd = np.array([[0, 2, 1], [2, 4, 1], [4, 14, 1], [14, 24, 1], [24, 22, 1], [22, 20, 1], [20, 10, 1],
                    [10, 0, 1]], dtype=np.int64)
    q2 = M.QuadMesh(fine.xy, np.array(conn, dtype=np.int64), bnd, {1: "farfield"})
    kw = dict(poly_order=3, compat=False, riemann="Roe", rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=10.0,
              bcs=[(1, "farfield")])
    U = M.random_state(4, 16, 3, 1.4, 1.2, 1.0e5, 0.05)
    R1 = FRSolver(q1, make_params(**kw)).rhs(U)
    R2 = FRSolver(q2, make_params(**kw)).rhs(U)
    assert T.rel_err(R2, R1, T.euler_flux_scale(U) * 0.2) <= 1e-12


# ------------------------------------------------------------ Navier-Stokes --

def make_ns_pair(oracle_mod, mesh, bcs, P, flux, riem, Re=50.0, rho=1.2, p=1.0e5, mach=0.4,
                 aoa=10.0):
    prm = make_params(poly_order=P, rho_inf=rho, p_inf=p, Mach=mach, AoA=aoa, flux_type=flux,
                      riemann=riem, compat=False, viscous=True, Re=Re, Pr=0.72, bcs=bcs,
                      T_inf=8.5e4)
    s = FRSolver(mesh, prm)
    tags = [(b["tag"], L.BC_TYPES[b["type"]], b.get("p_static", 0.0)) for b in bcs]
    orc = oracle_mod.Oracle(mesh, P, 1.4, rho, p, mach, aoa, tags=tags)
    orc.set_physics(FLUX.index(flux), RIEMANN.index(riem), True, Re, 0.72, 8.5e4)
    orc.set_bc_extra([(b["tag"], b.get("p_total", 0.0), b.get("T_total", 0.0), b.get("dir_x", 1.0),
                       b.get("dir_y", 0.0), b.get("T_wall", 0.0)) for b in bcs])
    return s, orc


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("bcs", [BCS_A, BCS_B], ids=["A", "B"])
def test_ns_rhs_matches_physics_oracle(zjlib, oracle_mod, P, riem, bcs):
    mesh = case_mesh(bcs)
    flux = FLUX[(P + 2 * RIEMANN.index(riem)) % 4]
    s, orc = make_ns_pair(oracle_mod, mesh, bcs, P, flux, riem)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 51 + P, 1.4, 1.2, 1.0e5, 0.1)
    R = s.rhs(U)
    Ro = orc.rhs_phys(U)
    scale = T.euler_flux_scale(U, orc.geometry()[1])
    assert T.rel_err(R, Ro, scale) <= TOL


def test_ns_steps_match_physics_oracle(zjlib, oracle_mod):
    mesh = case_mesh(BCS_A)
    s, orc = make_ns_pair(oracle_mod, mesh, BCS_A, 3, "HU", "Roe", Re=20.0)
    U = M.random_state(mesh.n_elem, 16, 79, 1.4, 1.2, 1.0e5, 0.05)
    s.copyToDevice(U)
    s.advance(2e-8, 3)
    Uo, Ro = orc.step_phys(U, 2e-8, 3)
    assert T.rel_err(s.copyToHost(), Uo, T.euler_flux_scale(Uo)) <= TOL
    no = float(np.sqrt(np.sum(Ro * Ro)))
    assert abs(s.computeResidual() - no) <= 1e-11 * no


def test_ns_full_size_tgv(zjlib, oracle_mod):
    """The Taylor-Green configuration of the benchmark (256x256 jittered, P3,
    Roe, Re 5000, Pr 0.72): residual against the oracle at full size."""
    import os
    mesh = M.tgv_mesh(256, seed=1)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      compat=False, viscous=True, Re=5000.0, Pr=0.72, bcs=[(1, "slipwall")])
    s = FRSolver(mesh, prm)
    orc = oracle_mod.Oracle(mesh, 3, 1.4, 1.0, 1.0 / (1.4 * 0.09), 0.3, 0.0,
                            threads=os.cpu_count() or 1)
    orc.set_physics(2, 1, True, 5000.0, 0.72)
    U = M.taylor_green(s.solution_point_coords())
    R = s.rhs(U)
    Ro = orc.rhs_phys(U)
    assert T.rel_err(R, Ro, T.euler_flux_scale(U, orc.geometry()[1])) <= TOL
    # the allocation-free entry point covers the viscous path too
    import ctypes as C
    import torch
    Ud = torch.from_numpy(U).cuda()
    Rd = torch.empty_like(Ud)
    torch.cuda.synchronize()
    code = zjlib.zj_rhs_noalloc(s.h, C.c_void_p(Ud.data_ptr()), C.c_void_p(Rd.data_ptr()))
    assert code == L.ERR_ARG   # 65 536 P3 elements need 3 trace buffers: above the static limit
