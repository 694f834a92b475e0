"""Curved elements (geometric order 2 and 4) in physics mode on the GPU:
the conservative face term takes the face normal and the edge Jacobian of
every flux point (zj_solver builds them from the element mapping, the shape
functions of basis.cpp:717-847), against the oracle, which computes them
independently.

Bars: FP64 1e-12 of the flux scale per residual and per three steps (the
physics tests' bar); the precision form 1e-5 and the split-BF16 form 3e-5
(their own bars); a uniform flow stays steady to 1e-12 of the flux where the
solution order reaches the geometric order."""
import math
import os

import numpy as np
import pytest

from tests import _util as T
from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params
from tests.test_physics_gpu import BCS_A, BCS_B, FLUX, RIEMANN

pytestmark = pytest.mark.gpu
GM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gmsh")
KW = dict(rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=10.0, T_inf=8.5e4)


def curved_mesh(order, bcs, n=5):
    names = {b["tag"]: b["type"] for b in bcs}
    return M.curved_quads(n, n, order, 0.0, 1.0, 0.0, 1.0, 0.04, (1, 2, 3, 4), names)


def pair(oracle_mod, mesh, bcs, P, flux, riem, viscous, precision="fp64", Re=50.0):
    kw = dict(poly_order=P, flux_type=flux, riemann=riem, compat=False, viscous=viscous, Re=Re, Pr=0.72,
              bcs=bcs, **KW)
    s = FRSolver(mesh, make_params(precision=precision, **kw))
    tags = [(b["tag"], L.BC_TYPES[b["type"]], b.get("p_static", 0.0)) for b in bcs]
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 10.0, tags=tags)
    orc.set_physics(FLUX.index(flux), RIEMANN.index(riem), viscous, Re, 0.72, 8.5e4)
    orc.set_bc_extra([(b["tag"], b.get("p_total", 0.0), b.get("T_total", 0.0), b.get("dir_x", 1.0),
                       b.get("dir_y", 0.0), b.get("T_wall", 0.0)) for b in bcs])
    return s, orc


@pytest.mark.parametrize("order,P", [(2, 2), (2, 3), (2, 4), (2, 5), (4, 3), (4, 4), (4, 5)])
@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("viscous", [False, True], ids=["euler", "ns"])
def test_curved_rhs_against_oracle(zjlib, oracle_mod, order, P, riem, viscous):
    bcs = BCS_A if (P + RIEMANN.index(riem)) % 2 else BCS_B
    mesh = curved_mesh(order, bcs)
    flux = FLUX[(P + order + RIEMANN.index(riem)) % 4]
    s, orc = pair(oracle_mod, mesh, bcs, P, flux, riem, viscous)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 61 + P, 1.4, 1.2, 1.0e5, 0.05)
    R, Ro = s.rhs(U), orc.rhs_phys(U)
    assert T.rel_err(R, Ro, T.euler_flux_scale(U, orc.geometry()[1])) <= 1e-12


@pytest.mark.parametrize("order,P", [(2, 3), (4, 4)])
def test_curved_steps_against_oracle(zjlib, oracle_mod, order, P):
    mesh = curved_mesh(order, BCS_A)
    s, orc = pair(oracle_mod, mesh, BCS_A, P, "HU", "Roe", True)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 7, 1.4, 1.2, 1.0e5, 0.05)
    s.copyToDevice(U)
    s.advance(2e-8, 3)
    Uo, _ = orc.step_phys(U, 2e-8, 3)
    assert T.rel_err(s.copyToHost(), Uo, T.euler_flux_scale(Uo)) <= 1e-12


@pytest.mark.parametrize("precision,tol", [("mixed", 1e-5), ("split_bf16", 3e-5)])
@pytest.mark.parametrize("P", [4, 5])
def test_curved_precision_forms_against_oracle(zjlib, oracle_mod, precision, tol, P):
    mesh = curved_mesh(2, BCS_B, n=6)
    s, orc = pair(oracle_mod, mesh, BCS_B, P, "GA", "HLLC", True, precision=precision)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 13, 1.4, 1.2, 1.0e5, 0.05)
    assert T.rel_err(s.rhs(U), orc.rhs_phys(U), T.euler_flux_scale(U, orc.geometry()[1])) <= tol


@pytest.mark.parametrize("order,P", [(2, 2), (2, 4), (4, 4), (4, 5)])
def test_curved_freestream_on_gpu(zjlib, oracle_mod, order, P):
    """A uniform flow on curved quads with far field all round: steady to
    1e-12 of the flux scale (flux x largest metric term) in FP64; in FP32 to
    3e-5 of it -- the uniform state's face flux is evaluated two ways there
    (the Roe flux of two equal states, the reference state's Euler flux),
    which differ by a few FP32 ulps, and the correction derivatives at the
    edges (about (P+1)^2 / 2) amplify them."""
    mesh = M.curved_quads(6, 6, order, -1.0, 1.0, -1.0, 1.0, 0.04)
    metric = float(np.abs(oracle_mod.Oracle(mesh, P).geometry()[1]).max())
    for precision, tol in (("fp64", 1e-12), ("mixed", 3e-5)):
        s = FRSolver(mesh, make_params(poly_order=P, compat=False, viscous=True, Re=100.0, riemann="Roe",
                                       bcs=[(1, "farfield")], precision=precision, **KW))
        c = math.sqrt(1.4 * 1.0e5 / 1.2)
        u, v = 0.4 * c * math.cos(math.radians(10.0)), 0.4 * c * math.sin(math.radians(10.0))
        U = np.broadcast_to(M.prim_to_cons(1.2, u, v, 1.0e5, 1.4), (s.n_elem, s.n_sp, 4)).copy()
        flux = (1.0e5 + U[0, 0, 3]) * c
        assert np.abs(s.rhs(U)).max() <= tol * flux * metric


@pytest.mark.parametrize("name,P", [("quad2_v41", 2), ("quad2_v41", 3), ("quad2_v41", 5)])
def test_curved_gmsh_files_in_physics_mode(zjlib, oracle_mod, name, P):
    """The curved Q2 Gmsh fixture (bent and jittered), solvers created from
    the file in physics mode (Navier-Stokes, boundary types from the physical
    names): the file and the arrays give the same residual, within 1e-12 of
    the oracle."""
    from zhijian_b200.gmsh import read_gmsh
    path = os.path.join(GM, name + ".msh")
    mesh = read_gmsh(path).to_quad_mesh()
    kw = dict(poly_order=P, compat=False, viscous=True, Re=50.0, Pr=0.72, riemann="Roe", flux_type="SD", **KW)
    s_file = FRSolver.from_gmsh(path, make_params(**kw))
    s_arr = FRSolver(mesh, make_params(bcs=[(t, n) for t, n in sorted(mesh.tag_names.items())], **kw))
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 23, 1.4, 1.2, 1.0e5, 0.05)
    R = s_file.rhs(U)
    assert np.array_equal(R, s_arr.rhs(U))
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 10.0)
    orc.set_physics(1, 1, True, 50.0, 0.72, 8.5e4)
    assert T.rel_err(R, orc.rhs_phys(U), T.euler_flux_scale(U, orc.geometry()[1])) <= 1e-12


def test_differentiation_refused_on_curved_meshes(zjlib):
    import ctypes as C
    import torch
    mesh = M.curved_quads(3, 3, 2, 0.0, 1.0, 0.0, 1.0, 0.04)
    s = FRSolver(mesh, make_params(poly_order=2, compat=False, viscous=True, bcs=[(1, "farfield")], **KW))
    U = torch.zeros(s.n_elem * s.n_sp * 4, dtype=torch.float64, device="cuda")
    code = zjlib.zj_rhs_vjp(s.h, C.c_void_p(U.data_ptr()), C.c_void_p(U.data_ptr()),
                            C.c_void_p(U.data_ptr()), None)
    assert code == L.ERR_UNSUPPORTED
