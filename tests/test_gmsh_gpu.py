"""Solvers created from Gmsh files (zj_solver_create_from_gmsh): the residual
equals the residual of the same mesh given as arrays, and the oracle's, in
compat mode (Q1, curved Q2, serendipity) and in physics mode (Navier-Stokes on
Q1, and on a file of triangles and quads against the mixed-mesh oracle).
Boundary types come from the files' physical names."""
import os

import numpy as np
import pytest

from tests import _util as T
from zhijian_b200 import meshgen as M
from zhijian_b200.gmsh import read_gmsh
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu
GM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "gmsh")
KW = dict(rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=10.0, T_inf=8.5e4)


def pair(name, P, **kw):
    path = os.path.join(GM, name + ".msh")
    mesh = read_gmsh(path).to_quad_mesh()
    bcs = [(t, n) for t, n in sorted(mesh.tag_names.items())]
    s_file = FRSolver.from_gmsh(path, make_params(poly_order=P, **KW, **kw))
    s_arr = FRSolver(mesh, make_params(poly_order=P, bcs=bcs, **KW, **kw))
    return s_file, s_arr, mesh


@pytest.mark.parametrize("name,P", [("quad_v22", 3), ("quad_v41", 2), ("quad2_v41", 3),
                                    ("serendipity_v22", 2)])
def test_compat_from_gmsh(zjlib, oracle_mod, name, P):
    s_file, s_arr, mesh = pair(name, P)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 5 + P, 1.4, 1.2, 1.0e5, 0.05)
    R = s_file.rhs(U)
    assert np.array_equal(R, s_arr.rhs(U))
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 10.0)
    Ro = orc.rhs(U)
    assert T.rel_err(R, Ro, T.euler_flux_scale(U, orc.geometry()[1])) <= 1e-12


def test_physics_ns_from_gmsh(zjlib, oracle_mod):
    s_file, s_arr, mesh = pair("quad_v41", 3, compat=False, viscous=True, Re=50.0, Pr=0.72,
                               riemann="Roe", flux_type="SD")
    U = M.random_state(mesh.n_elem, 16, 17, 1.4, 1.2, 1.0e5, 0.05)
    R = s_file.rhs(U)
    assert np.array_equal(R, s_arr.rhs(U))
    orc = oracle_mod.Oracle(mesh, 3, 1.4, 1.2, 1.0e5, 0.4, 10.0)
    orc.set_physics(1, 1, True, 50.0, 0.72, 8.5e4)
    Ro = orc.rhs_phys(U)
    assert T.rel_err(R, Ro, T.euler_flux_scale(U, orc.geometry()[1])) <= 1e-12


def test_physics_ns_mixed_from_gmsh(zjlib):
    """Triangles and quadrilaterals read from an MSH 4.1 file: the solver
    from the file equals the one from the arrays bit for bit and the mixed
    oracle to its bar (1e-11 of the flux scale)."""
    from oracle import mixed_oracle as MO
    from tests.test_mixed_mesh_gpu import smooth_state
    path = os.path.join(GM, "triquad_v41.msh")
    data = read_gmsh(path)
    assert set(data.elem_type.tolist()) == {0, 1}
    mesh = data.to_mixed_mesh()
    P = 3
    kw = dict(poly_order=P, compat=False, viscous=True, Re=50.0, Pr=0.72, riemann="Roe", flux_type="SD", **KW)
    s_file = FRSolver.from_gmsh(path, make_params(**kw))
    s_arr = FRSolver(mesh, make_params(bcs=[(t, n) for t, n in sorted(mesh.tag_names.items())], **kw))
    U = smooth_state(s_arr, 29)
    R = s_file.rhs(U)
    assert np.array_equal(R, s_arr.rhs(U))
    mo = MO.MixedOracle(mesh, P, 1.4, 1.2, 1.0e5, 0.4, 10.0, flux_type=1, riemann=1, viscous=True,
                        Re=50.0, Pr=0.72, T_inf=8.5e4)
    Ro = mo.rhs(U)
    m = s_arr.slot_mask()
    scale = T.euler_flux_scale(U[m], np.concatenate([mo.Ji[e] for e in range(mo.E)]))
    assert T.rel_err(R[m], Ro[m], scale) <= 1e-11
