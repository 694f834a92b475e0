"""The allocation-free residual, zj_rhs_noalloc.

It exists for callers that may not allocate device memory at the point where
they need a residual -- a host application whose device memory is reserved up
front by its own allocator, or a time-critical loop that must not hit the
implicit synchronisation of cudaMalloc/cudaFree.  Its scratch lives in one
static device array inside the library that every call shares and that keeps
the previous call's contents, so the check runs two calls in a row, each
against the allocating entry point zj_rhs on the same state, through the
C-ABI.  This file is collected last so a failure here cannot hide the rest of
the suite, and it needs nothing the other tests set up.
"""
import ctypes as C

import numpy as np
import pytest

from tests import _util as T
from tests.golden import make_golden as G
from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu
TOL = 1e-12   # the parity bar of the residual tests


def _solver(case):
    rho, p, mach, aoa = case["prm"]
    prm = make_params(poly_order=case["P"], gamma=G.GAMMA, rho_inf=rho, p_inf=p, Mach=mach,
                      AoA=aoa, bcs=case["tags"])
    return FRSolver(case["mesh"], prm)


def _run(lib, fn, s, U):
    import torch
    Ud = torch.from_numpy(U).cuda()
    Rd = torch.full_like(Ud, float("nan"))
    torch.cuda.synchronize()
    L.check(fn(s.h, C.c_void_p(Ud.data_ptr()), C.c_void_p(Rd.data_ptr())), s.h)
    L.check(lib.zj_synchronize(s.h), s.h)
    return Rd.cpu().numpy()


def test_noalloc_matches_rhs_on_two_calls_in_a_row(zjlib):
    case = G.case_defs()["mixed_p3"]
    s = _solver(case)
    xy = s.solution_point_coords()
    states = [G.make_state(case, xy),
              M.random_state(s.n_elem, s.n_sp, 99, G.GAMMA, 1.2, 1.0e5, 0.1)]
    for U in states:
        ref = _run(zjlib, zjlib.zj_rhs, s, U)
        got = _run(zjlib, zjlib.zj_rhs_noalloc, s, U)
        scale = T.euler_flux_scale(U, None) * T.metric_scale(case["mesh"], case["P"])
        assert np.isfinite(got).all()
        assert T.rel_err(got, ref, scale) <= TOL
    s.close()


def _physics(mesh, precision):
    """Navier-Stokes in physics mode (Roe, HU, slip walls, Re 5000) at P3."""
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      flux_type="HU", compat=False, viscous=True, Re=5000.0, Pr=0.72,
                      bcs=[(1, "slipwall")], precision=precision)
    return FRSolver(mesh, prm)


def _tgv_states(s):
    U = M.taylor_green(s.solution_point_coords())
    r = M.uniform01(123, U.size).reshape(U.shape)
    return [U, U * (1.0 + 1.0e-3 * (2.0 * r - 1.0))]


# The Navier-Stokes branches keep the gradient traces in the same scratch
# (three trace blocks), the precision form FP32 traces with the FP64 partial
# sums behind them, and a mesh of quads and triangles the triangles' partial
# sums after the quads'.  Bars: the FP64 parity bar, and the precision form's
# 1e-5 of the flux scale.
NS_CASES = [("quads", "fp64", TOL), ("quads", "mixed", 1e-5),
            ("quads+triangles", "fp64", TOL), ("quads+triangles", "mixed", 1e-5)]


@pytest.mark.parametrize("kind,precision,tol", NS_CASES)
def test_noalloc_navier_stokes_matches_rhs_on_two_calls_in_a_row(zjlib, kind, precision, tol):
    mesh = M.tgv_mesh(32, seed=1)
    if kind != "quads":
        mesh = M.split_quads(mesh, 0.3, 3)
    s = _physics(mesh, precision)
    used = s.slot_mask()   # a triangle fills (P+1)(P+2)/2 of its (P+1)^2 slots
    for U in _tgv_states(s):
        ref = _run(zjlib, zjlib.zj_rhs, s, U)[used]
        got = _run(zjlib, zjlib.zj_rhs_noalloc, s, U)[used]
        assert np.isfinite(got).all()
        # flux scale x the metric 2/h of elements of side h = pi/32
        assert T.rel_err(got, ref, T.euler_flux_scale(U) * 64.0 / np.pi) <= tol
    s.close()


def test_noalloc_rejects_a_mesh_beyond_its_scratch(zjlib):
    # P5 traces take 768 bytes per element: 210 x 210 elements need ~34 MB.
    mesh = M.tgv_mesh(210, seed=2)
    s = FRSolver(mesh, make_params(poly_order=5, rho_inf=1.0, p_inf=10.0, bcs=[(1, "slipwall")]))
    import torch
    U = torch.zeros(s.n_elem * s.n_sp * 4, dtype=torch.float64, device="cuda")
    R = torch.zeros_like(U)
    code = zjlib.zj_rhs_noalloc(s.h, C.c_void_p(U.data_ptr()), C.c_void_p(R.data_ptr()))
    assert code == L.ERR_ARG
    assert b"static limit" in zjlib.zj_last_error(s.h)
    s.close()
