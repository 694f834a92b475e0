"""The mixed-precision form (precision = mixed: FP32 volume, face, gradient
and operator work; FP64 state, SSP-RK3 accumulation and norm reductions)
against the FP64 oracle and the FP64 GPU path.

Tolerances, stated per check:
* one residual on a random state: 1e-5 of the flux scale (the parity metric of
  the FP64 tests, whose bar is 1e-12) -- FP32 rounding of the fluxes
  (2^-24 relative) amplified by the operator row sums;
* the Taylor-Green configuration of the benchmark (256x256 jittered, P3, Roe)
  after 1000 SSP-RK3 steps against the FP64 path (which matches the FP64
  oracle to 1e-12 per residual, test_physics_gpu.py): relative L2 error
  <= 1e-6 in each of rho, rho u, rho v, rho E for the inviscid case; for
  Navier-Stokes (Re 5000) see test_mixed_tgv_ns_1000_steps."""
import numpy as np
import pytest

from tests import _util as T
from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.norms import state_errors
from zhijian_b200.solver import FRSolver, make_params
from tests.test_physics_gpu import BCS_A, BCS_B, FLUX, RIEMANN, case_mesh

pytestmark = pytest.mark.gpu
TOL_RHS = 1e-5


def pair(oracle_mod, mesh, bcs, P, flux, riem, viscous, Re=50.0, rho=1.2, p=1.0e5, mach=0.4,
         aoa=10.0):
    kw = dict(poly_order=P, rho_inf=rho, p_inf=p, Mach=mach, AoA=aoa, flux_type=flux, riemann=riem,
              compat=False, viscous=viscous, Re=Re, Pr=0.72, bcs=bcs, T_inf=8.5e4)
    s = FRSolver(mesh, make_params(precision="mixed", **kw))
    tags = [(b["tag"], L.BC_TYPES[b["type"]], b.get("p_static", 0.0)) for b in bcs]
    orc = oracle_mod.Oracle(mesh, P, 1.4, rho, p, mach, aoa, tags=tags)
    orc.set_physics(FLUX.index(flux), RIEMANN.index(riem), viscous, Re, 0.72, 8.5e4)
    orc.set_bc_extra([(b["tag"], b.get("p_total", 0.0), b.get("T_total", 0.0), b.get("dir_x", 1.0),
                       b.get("dir_y", 0.0), b.get("T_wall", 0.0)) for b in bcs])
    return s, orc


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("viscous", [False, True], ids=["euler", "ns"])
def test_mixed_rhs_against_oracle(zjlib, oracle_mod, P, riem, viscous):
    bcs = BCS_A if (P + RIEMANN.index(riem)) % 2 else BCS_B
    mesh = case_mesh(bcs)
    flux = FLUX[(P + RIEMANN.index(riem)) % 4]
    s, orc = pair(oracle_mod, mesh, bcs, P, flux, riem, viscous)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 91 + P, 1.4, 1.2, 1.0e5, 0.1)
    R = s.rhs(U)
    Ro = orc.rhs_phys(U)
    err = T.rel_err(R, Ro, T.euler_flux_scale(U, orc.geometry()[1]))
    assert err <= TOL_RHS, err
    assert err > 0.0          # the FP32 arithmetic really ran


def tgv_solver(precision, viscous=True, n=256):
    mesh = M.tgv_mesh(n, seed=1)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      compat=False, viscous=viscous, Re=5000.0, Pr=0.72, bcs=[(1, "slipwall")],
                      precision=precision)
    return FRSolver(mesh, prm)


def run_pair(viscous, steps=1000):
    s64, s32 = tgv_solver("fp64", viscous), tgv_solver("mixed", viscous)
    U0 = M.taylor_green(s64.solution_point_coords())
    s64.copyToDevice(U0)
    dt = s64.computeTimeStep()
    for s in (s64, s32):
        s.copyToDevice(U0)
        s.advance(dt, steps)
    return s64, s32, U0, dt


def test_mixed_tgv_euler_1000_steps(zjlib):
    """Inviscid Taylor-Green case, 1000 SSP-RK3 steps at CFL 0.5 in both
    precisions: relative L2 error <= 1e-6 in rho, rho u, rho v, rho E."""
    s64, s32, _, _ = run_pair(False)
    e = state_errors(s32.copyToHost(), s64.copyToHost())
    print("euler mixed vs fp64 after 1000 steps:", e)
    assert max(e["l2"]) <= 1e-6, e


def test_mixed_tgv_ns_1000_steps(zjlib):
    """The Navier-Stokes case of the benchmark (Re 5000), 1000 steps at CFL 0.5:
    the precision form within 1e-6 relative L2 of the FP64 path per variable,
    in the whole domain and in the interior (20 or more elements from every
    wall).  The FP64 run from the initial state rounded once to FP32 (the
    conditioning floor) is printed beside it: with the walls' Neumann data on
    the common viscous flux the scheme no longer amplifies perturbations at
    the slip-walled corners, and the floor sits at the rounding level."""
    s64, s32, U0, dt = run_pair(True)
    U64, U32 = s64.copyToHost(), s32.copyToHost()
    e = state_errors(U32, U64)
    sr = tgv_solver("fp64", True)
    sr.copyToDevice(U0.astype(np.float32).astype(np.float64))
    sr.advance(dt, 1000)
    floor = state_errors(sr.copyToHost(), U64)
    print("ns mixed vs fp64:", e)
    print("ns fp64 from the FP32-rounded initial state vs fp64:", floor)
    assert np.all(np.isfinite(U32))
    assert max(e["l2"]) <= 1e-6, e
    assert max(floor["l2"]) <= 1e-7, floor
    n = 256
    i = np.arange(n)
    d = np.minimum(i, n - 1 - i)
    interior = np.minimum(d[:, None], d[None, :]) >= 20
    inner = state_errors(U32.reshape(n, n, -1, 4)[interior], U64.reshape(n, n, -1, 4)[interior])
    assert max(inner["l2"]) <= 1e-6, inner
    # the residual norms of the last step agree to the FP32 residual's own
    # rounding (up to ~1e-3 of the flux scale per point)
    n64, n32 = s64.computeResidual(), s32.computeResidual()
    assert abs(n32 - n64) <= 5e-4 * n64
