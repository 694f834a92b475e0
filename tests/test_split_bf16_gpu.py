"""The split-BF16 form (precision = split_bf16): the precision form whose
Navier-Stokes stage at P4/P5 takes its dense operator product -- the
divergence D_xi F~ + D_eta G~ and the edge traces of the transformed flux,
the reference's diff_xi / diff_eta / interp operators (basis.cpp:503-569) --
on the tensor cores (tcgen05.mma, BF16 hi/lo pairs, three products
accumulated in FP32), with the operator image staged by TMA.

Tolerances, stated per check:
* one residual against the FP64 oracle: 3e-5 of the flux scale, for P4 and
  P5, every Riemann solver, both boundary sets, on a random state (10%
  point noise) and on the Taylor-Green state of the P5 configuration.  A
  BF16 pair represents each factor to 2^-18 of itself, and the three
  products drop the lo x lo term (2^-18 again), so each product carries up
  to ~1.1e-5 relative error before the operator's row sums (measured
  maxima: 2.2e-5 on the coarse random and smooth states, 1.1e-5 on the
  Taylor-Green state; the FP32 SIMT form stays below 6e-6);
* the residual differs from the SIMT precision form's (the tensor-core
  product really ran) and the kernel's bounded waits never gave up;
* the P5 Taylor-Green configuration (512x512 jittered, Roe, Re 5000, CFL
  0.3) after 1000 SSP-RK3 steps against the FP64 path: relative L2 error
  <= 1e-6 in each of rho, rho u, rho v, rho E;
* P1-P3 (no tensor-core product at those orders) equals the mixed form bit
  for bit."""
import numpy as np
import pytest

from tests import _util as T
from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.norms import state_errors
from zhijian_b200.solver import FRSolver, make_params
from tests.test_physics_gpu import BCS_A, BCS_B, FLUX, RIEMANN, case_mesh

pytestmark = pytest.mark.gpu
TOL_RHS = 3e-5


def triple(oracle_mod, mesh, bcs, P, flux, riem, Re=50.0, rho=1.2, p=1.0e5, mach=0.4, aoa=10.0):
    kw = dict(poly_order=P, rho_inf=rho, p_inf=p, Mach=mach, AoA=aoa, flux_type=flux, riemann=riem,
              compat=False, viscous=True, Re=Re, Pr=0.72, bcs=bcs, T_inf=8.5e4)
    s = FRSolver(mesh, make_params(precision="split_bf16", **kw))
    sm = FRSolver(mesh, make_params(precision="mixed", **kw))
    tags = [(b["tag"], L.BC_TYPES[b["type"]], b.get("p_static", 0.0)) for b in bcs]
    orc = oracle_mod.Oracle(mesh, P, 1.4, rho, p, mach, aoa, tags=tags)
    orc.set_physics(FLUX.index(flux), RIEMANN.index(riem), True, Re, 0.72, 8.5e4)
    orc.set_bc_extra([(b["tag"], b.get("p_total", 0.0), b.get("T_total", 0.0), b.get("dir_x", 1.0),
                       b.get("dir_y", 0.0), b.get("T_wall", 0.0)) for b in bcs])
    return s, sm, orc


@pytest.mark.parametrize("P", [4, 5])
@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("bset", ["A", "B"])
def test_split_rhs_against_oracle(zjlib, oracle_mod, P, riem, bset):
    bcs = BCS_A if bset == "A" else BCS_B
    mesh = case_mesh(bcs, n=7)          # 49 elements: the last CTA of 8 is partly empty
    flux = FLUX[(P + RIEMANN.index(riem)) % 4]
    s, sm, orc = triple(oracle_mod, mesh, bcs, P, flux, riem)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 191 + P, 1.4, 1.2, 1.0e5, 0.1)
    R, Rm, Ro = s.rhs(U), sm.rhs(U), orc.rhs_phys(U)
    scale = T.euler_flux_scale(U, orc.geometry()[1])
    err = T.rel_err(R, Ro, scale)
    assert err <= TOL_RHS, err
    assert not np.array_equal(R, Rm)          # the tensor-core product ran
    s.check_state()                            # no bounded wait gave up
    s.copyToDevice(U)
    s.advance(1e-9, 3)
    s.check_state()


@pytest.mark.parametrize("P", [4, 5])
def test_split_rhs_on_the_taylor_green_state(zjlib, oracle_mod, P):
    """The configuration's own state: Taylor-Green on 64x64 jittered quads
    (seed 2), Roe, HU, Re 5000."""
    import os
    mesh = M.tgv_mesh(64, seed=2)
    kw = dict(poly_order=P, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe", flux_type="HU",
              compat=False, viscous=True, Re=5000.0, Pr=0.72, bcs=[(1, "slipwall")])
    s = FRSolver(mesh, make_params(precision="split_bf16", **kw))
    orc = oracle_mod.Oracle(mesh, P, 1.4, 1.0, 1.0 / (1.4 * 0.09), 0.3, 0.0, threads=os.cpu_count() or 1)
    orc.set_physics(2, 1, True, 5000.0, 0.72)
    U = M.taylor_green(s.solution_point_coords())
    err = T.rel_err(s.rhs(U), orc.rhs_phys(U), T.euler_flux_scale(U, orc.geometry()[1]))
    assert err <= TOL_RHS, err


@pytest.mark.parametrize("P", [1, 3])
def test_split_below_p4_is_the_mixed_form(zjlib, P):
    mesh = case_mesh(BCS_B)
    kw = dict(poly_order=P, rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=10.0, riemann="Roe", compat=False,
              viscous=True, Re=50.0, Pr=0.72, bcs=BCS_B)
    s = FRSolver(mesh, make_params(precision="split_bf16", **kw))
    sm = FRSolver(mesh, make_params(precision="mixed", **kw))
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 17, 1.4, 1.2, 1.0e5, 0.1)
    assert np.array_equal(s.rhs(U), sm.rhs(U))


def p5_tgv(precision, n=512):
    mesh = M.tgv_mesh(n, seed=2)
    prm = make_params(poly_order=5, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      flux_type="HU", compat=False, viscous=True, Re=5000.0, Pr=0.72, CFL=0.3,
                      bcs=[(1, "slipwall")], precision=precision)
    return FRSolver(mesh, prm)


def test_split_p5_tgv_1000_steps(zjlib):
    """The precision form's P5 Taylor-Green configuration (512x512 jittered
    quads, seed 2, Re 5000, Roe, HU, CFL 0.3) in the split-BF16 form: within
    1e-6 relative L2 of the FP64 path per variable after 1000 steps."""
    s64, sb = p5_tgv("fp64"), p5_tgv("split_bf16")
    U0 = M.taylor_green(s64.solution_point_coords())
    s64.copyToDevice(U0)
    dt = s64.computeTimeStep()
    for s in (s64, sb):
        s.copyToDevice(U0)
        s.advance(dt, 1000)
    sb.check_state()
    e = state_errors(sb.copyToHost(), s64.copyToHost())
    print("split_bf16 P5 vs fp64 after 1000 steps:", e)
    assert max(e["l2"]) <= 1e-6, e
