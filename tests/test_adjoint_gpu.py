"""Differentiation of the physics-mode residual and stepper (FP64):
Jacobian-vector products (dual numbers) against central finite differences,
the hand-written vector-Jacobian products against the JVP (dot-product
test), the adjoint of one SSP-RK3 step against finite differences, and the
checkpointed discrete adjoint of the Taylor-Green configuration (128x128
jittered, P3, Roe, Re 5000, 200 steps, checkpoints every 20 steps) against
central differences with h = 1e-6 on 64 seeded directions, plus dJ/dRe and
dJ/dMach.

Tolerances: dot test 1e-11 relative (both sides exact to rounding); JVP vs
FD 1e-6 relative (h = 1e-6 relative steps, O(h^2) truncation); discrete
adjoint vs FD 1e-6 relative per direction."""
import math

import numpy as np
import pytest
import torch

from tests.test_physics_gpu import BCS_A, BCS_B, FLUX, RIEMANN, case_mesh
from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200.objectives import kinetic_energy, quadrature_weights
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu


def dev(x):
    return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def small_solver(P, riem, bcs, viscous, Re=50.0, flux=None):
    mesh = case_mesh(bcs)
    prm = make_params(poly_order=P, rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=10.0,
                      flux_type=flux or FLUX[P % 4], riemann=riem, compat=False, viscous=viscous,
                      Re=Re, Pr=0.72, bcs=bcs, T_inf=8.5e4)
    return FRSolver(mesh, prm), mesh


def seeded(shape, seed):
    return (M.uniform01(seed, int(np.prod(shape))).reshape(shape) * 2.0 - 1.0)


@pytest.mark.parametrize("P", [1, 2, 3, 4, 5])
@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("viscous", [False, True], ids=["euler", "ns"])
def test_dot_product_vjp_jvp(zjlib, P, riem, viscous):
    bcs = BCS_A if (P + RIEMANN.index(riem)) % 2 else BCS_B
    s, mesh = small_solver(P, riem, bcs, viscous)
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 131 + P, 1.4, 1.2, 1.0e5, 0.1)
    V = seeded(U.shape, 7 + P) * np.abs(U)
    Lm = seeded(U.shape, 11 + P)
    Ud, Vd, Ld = dev(U), dev(V), dev(Lm)
    JV, W = torch.empty_like(Ud), torch.empty_like(Ud)
    s.rhs_jvp(Ud.data_ptr(), Vd.data_ptr(), JV.data_ptr())
    s.rhs_vjp(Ud.data_ptr(), Ld.data_ptr(), W.data_ptr())
    a = float(np.sum(Lm * host(JV)))
    b = float(np.sum(host(W) * V))
    scale = float(np.sum(np.abs(Lm * host(JV))))
    assert abs(a - b) <= 1e-11 * scale, (a, b)


@pytest.mark.parametrize("riem", RIEMANN)
@pytest.mark.parametrize("viscous", [False, True], ids=["euler", "ns"])
def test_jvp_against_central_differences(zjlib, riem, viscous):
    s, mesh = small_solver(3, riem, BCS_A, viscous)
    U = M.random_state(mesh.n_elem, 16, 211, 1.4, 1.2, 1.0e5, 0.05)
    V = seeded(U.shape, 17) * np.abs(U)
    h = 1e-6
    fd = (s.rhs(U + h * V) - s.rhs(U - h * V)) / (2 * h)
    JV = torch.empty(U.shape, dtype=torch.float64, device="cuda")
    R = torch.empty_like(JV)
    Ud, Vd, Z = dev(U), dev(V), dev(np.zeros_like(U))   # kept alive across the calls
    s.rhs_jvp(Ud.data_ptr(), Vd.data_ptr(), JV.data_ptr(), R.data_ptr())
    jv = host(JV)
    assert np.abs(host(R) - s.rhs(U)).max() <= 1e-12 * np.abs(s.rhs(U)).max()
    assert np.linalg.norm(jv - fd) <= 1e-6 * np.linalg.norm(jv)
    if viscous:
        # the Reynolds-number tangent
        Re, hr = 50.0, 1e-6 * 50.0
        sp, _ = small_solver(3, riem, BCS_A, True, Re=Re + hr)
        sm, _ = small_solver(3, riem, BCS_A, True, Re=Re - hr)
        fdr = (sp.rhs(U) - sm.rhs(U)) / (2 * hr)
        s.rhs_jvp(Ud.data_ptr(), Z.data_ptr(), JV.data_ptr(), dRe=1.0)
        jr = host(JV)
        assert np.linalg.norm(jr - fdr) <= 1e-6 * np.linalg.norm(jr)
        # the VJP's L . dR/dRe against the JVP's
        Lm = seeded(U.shape, 41)
        Ld, W = dev(Lm), torch.empty_like(JV)
        dre = s.rhs_vjp(Ud.data_ptr(), Ld.data_ptr(), W.data_ptr(), with_re=True)
        ref = float(np.sum(Lm * jr))
        assert abs(dre - ref) <= 1e-11 * float(np.sum(np.abs(Lm * jr))), (dre, ref)


def test_step_vjp_against_central_differences(zjlib):
    s, mesh = small_solver(3, "Roe", BCS_A, True, Re=20.0)
    U = M.random_state(mesh.n_elem, 16, 311, 1.4, 1.2, 1.0e5, 0.02)
    V = seeded(U.shape, 23) * np.abs(U)
    B = seeded(U.shape, 29)
    dt = 2e-8
    A = torch.empty(U.shape, dtype=torch.float64, device="cuda")
    Ud, Bd = dev(U), dev(B)
    s.step_vjp(Ud.data_ptr(), dt, Bd.data_ptr(), A.data_ptr())
    lhs = float(np.sum(host(A) * V))

    def step(X):
        s.copyToDevice(X)
        s.advance(dt, 1)
        return s.copyToHost()
    h = 1e-6
    rhs = float(np.sum(B * (step(U + h * V) - step(U - h * V)) / (2 * h)))
    assert abs(lhs - rhs) <= 1e-6 * abs(rhs), (lhs, rhs)


def directions(shape, count, seed=5, modes=4):
    """count smooth seeded directions: per variable, sin-mode combinations on
    the element-centre grid with SplitMix64 coefficients (seed + index)."""
    n = int(round(math.sqrt(shape[0])))
    out = []
    for d in range(count):
        c = M.uniform01(seed + d, 4 * modes * modes).reshape(4, modes, modes) * 2.0 - 1.0
        ii, jj = np.meshgrid(np.arange(n), np.arange(n))
        x = (ii.ravel() + 0.5) / n * math.pi
        y = (jj.ravel() + 0.5) / n * math.pi
        V = np.zeros(shape)
        for v in range(4):
            f = np.zeros(n * n)
            for a in range(modes):
                for b in range(modes):
                    f += c[v, a, b] * np.sin((a + 1) * x) * np.sin((b + 1) * y)
            V[..., v] = f[:, None]
        out.append(V)
    return out


def tgv_c5(mach=0.3, Re=5000.0):
    mesh = M.tgv_mesh(128, seed=4)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * mach * mach), Mach=mach,
                      riemann="Roe", compat=False, viscous=True, Re=Re, Pr=0.72, bcs=[(1, "slipwall")])
    return FRSolver(mesh, prm), mesh


def test_discrete_adjoint_tgv_128(zjlib):
    steps, k = 200, 20
    s, mesh = tgv_c5()
    xy = s.solution_point_coords()
    U0 = M.taylor_green(xy)
    s.copyToDevice(U0)
    dt = s.computeTimeStep()
    wq = quadrature_weights(mesh, 3)

    def J_of(solver, U):
        solver.copyToDevice(U)
        solver.advance(dt, steps)
        return kinetic_energy(solver.copyToHost(), wq)

    J0, Gf = J_of(s, U0)
    s.copyToDevice(U0)
    G = dev(Gf)
    info = s.adjoint_run(dt, steps, k, G.data_ptr())
    g = host(G)
    assert np.allclose(s.copyToHost(), U0, rtol=0, atol=0)   # state left unchanged
    h = 1e-6
    worst = 0.0
    for V in directions(U0.shape, 64):
        V = V * np.abs(U0).max(axis=(0, 1))     # per-variable scale
        fd = (J_of(s, U0 + h * V)[0] - J_of(s, U0 - h * V)[0]) / (2 * h)
        ad = float(np.sum(g * V))
        worst = max(worst, abs(ad - fd) / abs(fd))
    print("adjoint vs FD, worst relative error over 64 directions:", worst, info)
    assert worst <= 1e-6
    # dJ/dRe against central differences in Re
    Re, hr = 5000.0, 1e-6 * 5000.0
    fdr = (J_of(tgv_c5(Re=Re + hr)[0], U0)[0] - J_of(tgv_c5(Re=Re - hr)[0], U0)[0]) / (2 * hr)
    assert abs(info["dRe"] - fdr) <= 1e-6 * abs(fdr), (info["dRe"], fdr)
    # dJ/dMach through the initial pressure p0 = 1/(gamma M^2) + ...
    dM = 1e-6 * 0.3
    Up = M.taylor_green(xy, mach=0.3 + dM)
    Um = M.taylor_green(xy, mach=0.3 - dM)
    dU0 = (Up - Um) / (2 * dM)
    fdm = (J_of(s, Up)[0] - J_of(s, Um)[0]) / (2 * dM)
    adm = float(np.sum(g * dU0))
    assert abs(adm - fdm) <= 1e-6 * abs(fdm), (adm, fdm)
