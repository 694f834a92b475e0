"""Size-independent properties on the benchmark's full workload (TGV on the
256x256 jittered mesh, P3, Navier-Stokes Re 5000, slip walls): the oracle
finishes only small meshes in seconds, so at full size the checks are what
the scheme guarantees whatever the size.

- Discrete conservation: with slip walls no mass or energy crosses the
  boundary, and every interior face's common flux enters both elements with
  opposite signs, so sum_e sum_sp w_sp J_sp R_sp vanishes for rho and rhoE to
  rounding: below tol * s_F * |domain|, s_F the parity tests' flux scale
  (max|F| max|metric|) and |domain| = sum w J (FP64: tol 1e-12; the precision
  form's FP32 arithmetic: 1e-6).
- Partitions: 4 RCB parts of the full mesh step to the whole mesh's state bit
  for bit (every part evaluates each face from the same inputs)."""
import numpy as np
import pytest

from tests import _util as T
from zhijian_b200 import meshgen as M
from zhijian_b200 import partition as PT
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu


def bench_params(precision):
    return make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                       flux_type="HU", compat=False, viscous=True, Re=5000.0, Pr=0.72,
                       bcs=[(1, "slipwall")], precision=precision)


@pytest.fixture(scope="module")
def bench_mesh():
    return M.tgv_mesh(256, seed=1)


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-6)])
def test_full_size_residual_conserves_mass_and_energy(zjlib, oracle_mod, bench_mesh, precision, tol):
    s = FRSolver(bench_mesh, bench_params(precision))
    J, Jinv = oracle_mod.Oracle(bench_mesh, 3, 1.4, 1.0, 1.0 / (1.4 * 0.09), 0.3, 0.0).geometry()
    U = M.taylor_green(s.solution_point_coords())
    s.copyToDevice(U)
    s.advance(2e-4, 3)                 # a state the scheme produced, not only the initial one
    for state in (U, s.copyToHost()):
        R = s.rhs(state)
        w1 = np.polynomial.legendre.leggauss(4)[1]
        w = np.outer(w1, w1).ravel()
        tot = np.einsum("s,es,esv->v", w, J, R)
        scale = T.euler_flux_scale(state, Jinv) * float(np.einsum("s,es->", w, J))
        assert abs(tot[0]) <= tol * scale, (tot[0], scale)
        assert abs(tot[3]) <= tol * scale, (tot[3], scale)
    s.close()


def test_full_size_partition_equals_the_whole_mesh(zjlib, bench_mesh):
    prm = bench_params("mixed")
    whole = FRSolver(bench_mesh, prm)
    U0 = M.taylor_green(whole.solution_point_coords())
    whole.copyToDevice(U0)
    whole.advance(2e-4, 3)
    parts = PT.PartitionedSolver(bench_mesh, prm, 4)
    parts.copyToDevice(U0)
    parts.advance(2e-4, 3)
    assert np.array_equal(parts.copyToHost(), whole.copyToHost())
    parts.close()
    whole.close()
