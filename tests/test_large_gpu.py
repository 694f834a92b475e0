"""Maximum sizes: a 2048x2048 jittered quad mesh at P3 (4 194 304 elements,
67 M solution points, 2.1 GB per state array; grids of 262 144 CTAs), far
field all round, a uniform free stream.  Size-independent properties: the
FP64 residual vanishes to rounding and three SSP-RK3 steps leave the state
where it was; the precision form's residual vanishes to FP32 rounding."""
import math

import numpy as np
import pytest

from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu
N = 2048
RHO, P_INF, MACH, AOA = 1.2, 1.0e5, 0.4, 25.0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_free_stream_on_a_4m_element_mesh(zjlib, precision):
    mesh = M.structured_quads(N, N, 0.0, 1.0, 0.0, 1.0, 0.15, 7, (1, 1, 1, 1), {1: "farfield"})
    prm = make_params(poly_order=3, rho_inf=RHO, p_inf=P_INF, Mach=MACH, AoA=AOA, riemann="Roe",
                      flux_type="HU", compat=False, bcs=[(1, "farfield")], precision=precision)
    s = FRSolver(mesh, prm)
    assert s.n_elem == N * N
    c = math.sqrt(1.4 * P_INF / RHO)
    q = M.prim_to_cons(RHO, MACH * c * math.cos(math.radians(AOA)), MACH * c * math.sin(math.radians(AOA)),
                       P_INF, 1.4)
    U = np.broadcast_to(q, s.shape).copy()
    R = s.rhs(U)
    # flux scale of the free stream times the largest metric term (h = 1/2048)
    scale = (P_INF + q[3]) * c * 2.0 * N
    bar = 1e-10 if precision == "fp64" else 1e-5
    assert np.isfinite(R).all()
    assert np.abs(R).max() <= bar * scale, np.abs(R).max() / scale
    if precision == "fp64":
        s.copyToDevice(U)
        s.advance(s.computeTimeStep(), 3)
        s.check_state()
        V = s.copyToHost()
        assert np.abs(V - U).max() <= 1e-12 * np.abs(U).max()
    s.close()
