"""Step graphs (zj_set_step_graphs): zj_step replays blocks of six steps from
CUDA graphs captured at first use.  The states, time, iteration and residual
norm equal those of plain launches bit for bit, for every kind of handle and
from every starting phase of the rotating buffers; inside a graph the caller
is capturing, the steps are launched plainly and become part of it."""
import numpy as np
import pytest

from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu
TGV = dict(rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, bcs=[(1, "slipwall")])


def cases():
    tgv = M.tgv_mesh(32, seed=1)
    ns = dict(compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72, **TGV)
    q = M.structured_quads(16, 16, 0.0, 1.0, 0.0, 1.0, 0.1, 3, (1, 1, 1, 1), {1: "slipwall"})
    return {
        "ns_fp64": (tgv, make_params(poly_order=3, **ns)),
        "ns_mixed": (tgv, make_params(poly_order=3, precision="mixed", **ns)),
        "compat": (tgv, make_params(poly_order=3, riemann="Rusanov", flux_type="HU", **TGV)),
        "mixed_mesh_ns": (M.split_quads(q, 0.4, 5),
                          make_params(poly_order=3, compat=False, viscous=True, riemann="HLLC", flux_type="GA",
                                      Re=2000.0, Pr=0.72, **TGV)),
    }


@pytest.mark.parametrize("name", ["ns_fp64", "ns_mixed", "compat", "mixed_mesh_ns"])
def test_graph_steps_equal_plain_steps(zjlib, name):
    mesh, prm = cases()[name]
    runs = []
    for graphs in (True, False):
        s = FRSolver(mesh, prm)
        s.set_step_graphs(graphs)
        s.setInitialCondition(M.taylor_green)
        dt = 0.2 * s.computeTimeStep()
        out = []
        for n in (20, 13, 7):                 # each call starts at another buffer phase
            s.advance(dt, n)
            out.append((s.copyToHost(), s.time, s.iteration, s.computeResidual()))
        s.close()
        runs.append(out)
    for (Ua, ta, ia, ra), (Ub, tb, ib, rb) in zip(*runs):
        assert np.array_equal(Ua, Ub)
        assert ta == tb and ia == ib and ra == rb
    assert runs[0][-1][2] == 40


def test_steps_inside_a_caller_graph(zjlib):
    """The caller captures zj_step into its own graph (PyTorch here): the
    library launches plainly into the capture, and one replay equals the same
    steps run directly."""
    import torch
    mesh, prm = cases()["ns_mixed"]
    U0 = None
    res = []
    for captured in (True, False):
        s = FRSolver(mesh, prm)
        st = torch.cuda.Stream()
        s.set_stream(st.cuda_stream)
        if U0 is None:
            U0 = M.taylor_green(s.solution_point_coords())
        s.copyToDevice(U0)
        dt = 0.2 * s.computeTimeStep()
        s.advance(dt, 1)                       # dt on the device, traces valid
        if captured:
            g = torch.cuda.CUDAGraph()
            with torch.cuda.graph(g, stream=st):
                s.advance(dt, 7, sync=False)
            g.replay()
            torch.cuda.synchronize()
        else:
            s.advance(dt, 7)
        res.append(s.copyToHost())
        s.close()
    assert np.array_equal(res[0], res[1])


def test_legacy_default_stream_steps_plainly(zjlib):
    """On the legacy default stream (not capturable) zj_step launches
    directly; the result equals the graphs-off handle's."""
    mesh, prm = cases()["ns_fp64"]
    res = []
    for legacy in (True, False):
        s = FRSolver(mesh, prm)
        if legacy:
            s.set_stream(0)
        else:
            s.set_step_graphs(False)
        s.setInitialCondition(M.taylor_green)
        dt = 0.2 * s.computeTimeStep()
        s.advance(dt, 14)
        res.append((s.copyToHost(), s.iteration))
        s.close()
    assert np.array_equal(res[0][0], res[1][0]) and res[0][1] == res[1][1] == 14
