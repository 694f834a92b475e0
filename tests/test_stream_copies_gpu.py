"""Queued host copies (zj_set_state_async / zj_get_state_async): independent
states streamed through two handles on two streams, each handle's copies
overlapping the other's steps, give exactly the states of the blocking path
(copyToDevice, advance, copyToHost) on one handle."""
import numpy as np
import pytest

from zhijian_b200 import meshgen as M
from zhijian_b200.solver import FRSolver, make_params

pytestmark = pytest.mark.gpu


def solver(mesh, precision):
    prm = make_params(poly_order=3, gamma=1.4, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3,
                      compat=False, viscous=True, riemann="Roe", flux_type="HU", Re=5000.0, Pr=0.72,
                      bcs=[(1, "slipwall")], precision=precision)
    return FRSolver(mesh, prm)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_handles_two_streams_match_blocking_path(zjlib, precision):
    import torch
    mesh = M.tgv_mesh(48, seed=3)
    ref = solver(mesh, precision)
    U0 = M.taylor_green(ref.solution_point_coords())
    dt, nsteps, nstates = 2.0e-4, 2, 6
    # independent inputs: the Taylor-Green state scaled per input
    inputs = [U0 * (1.0 + 0.01 * i) for i in range(nstates)]
    expect = []
    for U in inputs:
        ref.copyToDevice(U)
        ref.advance(dt, nsteps)
        expect.append(ref.copyToHost())
    ref.close()

    streams = [torch.cuda.Stream(), torch.cuda.Stream()]
    handles = [solver(mesh, precision), solver(mesh, precision)]
    for h, st in zip(handles, streams):
        h.set_stream(st.cuda_stream)
    hin = [torch.from_numpy(U.copy()).pin_memory().numpy() for U in inputs]
    hout = [torch.empty(U.shape, dtype=torch.float64).pin_memory().numpy() for U in inputs]
    for i in range(nstates):
        h = handles[i % 2]
        h.copyToDeviceAsync(hin[i])
        h.advance(dt, nsteps, sync=False)
        h.copyToHostAsync(hout[i])
    for h in handles:
        h.synchronize()
    for i in range(nstates):
        assert np.array_equal(hout[i], expect[i]), i
    # a queued set resets time and iteration like the blocking one
    assert handles[0].iteration == nsteps
    for h in handles:
        h.close()
