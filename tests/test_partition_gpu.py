"""Partitioned meshes on the GPU: the parts of a mesh as handles driven
together by zj_parts_rhs / zj_parts_step (their cut faces' traces and
gradient traces copied into each other's ghost rows after every launch that
writes them), on one device here -- the same driver moves the rows with peer
copies when the parts sit on different GPUs.  Every part evaluates each face
from the same inputs with the same orientation as the whole-mesh handle, so
residuals and steps equal the whole mesh's bit for bit; the residual norm sums
the parts' partial sums in another order (within 1e-13)."""
import ctypes as C

import numpy as np
import pytest

from zhijian_b200 import _lib as L
from zhijian_b200 import meshgen as M
from zhijian_b200 import partition as PT
from zhijian_b200.solver import FRSolver, make_params
from tests.test_physics_gpu import BCS_A, BCS_B

pytestmark = pytest.mark.gpu
KW = dict(rho_inf=1.2, p_inf=1.0e5, Mach=0.4, AoA=10.0, T_inf=8.5e4)


def mesh_of(kind, bcs):
    names = {b["tag"]: b["type"] for b in bcs}
    if kind == "curved":
        return M.curved_quads(7, 6, 2, 0.0, 1.0, 0.0, 1.0, 0.04, (1, 2, 3, 4), names)
    return M.structured_quads(9, 7, 0.0, 1.0, 0.0, 1.0, 0.15, 5, (1, 2, 3, 4), names)


@pytest.mark.parametrize("nparts", [2, 3])
@pytest.mark.parametrize("kind", ["jittered", "curved"])
@pytest.mark.parametrize("viscous,precision", [(False, "fp64"), (True, "fp64"), (True, "mixed")])
def test_parts_rhs_equals_whole_mesh(zjlib, nparts, kind, viscous, precision):
    bcs = BCS_A if nparts == 2 else BCS_B
    mesh = mesh_of(kind, bcs)
    P = 3 if kind == "jittered" else 4
    prm = make_params(poly_order=P, riemann="Roe", flux_type="HU", compat=False, viscous=viscous, Re=50.0,
                      Pr=0.72, bcs=bcs, precision=precision, **KW)
    whole = FRSolver(mesh, prm)
    parts = PT.PartitionedSolver(mesh, prm, nparts)
    assert np.array_equal(parts.solution_point_coords(), whole.solution_point_coords())
    U = M.random_state(mesh.n_elem, (P + 1) ** 2, 71, 1.4, 1.2, 1.0e5, 0.05)
    assert np.array_equal(parts.rhs(U), whole.rhs(U))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_parts_steps_equal_whole_mesh(zjlib, precision):
    mesh = M.tgv_mesh(24, seed=1)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      compat=False, viscous=True, Re=5000.0, Pr=0.72, bcs=[(1, "slipwall")], precision=precision)
    whole = FRSolver(mesh, prm)
    parts = PT.PartitionedSolver(mesh, prm, 4)
    U0 = M.taylor_green(whole.solution_point_coords())
    whole.copyToDevice(U0)
    parts.copyToDevice(U0)
    dt = whole.computeTimeStep()
    assert parts.computeTimeStep() == dt
    whole.advance(dt, 7)
    parts.advance(dt, 7)
    assert np.array_equal(parts.copyToHost(), whole.copyToHost())
    nw, npart = whole.computeResidual(), parts.computeResidual()
    assert abs(nw - npart) <= 1e-13 * nw


def test_a_part_refuses_single_handle_stepping(zjlib):
    mesh = M.tgv_mesh(8, seed=1)
    prm = make_params(poly_order=2, compat=False, bcs=[(1, "slipwall")], **KW)
    parts = PT.PartitionedSolver(mesh, prm, 2)
    assert zjlib.zj_step(parts.parts[0].h, 1e-6, 1) == L.ERR_UNSUPPORTED
    one = (C.c_void_p * 1)(parts.parts[0].h)
    assert zjlib.zj_parts_step(one, 1, 1e-6, 1) == L.ERR_ARG       # a 2-part partition needs both parts
    with pytest.raises(L.ZJError) as e:
        PT.PartitionedSolver(mesh, make_params(poly_order=2, compat=True, bcs=[(1, "slipwall")], **KW), 2)
    assert e.value.code == L.ERR_UNSUPPORTED


def test_parts_step_graphs_match_plain_launches(zjlib):
    """The step graphs of a one-device partition replay exactly what the plain
    launches do (graphs off through the rank-0 part)."""
    mesh = M.tgv_mesh(16, seed=3)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="HLLC",
                      compat=False, viscous=True, Re=2000.0, Pr=0.72, bcs=[(1, "slipwall")], precision="mixed")
    runs = []
    for graphs in (True, False):
        parts = PT.PartitionedSolver(mesh, prm, 3)
        if not graphs:
            assert zjlib.zj_set_step_graphs(parts.parts[0].h, 0) == L.OK
        parts.copyToDevice(M.taylor_green(parts.solution_point_coords()))
        parts.advance(1e-4, 2)
        parts.advance(1e-4, 9)      # every buffer phase, graphs captured after the first call
        runs.append((parts.copyToHost(), parts.computeResidual()))
        parts.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]


def test_device_arrays_must_be_32_byte_aligned(zjlib):
    import torch
    mesh = M.tgv_mesh(8, seed=1)
    s = FRSolver(mesh, make_params(poly_order=2, compat=False, bcs=[(1, "slipwall")], **KW))
    n = s.n_elem * s.n_sp * 4
    buf = torch.zeros(2 * n + 8, dtype=torch.float64, device="cuda")
    base = buf.data_ptr()
    assert base % 256 == 0
    U, R = base, base + 8 * (n + 4)          # both 32-byte aligned
    assert zjlib.zj_rhs(s.h, C.c_void_p(U), C.c_void_p(R)) == L.OK
    for off in (8, 16):                          # 8- and 16-byte aligned: refused before any launch
        assert zjlib.zj_rhs(s.h, C.c_void_p(U + off), C.c_void_p(R)) == L.ERR_ARG
        assert zjlib.zj_rhs(s.h, C.c_void_p(U), C.c_void_p(R + off)) == L.ERR_ARG
    torch.cuda.synchronize()
    s.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_one_part_per_thread_with_a_caller_transport(zjlib, precision):
    """zj_part_step: each part stepped alone by its own host thread, its cut-face
    rows moved by the caller's transport (LocalExchange: one process, one
    device; nccl_exchange is the same contract over torch.distributed), equals
    the whole mesh bit for bit."""
    import threading
    mesh = M.tgv_mesh(16, seed=5)
    prm = make_params(poly_order=3, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Roe",
                      compat=False, viscous=True, Re=3000.0, Pr=0.72, bcs=[(1, "slipwall")], precision=precision)
    whole = FRSolver(mesh, prm)
    U0 = M.taylor_green(whole.solution_point_coords())
    whole.copyToDevice(U0)
    dt = whole.computeTimeStep()
    whole.advance(dt, 5)
    part = PT.partition(mesh, 3)
    procs = [PT.PartProcess(mesh, prm, part, r) for r in range(3)]
    xchg = PT.LocalExchange([p.plan for p in procs])
    for p in procs:
        p.copyToDevice(U0)
    errors = []

    def run(r):
        try:
            procs[r].advance(dt, 2, xchg.for_rank(r))
            procs[r].advance(dt, 3, xchg.for_rank(r))
        except Exception as e:
            errors.append(e)
    threads = [threading.Thread(target=run, args=(r,)) for r in range(3)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    out = np.empty_like(U0)
    for p in procs:
        out[p.elems] = p.copyToHost()
    assert np.array_equal(out, whole.copyToHost())
    norms = [p.solver.computeResidual() for p in procs]
    assert abs(np.sqrt(sum(n * n for n in norms)) - whole.computeResidual()) <= 1e-13 * whole.computeResidual()
    for p in procs:
        p.close()


def test_part_step_reports_a_failed_transport(zjlib):
    mesh = M.tgv_mesh(8, seed=1)
    prm = make_params(poly_order=2, compat=False, bcs=[(1, "slipwall")], **KW)
    part = PT.partition(mesh, 2)
    p = PT.PartProcess(mesh, prm, part, 0)
    p.copyToDevice(M.random_state(mesh.n_elem, 9, 3, 1.4, 1.2, 1.0e5, 0.05))
    with pytest.raises(RuntimeError):
        p.advance(1e-6, 1, lambda *args: (_ for _ in ()).throw(RuntimeError("link down")))
    failing = L.EXCHANGE_FN(lambda *args: 3)
    assert zjlib.zj_part_step(p.solver.h, 1e-6, 1, failing, None) == L.ERR_IO
    p.close()


def test_a_one_part_partition_is_the_whole_mesh(zjlib):
    """No cut faces: every exchange moves zero rows, through both drivers."""
    mesh = M.tgv_mesh(12, seed=2)
    prm = make_params(poly_order=2, rho_inf=1.0, p_inf=1.0 / (1.4 * 0.09), Mach=0.3, riemann="Rusanov",
                      compat=False, viscous=True, Re=1000.0, Pr=0.72, bcs=[(1, "slipwall")])
    whole = FRSolver(mesh, prm)
    U0 = M.taylor_green(whole.solution_point_coords())
    whole.copyToDevice(U0)
    whole.advance(1e-4, 4)
    parts = PT.PartitionedSolver(mesh, prm, 1)
    parts.copyToDevice(U0)
    parts.advance(1e-4, 4)
    assert np.array_equal(parts.copyToHost(), whole.copyToHost())
    parts.close()
    one = PT.PartProcess(mesh, prm, np.zeros(mesh.n_elem, dtype=np.int32), 0)
    one.copyToDevice(U0)
    calls = []
    one.advance(1e-4, 4, lambda kind, row_bytes, send, recv, stream: calls.append((kind, row_bytes)) or 0)
    assert np.array_equal(one.copyToHost(), whole.copyToHost())
    # the state traces once, then per stage the gradient traces and the new traces
    assert calls[0] == (L.XCHG_TRACES, 3 * 4 * 8) and len(calls) == 1 + 4 * 3 * 2
    one.close()
